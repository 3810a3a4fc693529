"""Block Gauss-Seidel smoother (multigrid/BlockGaussseidelSmoother.java) on
the GPU against the numpy oracle (oracle/block_gs.py): an FE system cut into
three blocks, and a saddle-point system whose zero diagonal block is
replaced by the identity as BlockSparseMatrix.getInvertedDiagonalMatrix does."""
import numpy as np
import pytest

from oracle.block_gs import block_gauss_seidel
from fixtures import coo_oracle, fe_system
from jfem_b200.schur import BlockGaussSeidelSmoother, BlockSparseMatrix

pytestmark = pytest.mark.gpu


def split(D, cuts):
    starts, ends = list(cuts[:-1]), list(cuts[1:])
    dense, keyed = {}, {}
    for i, (a, b) in enumerate(zip(starts, ends)):
        for j, (c, d) in enumerate(zip(starts, ends)):
            blk = D[a:b, c:d]
            if np.any(blk) or i == j:
                dense[(i, j)] = blk.copy()
                keyed[(a, c)] = blk.copy()
    return dense, keyed, starts, ends


@pytest.mark.parametrize("p,cells", [(1, 12), (2, 6)])
def test_block_gs_matches_oracle(ctx, p, cells):
    sp, sy = fe_system(p, cells)
    D = coo_oracle(sy).dense()
    n = sy.n
    dense, keyed, st, en = split(D, [0, n // 4, n // 2 + 3, n])
    bm = BlockSparseMatrix(keyed, n, ctx=ctx)
    sm = BlockGaussSeidelSmoother(bm, 3)
    x0 = np.random.default_rng(1).standard_normal(n)
    got = sm.smooth(bm, sy.rhs, x0)
    ref = block_gauss_seidel(dense, st, en, sy.rhs, x0, 3)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())
    r0 = np.linalg.norm(D @ x0 - sy.rhs)
    assert np.linalg.norm(D @ got - sy.rhs) < r0


def test_block_gs_saddle_point_identity_block(ctx):
    rng = np.random.default_rng(3)
    sp, sy = fe_system(1, 6)
    A = coo_oracle(sy).dense()
    nv = sy.n
    B = rng.standard_normal((5, nv)) * (rng.random((5, nv)) < 0.1)
    S = np.block([[A, B.T], [B, np.zeros((5, 5))]])
    dense, keyed, st, en = split(S, [0, nv, nv + 5])
    bm = BlockSparseMatrix(keyed, nv + 5, ctx=ctx)
    sm = BlockGaussSeidelSmoother(bm, 2)
    b = rng.standard_normal(nv + 5)
    x0 = rng.standard_normal(nv + 5)
    got = sm.smooth(bm, b, x0)
    ref = block_gauss_seidel(dense, st, en, b, x0, 2)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())
