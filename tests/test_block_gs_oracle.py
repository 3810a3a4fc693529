"""The block Gauss-Seidel oracle (oracle/block_gs.py, a restatement of
multigrid/BlockGaussseidelSmoother.java) pinned on the CPU: with every
unknown its own block it is the pointwise Gauss-Seidel smoother of the C
oracle (GaussSeidelSmoother.java: x = (L + D)^-1 (b - R x)); with one block
it is a direct solve; as a smoother of an SPD system it reduces the error in
the energy norm."""
import numpy as np

import oracle as O
from oracle.block_gs import block_gauss_seidel
from fixtures import coo_oracle, fe_system


def blocks_of(D, cuts):
    starts = list(cuts[:-1])
    ends = list(cuts[1:])
    blocks = {}
    for i, (a, b) in enumerate(zip(starts, ends)):
        for j, (c, d) in enumerate(zip(starts, ends)):
            blk = D[a:b, c:d]
            if np.any(blk) or i == j:
                blocks[(i, j)] = blk.copy()
    return blocks, starts, ends


def test_scalar_blocks_are_gauss_seidel():
    sp, sy = fe_system(1, 8)
    A = coo_oracle(sy)
    D = A.dense()
    n = sy.n
    x0 = np.random.default_rng(0).standard_normal(n)
    blocks, st, en = blocks_of(D, list(range(n + 1)))
    got = block_gauss_seidel(blocks, st, en, sy.rhs, x0, 3)
    ref = O.gs_smooth(A, O.SMOOTH_GS, 3, sy.rhs, x0.copy())
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_one_block_is_a_direct_solve_and_smoothing_converges():
    sp, sy = fe_system(1, 10)
    D = coo_oracle(sy).dense()
    n = sy.n
    blocks, st, en = blocks_of(D, [0, n])
    x = block_gauss_seidel(blocks, st, en, sy.rhs, np.zeros(n), 1)
    np.testing.assert_allclose(D @ x, sy.rhs, rtol=1e-10, atol=1e-12)
    blocks, st, en = blocks_of(D, [0, n // 3, 2 * n // 3, n])
    xs = np.linalg.solve(D, sy.rhs)
    x = np.zeros(n)
    e_prev = np.sqrt((xs - x) @ D @ (xs - x))
    for _ in range(5):
        x = block_gauss_seidel(blocks, st, en, sy.rhs, x, 1)
        e = np.sqrt((xs - x) @ D @ (xs - x))
        assert e < e_prev
        e_prev = e
