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


def test_uninvertible_block_becomes_identity():
    """BlockSparseMatrix.getInvertedDiagonalMatrix (BlockSparseMatrix.java:194-220)
    replaces a diagonal block it cannot invert by the identity: with a zero
    (2, 2) block the second block of the result is its right-hand side minus
    the lower block times the first block's solution."""
    rng = np.random.default_rng(4)
    A = rng.standard_normal((4, 4)) + 4 * np.eye(4)
    B = rng.standard_normal((2, 4))
    blocks = {(0, 0): A, (0, 1): B.T.copy(), (1, 0): B, (1, 1): np.zeros((2, 2))}
    b = rng.standard_normal(6)
    x0 = rng.standard_normal(6)
    x = block_gauss_seidel(blocks, [0, 4], [4, 6], b, x0, 1)
    x1 = np.linalg.solve(A, b[:4] - B.T @ x0[4:])
    np.testing.assert_allclose(x[:4], x1, rtol=1e-12)
    np.testing.assert_allclose(x[4:], b[4:] - B @ x1, rtol=1e-12)
