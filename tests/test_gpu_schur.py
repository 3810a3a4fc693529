"""Schur-complement block solvers (AbstractSchurSolver and its explicit
subclasses) on the GPU against dense numpy block elimination."""
import numpy as np
import pytest

from fixtures import coo_oracle, fe_system
from jfem_b200.linalg import IllegalArgumentException
from jfem_b200.schur import (BlockSparseMatrix, DirectSchur, ExplicitSchurSolver, IterativeExplicitSchur,
                             RichardsonExplicitSchur)

pytestmark = pytest.mark.gpu


def block_system(seed=3, k=3):
    """A DLM-like block system: the Q1 16x16 Helmholtz matrix as the Schur
    block, k small SPD particle blocks, sparse coupling T_i and L_i = T_i^T."""
    sp, sy = fe_system(1, 16)
    A00 = coo_oracle(sy).dense()
    n0 = A00.shape[0]
    rng = np.random.default_rng(seed)
    blocks = {(0, 0): A00}
    sizes = [int(rng.integers(4, 10)) for _ in range(k)]
    n = n0 + sum(sizes)
    M = np.zeros((n, n))
    M[:n0, :n0] = A00
    s = n0
    for m in sizes:
        B = rng.standard_normal((m, m))
        D = B @ B.T + m * np.eye(m)
        T = np.where(rng.random((n0, m)) < 0.05, rng.standard_normal((n0, m)) * 0.1, 0.0)
        blocks[(s, s)] = D
        blocks[(0, s)] = T
        blocks[(s, 0)] = T.T.copy()
        M[s:s + m, s:s + m] = D
        M[:n0, s:s + m] = T
        M[s:s + m, :n0] = T.T
        s += m
    return blocks, M, n0, sizes


def dense_schur(M, n0, sizes):
    S = M[:n0, :n0].copy()
    s = n0
    for m in sizes:
        S -= M[:n0, s:s + m] @ np.linalg.inv(M[s:s + m, s:s + m]) @ M[s:s + m, :n0]
        s += m
    return S


def test_block_matrix_mvmul(ctx):
    blocks, M, n0, sizes = block_system()
    B = BlockSparseMatrix(blocks, M.shape[0], ctx=ctx)
    assert list(B.getBlockSizes()) == [n0] + sizes
    x = np.random.default_rng(1).standard_normal(M.shape[0])
    np.testing.assert_allclose(B.mvMul(x), M @ x, rtol=1e-13, atol=1e-13)


def test_explicit_schur_complement(ctx):
    blocks, M, n0, sizes = block_system()
    S = ExplicitSchurSolver(BlockSparseMatrix(blocks, M.shape[0], ctx=ctx)).getSchurComplement()
    ref = dense_schur(M, n0, sizes)
    r, c, v = S.coo()
    got = np.zeros_like(ref)
    got[r, c] = v
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("cls,rtol", [(DirectSchur, 1e-10), (IterativeExplicitSchur, 1e-7)])
def test_schur_solvers_solve_the_block_system(ctx, cls, rtol):
    blocks, M, n0, sizes = block_system(seed=5)
    solver = cls(BlockSparseMatrix(blocks, M.shape[0], ctx=ctx))
    f = np.random.default_rng(2).standard_normal(M.shape[0])
    x = solver.mvMul(f)
    ref = np.linalg.solve(M, f)
    assert np.linalg.norm(x - ref) <= rtol * np.linalg.norm(ref)


def test_richardson_schur_with_an_exact_preconditioner(ctx):
    blocks, M, n0, sizes = block_system(seed=7)
    B = BlockSparseMatrix(blocks, M.shape[0], ctx=ctx)
    solver = RichardsonExplicitSchur(B)
    Sinv = np.linalg.inv(dense_schur(M, n0, sizes))

    class Prec:
        def mvMul(self, v):
            return Sinv @ v

    solver.preconditioner = Prec()
    f = np.random.default_rng(3).standard_normal(M.shape[0])
    x = solver.mvMul(f)
    assert solver.iterations <= 3
    ref = np.linalg.solve(M, f)
    assert np.linalg.norm(x - ref) <= 1e-7 * np.linalg.norm(ref)


def test_missing_blocks_are_rejected(ctx):
    blocks, M, n0, sizes = block_system()
    del blocks[(n0, 0)]
    with pytest.raises(IllegalArgumentException, match="left block"):
        DirectSchur(BlockSparseMatrix(blocks, M.shape[0], ctx=ctx))


def test_implicit_schur_operator_and_solve(ctx):
    """ImplicitSchurSolver (linalg/ImplicitSchurSolver.java:17-57): the
    composed operator equals the dense Schur complement; IterativeImplicitSchur
    (IterativeImplicitSchur.java:19-23: PGMRES with the inverse of A00, 1e-9)
    solves the block system like the explicit solver does."""
    from jfem_b200.schur import ImplicitSchurSolver, IterativeImplicitSchur
    blocks, M, n0, sizes = block_system(seed=5)
    B = BlockSparseMatrix(blocks, M.shape[0], ctx=ctx)
    Sd = dense_schur(M, n0, sizes)
    op = ImplicitSchurSolver(B).schurMvMul()
    rng = np.random.default_rng(2)
    for _ in range(2):
        v = rng.standard_normal(n0)
        np.testing.assert_allclose(op.mvMul(v), Sd @ v, rtol=1e-12, atol=1e-12 * np.abs(Sd @ v).max())
    solver = IterativeImplicitSchur(B)
    f = rng.standard_normal(M.shape[0])
    u = solver.mvMul(f)
    np.testing.assert_allclose(u, np.linalg.solve(M, f), rtol=1e-7, atol=1e-7 * np.abs(u).max())
    assert solver.it.last.status == 0 and solver.it.iterations >= 1
    # the same PGMRES on the explicit complement: same iteration count within one
    ex = IterativeExplicitSchur(B)
    u2 = ex.mvMul(f)
    np.testing.assert_allclose(u2, u, rtol=1e-7, atol=1e-7 * np.abs(u).max())
    assert abs(ex.it.iterations - solver.it.iterations) <= 1


def test_implicit_schur_missing_block(ctx):
    from jfem_b200.schur import IterativeImplicitSchur
    blocks, M, n0, sizes = block_system(k=2)
    s = n0
    del blocks[(s, 0)]
    with pytest.raises(IllegalArgumentException):
        IterativeImplicitSchur(BlockSparseMatrix(blocks, M.shape[0], ctx=ctx))
