"""GPU dense LU (DenseMatrix.solve / inverse, JNI iSolve / iInverse) and the
SparseMatrix.solve drop-in."""
import numpy as np
import pytest

import oracle as O
from fixtures import fe_system, kat
from jfem_b200 import SingularMatrixException, SparseMatrix
from jfem_b200.linalg import DenseMatrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["symm", "nonsymm", "good_nonsymm"])
def test_kat(ctx, name):
    k = kat()["systems"][name]
    D = DenseMatrix(k["A"], ctx)
    np.testing.assert_allclose(D.solve(k["b"]), k["x"], atol=1e-13)
    np.testing.assert_allclose(D.inverse() @ np.array(k["A"], float), np.eye(3), atol=1e-13)


@pytest.mark.parametrize("n", [1, 7, 81, 300])
def test_random_dense(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal(n)
    D = DenseMatrix(a, ctx)
    np.testing.assert_allclose(D.solve(b), O.dense_solve(a, b), rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(D.inverse(), O.dense_inverse(a), rtol=1e-10, atol=1e-12)


def test_singular(ctx):
    with pytest.raises(SingularMatrixException):
        DenseMatrix(np.array([[1.0, 2.0], [2.0, 4.0]]), ctx).solve([1.0, 1.0])


def test_sparse_solve_dropin(ctx):
    sp, sy = fe_system(1, 24)
    A = SparseMatrix.from_coo(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    ref = O.dense_solve(O.CooMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals).dense(), sy.rhs)
    x = A.solve(sy.rhs)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-8


def test_sparse_solve_dropin_large(ctx):
    sp, sy = fe_system(1, 96)          # n = 9409 > 4096: iterative path
    A = SparseMatrix.from_coo(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    x = A.solve(sy.rhs)
    r = sy.rhs - O.CooMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals).mvmul(x)
    assert np.linalg.norm(r) <= 1e-11 * np.linalg.norm(sy.rhs)


@pytest.mark.parametrize("n", [33, 64, 257, 1000, 4096])
def test_blocked_lu_bit_identical(ctx, monkeypatch, n):
    """Matrices of more than 32 columns are factored in 32-column panels
    (panel, row interchanges, U12 triangular solve, A22 tile update); every
    entry receives the same updates in the same order with one rounding each
    as in the column-by-column loop (JFEM_LU_BLOCKED=0), so the solutions and
    inverses are equal bit for bit, pivoting included (the matrix has no
    dominant diagonal, so rows are interchanged); the solve matches the
    oracle's LU."""
    rng = np.random.default_rng(100 + n)
    a = rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("JFEM_LU_BLOCKED", flag)
        D = DenseMatrix(a, ctx)
        outs.append((D.solve(b), D.inverse() if n <= 1000 else None))
    assert np.array_equal(outs[0][0], outs[1][0])
    if n <= 1000:
        assert np.array_equal(outs[0][1], outs[1][1])
    x = outs[0][0]
    assert np.linalg.norm(a @ x - b) <= 1e-10 * np.linalg.norm(a) * np.linalg.norm(x) * n
    if n <= 1000:
        np.testing.assert_allclose(x, O.dense_solve(a, b), rtol=1e-7, atol=1e-9 * np.abs(x).max())


def test_direct_solver_caches_patch_inverses(ctx):
    """schwarz/DirectSolver.java:22-38 as a SystemSolver: the first solve for
    a patch inverts the given local system (device LU) and caches it under
    the patch number; later solves for that patch reuse the inverse, whatever
    system they pass."""
    from jfem_b200.schwarz import DirectSolver
    rng = np.random.default_rng(9)
    a = rng.standard_normal((12, 12)) + 12 * np.eye(12)
    b = rng.standard_normal(12)
    sp = SparseMatrix.from_coo(12, 12, *np.nonzero(a), a[np.nonzero(a)], ctx)
    ds = DirectSolver()
    np.testing.assert_allclose(ds.solve(sp, b, 3), np.linalg.solve(a, b), rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(ds.solve(DenseMatrix(2 * a, ctx), b, 3), np.linalg.solve(a, b), rtol=1e-12,
                               atol=1e-13)
    np.testing.assert_allclose(ds.solve(DenseMatrix(2 * a, ctx), b, 4), np.linalg.solve(2 * a, b), rtol=1e-12,
                               atol=1e-13)
    assert sorted(ds.inverses) == [3, 4]
