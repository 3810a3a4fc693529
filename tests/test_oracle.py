"""The CPU oracle against the reference's known answers (no GPU)."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, java_sparse, java_vector, kat, mg_levels


def dense_coo(a):
    a = np.asarray(a, dtype=np.float64)
    r, c = np.nonzero(a)
    return O.CooMatrix(a.shape[0], a.shape[1], r, c, a[r, c])


def test_java_random_pins():
    g = kat()["java_random_first_double"]
    for seed, val in g.items():
        assert O.java_random_doubles(int(seed), 1)[0] == val


@pytest.mark.parametrize("name", ["symm", "nonsymm", "good_nonsymm"])
def test_kat_dense_and_krylov(name):
    s = kat()["systems"][name]
    A, b, x = np.array(s["A"], float), np.array(s["b"], float), np.array(s["x"])
    # DenseMatrix.solve known answer
    np.testing.assert_allclose(O.dense_solve(A, b), x, rtol=0, atol=1e-13)
    M = dense_coo(A)
    I = dense_coo(np.eye(3))
    # GMResTest: GMRES2 (with and without identity preconditioner) reproduces solve(b)
    for r in (O.solve_gmres2(M, b, 1e-12), O.solve_gmres2(M, b, 1e-12, M=I), O.solve_gmres(M, b, 1e-12),
              O.solve_gmres(M, b, 1e-12, M=I)):
        assert r.status == O.OK
        np.testing.assert_allclose(r.x, x, atol=1e-10)
    if name == "good_nonsymm":
        Ainv = dense_coo(O.dense_inverse(A))
        r = O.solve_gmres2(M, b, 1e-12, M=Ainv)
        np.testing.assert_allclose(r.x, x, atol=1e-10)
    # BiCGStabTest: BiCGStab on the same systems
    r = O.solve_bicgstab(M, b, 1e-12)
    np.testing.assert_allclose(M.mvmul(r.x), b, atol=1e-9)


def test_identity_15():
    s = kat()["systems"]["identity15"]
    b = np.array(s["b"], float)
    I = dense_coo(np.eye(15))
    for r in (O.solve_gmres2(I, b, 1e-12), O.solve_gmres(I, b, 1e-12), O.solve_cg(I, b, 1e-12),
              O.solve_bicgstab(I, b, 1e-12)):
        np.testing.assert_allclose(r.x, b, atol=1e-12)


def test_sparse_mvmul_fixtures():
    """SparseMvMulTest: the COO scatter and the bucketed SparseMvMul agree
    (SparseMvMulTest.java:150-159)."""
    for rows, cols, seed, dens, integer, vseed, tseed in [
        (10, 10, 14239078, 0.1, True, 124350987, 124350987),
        (500, 700, 891765234, 0.01, False, 124876, 81726534),
    ]:
        ri, ci, v = java_sparse(rows, cols, seed, dens, integer)
        M = O.CooMatrix(rows, cols, ri, ci, v)
        x = java_vector(cols, vseed, integer)
        t = java_vector(rows, tseed, integer)
        np.testing.assert_allclose(M.mvmul(x), M.mvmul_rows(x), rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(M.tvmul(t), M.tvmul_cols(t), rtol=1e-13, atol=1e-13)
        D = M.dense()
        np.testing.assert_allclose(M.mvmul(x), D @ x, rtol=1e-12, atol=1e-12)


def test_cg_fe_system():
    sp, sy = fe_system(1, 16)
    A = coo_oracle(sy)
    bn = np.linalg.norm(sy.rhs)
    r = O.solve_cg(A, sy.rhs, 1e-10 * bn)
    assert r.status == O.OK
    D = A.dense()
    np.testing.assert_allclose(r.x, np.linalg.solve(D, sy.rhs), rtol=1e-8, atol=1e-10 * bn)
    assert r.iterations == len(r.history)
    assert r.history[-1] <= 1e-10 * bn


def test_bicgstab_gmres_fe_system():
    sp, sy = fe_system(1, 12)
    A = coo_oracle(sy)
    xs = np.linalg.solve(A.dense(), sy.rhs)
    tol = 1e-10 * np.linalg.norm(sy.rhs)
    for r in (O.solve_bicgstab(A, sy.rhs, tol), O.solve_gmres(A, sy.rhs, tol), O.solve_gmres2(A, sy.rhs, tol)):
        assert r.status in (O.OK, O.BREAKDOWN)
        np.testing.assert_allclose(r.x, xs, rtol=1e-7, atol=1e-9)


def _mg(h, smoother=(O.SMOOTH_JACOBI, 2, 2.0 / 3.0), cycles=3, use_fmg=True):
    mats = [coo_oracle(s) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    sm = [None] + [smoother] * (len(mats) - 1)
    return mats, O.MGPreconditioner(mats, prol, h.boundary, sm, cycles=cycles, use_fmg=use_fmg)


def test_mg_vcycle_contracts():
    h = mg_levels(1, 4, 4)
    mats, mg = _mg(h)
    A = mats[-1]
    b = h.finest.rhs
    x = np.zeros(A.rows)
    r0 = np.linalg.norm(b)
    for _ in range(5):
        x = mg.vcycle(x, b)
    r = np.linalg.norm(b - A.mvmul(x))
    assert r < 1e-3 * r0


def test_pcg_mg_iterations_small():
    """GMG-PCG converges in few iterations independent of the level count."""
    its = []
    for L in (3, 4, 5):
        h = mg_levels(2, 2, L, modes=4)
        mats, mg = _mg(h, cycles=1, use_fmg=False)
        b = h.finest.rhs
        r = O.solve_pcg(mats[-1], mg, b, 1e-8 * np.linalg.norm(b))
        assert r.status == O.OK
        its.append(r.iterations)
    assert max(its) <= 12 and max(its) - min(its) <= 3


def test_laplace_mg_gmres_pin():
    """examples/LaplaceMG.java:22-101: MG-preconditioned GMRES to 1e-8 needs
    fewer than 10 iterations (Richardson 0.1 x 8 smoothers, Q1, 4*2^r cells)."""
    for ref in (2, 3, 4):
        h = mg_levels(1, 4, ref + 1, mass=0.0)
        mats, mg = _mg(h, smoother=(O.SMOOTH_RICHARDSON, 8, 0.1))
        b = h.finest.rhs
        r = O.solve_gmres(mats[-1], b, 1e-8, M=mg)
        assert r.status == O.OK
        assert r.iterations < 10


def test_oracle_mmmul_tmmul_dense():
    """SparseMatrix.mmMul / Matrix.tmMul restatements against dense products;
    exact-zero sums are not stored."""
    rng = np.random.default_rng(11)
    for (m, k, n) in ((30, 20, 25), (1, 7, 3)):
        a = np.where(rng.random((m, k)) < 0.2, rng.integers(-3, 4, (m, k)), 0).astype(float)
        b = np.where(rng.random((k, n)) < 0.2, rng.integers(-3, 4, (k, n)), 0).astype(float)
        A = O.CooMatrix(m, k, *np.nonzero(a), a[np.nonzero(a)])
        B = O.CooMatrix(k, n, *np.nonzero(b), b[np.nonzero(b)])
        C = A.mmmul(B)
        assert np.array_equal(C.dense(), a @ b)
        assert C.v.size == np.count_nonzero(a @ b) and np.all(C.v != 0)
        c = np.where(rng.random((m, n)) < 0.2, rng.standard_normal((m, n)), 0.0)
        Cm = O.CooMatrix(m, n, *np.nonzero(c), c[np.nonzero(c)])
        np.testing.assert_allclose(A.tmmul(Cm).dense(), a.T @ c, rtol=1e-14, atol=1e-14)


def test_oracle_gauss_seidel_dense():
    """ForwardBackwardGaussSeidelSmoother / GaussSeidelSmoother restatements
    against dense triangular algebra, natural and permuted orderings."""
    rng = np.random.default_rng(5)
    n = 12
    a = rng.standard_normal((n, n))
    a = a + a.T + 12 * np.eye(n)
    a[np.abs(a) < 0.6] = 0.0
    A = O.CooMatrix(n, n, *np.nonzero(a), a[np.nonzero(a)])
    b, x0 = rng.standard_normal(n), rng.standard_normal(n)
    for rank in (None, rng.permutation(n).astype(np.int32)):
        p = np.arange(n) if rank is None else np.argsort(rank)      # p[k] = row at position k
        ap = a[np.ix_(p, p)]
        L, U, D = np.tril(ap), np.triu(ap), np.diag(np.diag(ap))
        bp, xp = b[p], x0[p]
        ref = xp + np.linalg.solve(L, D @ np.linalg.solve(U, bp - ap @ xp))
        got = O.gs_smooth(A, O.SMOOTH_FBGS, 1, b, x0, rank)
        np.testing.assert_allclose(got[p], ref, rtol=1e-13, atol=1e-13)
        ref = np.linalg.solve(L, bp - np.triu(ap, 1) @ xp)
        got = O.gs_smooth(A, O.SMOOTH_GS, 1, b, x0, rank)
        np.testing.assert_allclose(got[p], ref, rtol=1e-13, atol=1e-13)


def test_mg_wcycle_composition():
    """mgStepW (MGPreconditionerInterface.java:200-291) restated from public
    pieces: smooth, then twice [restrict the defect with zero boundary values,
    one V-cycle of the next coarser hierarchy from zero, prolong with zero
    boundary values, add], then smooth; mvMulW = boundary copy + FMG + W-cycles."""
    import scipy.sparse as sps
    L = 4
    h = mg_levels(1, 4, L, modes=4, seed=2)
    sm = (O.SMOOTH_JACOBI, 2, 2 / 3)
    mats = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
    mg = O.MGPreconditioner(mats, prol, h.boundary, [None] + [sm] * (L - 1), cycles=2, use_fmg=True, cycle="W")
    sub = O.MGPreconditioner(mats[:-1], prol[:-1], h.boundary[:-1], [None] + [sm] * (L - 2), cycles=1,
                             use_fmg=False)
    P = sps.csr_matrix((h.prolong[-1][2], (h.prolong[-1][0], h.prolong[-1][1])),
                       shape=(h.systems[-1].n, h.systems[-2].n))
    A = mats[-1]
    b = h.finest.rhs
    x0 = np.random.default_rng(5).standard_normal(b.size) * 0.1

    def zero(v, l):
        v = v.copy()
        v[np.asarray(h.boundary[l], dtype=np.int64)] = 0.0
        return v

    x = O.smooth(A, *sm, b, x0)
    for _ in range(2):
        rc = zero(P.T @ (b - A.mvmul(x)), L - 2)
        x = x + zero(P @ sub.vcycle(np.zeros(rc.size), rc), L - 1)
    x = O.smooth(A, *sm, b, x)
    np.testing.assert_allclose(mg.wcycle(x0, b), x, rtol=1e-12, atol=1e-14 * np.abs(x).max())
    # mvMulW with cycles = 2 (boundary values zero here: Dirichlet data 0)
    d = b.copy()
    it = mg.fmg(d)
    for _ in range(2):
        it = mg.wcycle(it, d)
    np.testing.assert_allclose(mg.mvmul(b), it, rtol=1e-13, atol=1e-15 * np.abs(it).max())
