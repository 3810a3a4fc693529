"""The numpy FGMRES oracle, pinned against the C restatement of the
reference's GMRES (no GPU)."""
import numpy as np

import oracle as O
from fixtures import coo_oracle, fe_system, mg_levels
from oracle.fgmres import OK, solve_fgmres


def test_fgmres_identity_matches_gmres():
    """With M = I, FGMRES from zero is GMRES from zero (GMRES.java:59-60):
    same iteration count, same residual estimates."""
    sp, sy = fe_system(1, 16, mass=5.0)
    A = coo_oracle(sy)
    tol = 1e-9 * np.linalg.norm(sy.rhs)
    ref = O.solve_gmres(A, sy.rhs, tol, x0=np.zeros(sy.n), restart=20, max_restarts=50)
    x, it, rs, st, hist = solve_fgmres(A.mvmul, lambda v: v, sy.rhs, tol, restart=20, max_restarts=50)
    assert st == OK and ref.status == O.OK
    assert it == ref.iterations and rs == ref.restarts
    # the estimates agree until rounding of the orthogonalisation shows
    np.testing.assert_allclose(hist, ref.history[:it], rtol=1e-6, atol=1e-8 * hist[0])
    np.testing.assert_allclose(x, ref.x, rtol=1e-6, atol=1e-9 * np.abs(ref.x).max())


def test_fgmres_fixed_preconditioner_is_right_preconditioned_gmres():
    """A fixed V-cycle preconditioner: FGMRES converges to the FP64 solution in
    few iterations and its true residual meets the absolute tolerance."""
    h = mg_levels(1, 4, 4, mass=5.0)
    mats = [coo_oracle(s) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    mg = O.MGPreconditioner(mats, prol, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2 / 3)] * 3, cycles=1,
                            use_fmg=False)
    A = mats[-1]
    b = h.finest.rhs
    tol = 1e-10 * np.linalg.norm(b)
    x, it, rs, st, hist = solve_fgmres(A.mvmul, mg.mvmul, b, tol, restart=30)
    assert st == OK
    assert it < 20
    assert np.linalg.norm(b - A.mvmul(x)) <= tol
    xs = np.linalg.solve(A.dense(), b)
    np.testing.assert_allclose(x, xs, rtol=1e-7, atol=1e-9 * np.abs(xs).max())


def test_fgmres_restart_rule():
    """restart = 2 forces cycles of four columns (j > restart ends a cycle) and
    the GMRES.java:92 restart rule; it still converges."""
    sp, sy = fe_system(1, 8, mass=5.0)
    A = coo_oracle(sy)
    tol = 1e-8 * np.linalg.norm(sy.rhs)
    x, it, rs, st, hist = solve_fgmres(A.mvmul, lambda v: v, sy.rhs, tol, restart=2, max_restarts=2000)
    assert st == OK and rs > 0
    assert np.linalg.norm(sy.rhs - A.mvmul(x)) <= tol
    ref = O.solve_gmres(A, sy.rhs, tol, x0=np.zeros(sy.n), restart=2, max_restarts=2000)
    assert it == ref.iterations and rs == ref.restarts
