"""Stokes (Taylor-Hood) saddle-point solve on the GPU against the oracle:
the block-diagonal preconditioner (velocity multigrid with coloured Schwarz
smoothing, lumped pressure mass) and left-preconditioned GMRES(50)."""
import numpy as np
import pytest

import oracle as O
from jfem_b200 import _native as N
from jfem_b200.stokes import StokesSolver, stokes_problem

pytestmark = pytest.mark.gpu


def oracle_setup(prob, solver):
    L = len(prob.spaces)
    mats = [O.CooMatrix(t.nv, t.nv, *prob.velocity_blocks[l]) for l, t in enumerate(prob.spaces)]
    prol = [O.CooMatrix(prob.spaces[l + 1].nv, prob.spaces[l].nv, *prob.prolongations[l]) for l in range(L - 1)]
    mg = O.MGPreconditioner(mats, prol, prob.velocity_boundary, [None] + [(O.SMOOTH_JACOBI, 1, 1.0)] * (L - 1),
                            cycles=1, use_fmg=False)
    keep = []
    for l in range(1, L):
        sw = solver.schwarz[l - 1]
        So = O.Schwarz(mats[l], O.SCHWARZ_COLORED, sw.patches, 1.0, colours=sw.colours)
        keep.append(So)
        mg.set_schwarz(l, So, 1)
    s = prob.system
    A = O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals)
    return A, O.BlockDiagonal(mg, prob.pressure_inverse), (mats, prol, keep)


@pytest.fixture(scope="module")
def small(ctx):
    prob = stokes_problem(16, 4, nu=1.0, seed=2, pin_pressure=False)
    return prob, StokesSolver(ctx, prob)


def test_preconditioner_matches_oracle(small):
    prob, sol = small
    A, P, keep = oracle_setup(prob, sol)
    v = np.random.default_rng(0).standard_normal(prob.system.n)
    got = sol.P.mvMul(v)
    ref = P.mvmul(v)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_gmres50_matches_oracle(small):
    prob, sol = small
    A, P, keep = oracle_setup(prob, sol)
    b = prob.system.rhs
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_gmres(A, b, tol, M=P, restart=50)
    x, it = sol.solve(tol, restart=50)
    assert ref.status == O.OK and it.last.status == N.OK
    # the first Arnoldi cycle agrees to rounding; after a restart of an
    # indefinite problem the two paths drift by a few iterations
    k = min(20, ref.iterations)
    np.testing.assert_allclose(it.last.history[:k], ref.history[:k], rtol=1e-6)
    assert abs(it.iterations - ref.iterations) <= max(3, ref.iterations // 10)
    xr = ref.x.copy()
    nv = prob.spaces[-1].nv
    xr[nv:] -= xr[nv]
    np.testing.assert_allclose(x, xr, rtol=1e-6, atol=1e-7 * np.abs(xr).max())


def test_pinned_system_solves(ctx):
    """The reference's own system (first pressure unknown pinned) converges to
    the same solution as the consistent singular system shifted to p0 = 0."""
    prob_p = stokes_problem(16, 4, seed=2, pin_pressure=True)
    prob_s = stokes_problem(16, 4, seed=2, pin_pressure=False)
    b = prob_p.system.rhs
    tol = 1e-10 * np.linalg.norm(b)
    xp, itp = StokesSolver(ctx, prob_p).solve(tol)
    xs, its = StokesSolver(ctx, prob_s).solve(tol)
    assert itp.last.status == N.OK and its.last.status == N.OK
    assert its.iterations < itp.iterations
    np.testing.assert_allclose(xp, xs, rtol=1e-6, atol=1e-6 * np.abs(xs).max())


def test_solution_is_discretely_divergence_free(small):
    prob, sol = small
    b = prob.system.rhs
    x, it = sol.solve(1e-10 * np.linalg.norm(b), restart=50)
    s = prob.system
    A = O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals)
    r = A.mvmul(x) - b
    nv = prob.spaces[-1].nv
    assert np.abs(r[nv:]).max() < 1e-7          # pressure rows: -B u = 0
    assert it.iterations < 120


def test_jacobi_and_fp32_variants_converge(ctx):
    prob = stokes_problem(16, 4, seed=5, pin_pressure=False)
    b = prob.system.rhs
    tol = 1e-8 * np.linalg.norm(b)
    for kw in ({"smoother": "jacobi", "runs": 2, "omega": 0.6}, {"fp32_vcycle": True}):
        sol = StokesSolver(ctx, prob, **kw)
        x, it = sol.solve(tol)
        assert it.last.status == N.OK, kw


@pytest.mark.parametrize("fp32", [False, True])
def test_fast_colour_steps_bit_identical(ctx, monkeypatch, fp32):
    """The colour steps with many patches run as batches of patches sharing
    one inverse (128^2 cells: ~455 patches per colour on the finest level),
    those with few patches (the coarser levels) with the inverse copied into
    shared memory; JFEM_SCHWARZ_FAST=0 runs one CTA per patch reading the
    inverse from global memory.  Both sum every row and every inverse product
    in the same order: the preconditioner is equal bit for bit, FP64 and with
    the FP32 V-cycle (FP32 inverses)."""
    prob = stokes_problem(128, 4, nu=1.0, seed=3, pin_pressure=False)
    v = np.random.default_rng(4).standard_normal(prob.system.n)
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("JFEM_SCHWARZ_FAST", flag)
        sol = StokesSolver(ctx, prob, fp32_vcycle=fp32)
        outs.append((sol.P.mvMul(v), sol.P.mvMul(2.0 * v)))
        del sol
    assert np.all(np.isfinite(outs[0][0]))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
