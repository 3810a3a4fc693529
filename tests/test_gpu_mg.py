"""GPU multigrid pieces (smoothers, V-cycle, FMG, preconditioner) against the oracle."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, mg_levels
from jfem_b200 import JacobiSmoother, MGPreconditioner, RichardsonSmoother
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu


def dev(sy, ctx):
    return DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)


@pytest.mark.parametrize("kind,runs,omega", [(O.SMOOTH_JACOBI, 3, 2 / 3), (O.SMOOTH_RICHARDSON, 4, 0.1)])
def test_smoother(ctx, kind, runs, omega):
    sp, sy = fe_system(2, 16)
    A = dev(sy, ctx)
    x0 = np.random.default_rng(0).standard_normal(sy.n)
    ref = O.smooth(coo_oracle(sy), kind, runs, omega, sy.rhs, x0)
    sm = JacobiSmoother(runs, omega) if kind == O.SMOOTH_JACOBI else RichardsonSmoother(omega, runs)
    got = sm.smooth(A, sy.rhs, x0)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def build(h, ctx, sm_tuple, cycles, use_fmg):
    mats_o = [coo_oracle(s) for s in h.systems]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [sm_tuple] * (len(mats_o) - 1), cycles=cycles,
                              use_fmg=use_fmg)
    mats = [dev(s, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(len(h.systems) - 1)]
    kind, runs, om = sm_tuple
    sm = JacobiSmoother(runs, om) if kind == O.SMOOTH_JACOBI else RichardsonSmoother(om, runs)
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [sm] * (len(mats) - 1), cycles=cycles, use_fmg=use_fmg,
                          ctx=ctx)
    return mg_o, mg, mats


@pytest.mark.parametrize("p,coarse,L", [(1, 4, 5), (2, 2, 5)])
@pytest.mark.parametrize("sm", [(O.SMOOTH_JACOBI, 2, 2 / 3), (O.SMOOTH_RICHARDSON, 8, 0.1)])
def test_vcycle_fmg_apply(ctx, p, coarse, L, sm):
    h = mg_levels(p, coarse, L, modes=6, seed=4)
    mg_o, mg, mats = build(h, ctx, sm, 3, True)
    b = h.finest.rhs
    x0 = np.random.default_rng(1).standard_normal(b.size) * 0.1
    for got, ref in ((mg.vCycle(x0, b), mg_o.vcycle(x0, b)),
                     (mg.fullVCycleCorrection(b), mg_o.fmg(b)),
                     (mg.mvMul(b), mg_o.mvmul(b))):
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_mg_single_level(ctx):
    """levels = 1: the preconditioner is the dense coarse solve."""
    sp, sy = fe_system(1, 4)
    A = dev(sy, ctx)
    mg = MGPreconditioner([A], [], [sy.boundary], [None], cycles=1, use_fmg=False, ctx=ctx)
    D = coo_oracle(sy).dense()
    np.testing.assert_allclose(mg.mvMul(sy.rhs), np.linalg.solve(D, sy.rhs), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("p,coarse,L", [(1, 4, 6), (2, 2, 6)])
@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed-fp16"])
def test_vcycle_tail_matches_per_launch(ctx, monkeypatch, p, coarse, L, precision):
    """The levels below a few thousand rows run as one cluster launch (the
    V-cycle tail, on by default; JFEM_MG_TAIL=0 runs one launch per
    operation).  The V-cycle, the preconditioner and a whole PCG solve agree
    with the per-launch path to rounding (the tail sums every row in column
    order; the per-launch kernels of the smallest levels split rows over 4-8
    threads), with the same iteration count; the FP64 V-cycle also matches
    the oracle to 1e-10."""
    from jfem_b200 import IterativeSolver
    h = mg_levels(p, coarse, L, modes=8, seed=5)
    b = h.finest.rhs
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("JFEM_MG_TAIL", flag)
        mats = [dev(s, ctx) for s in h.systems]
        prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
        mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2.0 / 3.0)] * (L - 1), cycles=1,
                              use_fmg=False, precision=precision, ctx=ctx)
        s = IterativeSolver(ctx=ctx)
        s.precision = "fp64" if precision == "fp64" else "mixed-precond"
        x = s.solvePCG(mats[-1], mg, b, 1e-9 * np.linalg.norm(b))
        v = mg.vCycle(np.zeros(b.size), b)
        outs.append((v, x, s.iterations, s.last.history.copy()))
    (v1, x1, i1, h1), (v0, x0, i0, h0) = outs
    np.testing.assert_allclose(v1, v0, rtol=1e-11, atol=1e-12 * np.abs(v0).max())
    assert i1 == i0
    np.testing.assert_allclose(h1, h0, rtol=1e-4 if precision != "fp64" else 1e-9)
    np.testing.assert_allclose(x1, x0, rtol=1e-7, atol=1e-9 * np.abs(x0).max())
    mats_o = [coo_oracle(s) for s in h.systems]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2.0 / 3.0)] * (L - 1),
                              cycles=1, use_fmg=False)
    ref = mg_o.vcycle(np.zeros(b.size), b)
    np.testing.assert_allclose(v1, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


@pytest.mark.parametrize("p,coarse,L", [(1, 4, 6), (1, 4, 4), (2, 2, 6)])
@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed-bf16"])
def test_vcycle_tail_local_levels_bit_identical(ctx, monkeypatch, p, coarse, L, precision):
    """The coarsest levels of the V-cycle tail are owned wholly by one CTA of
    the cluster (CTA barriers between their phases instead of cluster
    barriers; JFEM_MG_TAIL_LOCAL=0 spreads them over the cluster like the
    larger levels).  Every row is summed by the same thread code in the same
    column order either way, so the V-cycle, the preconditioner and a PCG
    solve are equal bit for bit, including hierarchies whose tail levels are
    all local (Q1 4 levels)."""
    from jfem_b200 import IterativeSolver
    h = mg_levels(p, coarse, L, modes=8, seed=9)
    b = h.finest.rhs
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("JFEM_MG_TAIL_LOCAL", flag)
        mats = [dev(s, ctx) for s in h.systems]
        prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
        mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2.0 / 3.0)] * (L - 1), cycles=1,
                              use_fmg=False, precision=precision, ctx=ctx)
        s = IterativeSolver(ctx=ctx)
        s.precision = "fp64" if precision == "fp64" else "mixed-precond"
        x = s.solvePCG(mats[-1], mg, b, 1e-9 * np.linalg.norm(b))
        v = mg.vCycle(np.zeros(b.size), b)
        w = mg.mvMul(b)
        outs.append((v, w, x, s.iterations))
    (v1, w1, x1, i1), (v0, w0, x0, i0) = outs
    assert np.all(np.isfinite(v1))
    assert np.array_equal(v1, v0) and np.array_equal(w1, w0) and np.array_equal(x1, x0) and i1 == i0


@pytest.mark.parametrize("p,coarse,L", [(1, 4, 5), (2, 2, 4)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wcycle_and_mvmulw(ctx, p, coarse, L, precision):
    """wCycle (MGPreconditionerInterface.java:300-305, mgStepW :200-291) and the
    preconditioner mvMulW (MGPreconditionerSpace.java:165-183: FMG + cycles
    W-cycles) against the oracle to 1e-10; the FP32 hierarchy inside a PCG
    solve reaches the tolerance in the oracle's FP64 iteration count."""
    from jfem_b200 import IterativeSolver
    h = mg_levels(p, coarse, L, modes=6, seed=7)
    sm = (O.SMOOTH_JACOBI, 2, 2 / 3)
    mats_o = [coo_oracle(s) for s in h.systems]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [sm] * (L - 1), cycles=2, use_fmg=True,
                              cycle="W")
    mats = [dev(s, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (L - 1), cycles=2,
                          use_fmg=True, precision=precision, ctx=ctx, cycle="W")
    b = h.finest.rhs
    x0 = np.random.default_rng(2).standard_normal(b.size) * 0.1
    for got, ref in ((mg.wCycle(x0, b), mg_o.wcycle(x0, b)), (mg.mvMul(b), mg_o.mvmul(b))):
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    # the W-cycle smooths more than the V-cycle: its error reduction is at least as good
    e_w = np.linalg.norm(b - mats_o[-1].mvmul(mg_o.wcycle(np.zeros(b.size), b)))
    e_v = np.linalg.norm(b - mats_o[-1].mvmul(mg_o.vcycle(np.zeros(b.size), b)))
    assert e_w <= e_v
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_pcg(mats_o[-1], mg_o, b, tol)
    s = IterativeSolver(ctx=ctx)
    s.precision = "fp64" if precision == "fp64" else "mixed-precond"
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert s.iterations == ref.iterations
    assert np.linalg.norm(b - mats_o[-1].mvmul(x)) <= tol
    if precision == "fp64":
        assert np.linalg.norm(x - ref.x) / np.linalg.norm(ref.x) < 1e-8
