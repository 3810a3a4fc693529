"""GPU Krylov solvers through the C ABI against the oracle (same seeded inputs)."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, kat, mg_levels
from jfem_b200 import IterativeSolver, MGPreconditioner, JacobiSmoother, RichardsonSmoother, SparseMatrix
from jfem_b200 import _native as N
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu

REL = 1e-8   # FP64 path: relative solution error against the oracle's solve


def dev(sy, ctx):
    return DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("graph", [True, False])
def test_cg_cfg0(ctx, graph):
    """Q1 64x64 (4,225 dofs), -Lap u + 5u = f, CG to 1e-10 ||b|| from e0."""
    sp, sy = fe_system(1, 64, modes=4, seed=0)
    tol = 1e-10 * np.linalg.norm(sy.rhs)
    ref = O.solve_cg(coo_oracle(sy), sy.rhs, tol)
    s = IterativeSolver(ctx=ctx)
    s.use_graph = graph
    x = s.solveCG(dev(sy, ctx), sy.rhs, tol)
    assert s.last.status == N.OK
    assert rel(x, ref.x) < REL
    assert abs(s.iterations - ref.iterations) <= 2
    assert s.last.final_residual <= tol * 1.01
    # CG residual histories agree until rounding differences (FMA, summation
    # order) are amplified by the loss of orthogonality
    np.testing.assert_allclose(s.last.history[:5], ref.history[:5], rtol=1e-8)


def test_cg_warm_start_and_reuse(ctx):
    sp, sy = fe_system(1, 32)
    tol = 1e-10 * np.linalg.norm(sy.rhs)
    s = IterativeSolver(ctx=ctx)
    A = dev(sy, ctx)
    x1 = s.solveCG(A, sy.rhs, tol)
    it1 = s.iterations
    x2 = s.solveCG(A, sy.rhs, tol)          # lastSolution warm start: converged already
    assert s.iterations == 0 and it1 > 0
    assert np.array_equal(x1, x2)


def _mg_pair(h, ctx, smoother, cycles, use_fmg, precision="fp64"):
    mats_o = [coo_oracle(s) for s in h.systems]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    kind, runs, om = smoother
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [smoother] * (len(mats_o) - 1), cycles=cycles,
                              use_fmg=use_fmg)
    mats = [dev(s, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(len(h.systems) - 1)]
    sm = JacobiSmoother(runs, om) if kind == O.SMOOTH_JACOBI else RichardsonSmoother(om, runs)
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [sm] * (len(mats) - 1), cycles=cycles, use_fmg=use_fmg,
                          precision=precision, ctx=ctx)
    return mats_o, mg_o, mats, mg


@pytest.mark.parametrize("cycles,use_fmg", [(3, True), (1, False)])
def test_pcg_mg_matches_oracle(ctx, cycles, use_fmg):
    h = mg_levels(2, 4, 4, modes=8, seed=1)     # Q2 32x32 finest
    mats_o, mg_o, mats, mg = _mg_pair(h, ctx, (O.SMOOTH_JACOBI, 2, 2.0 / 3.0), cycles, use_fmg)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_pcg(mats_o[-1], mg_o, b, tol)
    s = IterativeSolver(ctx=ctx)
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK
    assert s.iterations == ref.iterations
    assert rel(x, ref.x) < REL
    np.testing.assert_allclose(s.last.history, ref.history, rtol=1e-7)


def test_mixed_precision_pcg(ctx):
    h = mg_levels(2, 4, 5, modes=16, seed=2)    # Q2 64x64
    mats_o, mg_o, mats, mg = _mg_pair(h, ctx, (O.SMOOTH_JACOBI, 2, 2.0 / 3.0), 1, False, precision="mixed")
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_pcg(mats_o[-1], mg_o, b, tol)
    s = IterativeSolver(ctx=ctx)
    s.precision = "mixed"
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK
    assert s.last.final_residual <= tol
    assert rel(x, ref.x) < 1e-7
    assert s.last.outer_iterations >= 2
    s = IterativeSolver(ctx=ctx)
    s.precision = "mixed-precond"
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK and s.last.final_residual <= tol
    assert rel(x, ref.x) < 1e-7
    assert abs(s.iterations - ref.iterations) <= 1


@pytest.mark.parametrize("name", ["symm", "nonsymm", "good_nonsymm"])
def test_kat_gmres_bicgstab(ctx, name):
    k = kat()["systems"][name]
    a = np.array(k["A"], float)
    r, c = np.nonzero(a)
    A = SparseMatrix.from_coo(3, 3, r, c, a[r, c], ctx)
    b = np.array(k["b"], float)
    x = np.array(k["x"])
    for solve in ("solveGMRES", "solveBiCGStab"):
        s = IterativeSolver(ctx=ctx)
        got = getattr(s, solve)(A, b, 1e-12)
        np.testing.assert_allclose(got, x, atol=1e-9), solve
    s = IterativeSolver(ctx=ctx)
    got = s.solvePGMRES(A, SparseMatrix.identity(3, ctx), b, 1e-12)
    np.testing.assert_allclose(got, x, atol=1e-9)


@pytest.mark.parametrize("name", ["symm", "nonsymm", "good_nonsymm"])
def test_kat_gmres2(ctx, name):
    """GMResTest.java: GMRES2(1e-12).solve(A, b) and solve(A, I, b) equal solve(b)."""
    from jfem_b200.linalg import GMRES2, DenseMatrix
    k = kat()["systems"][name]
    a = np.array(k["A"], float)
    r, c = np.nonzero(a)
    A = SparseMatrix.from_coo(3, 3, r, c, a[r, c], ctx)
    b = np.array(k["b"], float)
    x = np.array(k["x"])
    np.testing.assert_allclose(GMRES2(1e-12, ctx).solve(A, b), x, atol=1e-9)
    np.testing.assert_allclose(GMRES2(1e-12, ctx).solve(A, SparseMatrix.identity(3, ctx), b), x, atol=1e-9)
    if name == "good_nonsymm":
        inv = DenseMatrix(a, ctx).inverse()
        ri, ci = np.nonzero(inv)
        Minv = SparseMatrix.from_coo(3, 3, ri, ci, inv[ri, ci], ctx)
        np.testing.assert_allclose(GMRES2(1e-12, ctx).solve(A, Minv, b), x, atol=1e-9)


def test_gmres2_fe_matches_oracle(ctx):
    from jfem_b200.linalg import GMRES2
    sp, sy = fe_system(1, 12)
    tol = 1e-9 * np.linalg.norm(sy.rhs)
    ref = O.solve_gmres2(coo_oracle(sy), sy.rhs, tol)
    g = GMRES2(tol, ctx)
    x = g.solve(dev(sy, ctx), sy.rhs)
    assert g.last.status == N.OK
    assert rel(x, ref.x) < 1e-7
    assert abs(g.iterations - ref.iterations) <= 2


def test_gmres_fe_matches_oracle(ctx):
    sp, sy = fe_system(1, 24)
    tol = 1e-10 * np.linalg.norm(sy.rhs)
    ref = O.solve_gmres(coo_oracle(sy), sy.rhs, tol, restart=30)
    s = IterativeSolver(ctx=ctx)
    s.gm.ITERATIONS_BEFORE_RESTART = 30
    x = s.solveGMRES(dev(sy, ctx), sy.rhs, tol)
    assert s.last.status == N.OK
    assert rel(x, ref.x) < REL
    assert abs(s.iterations - ref.iterations) <= 2


def test_pgmres_mg(ctx):
    h = mg_levels(1, 4, 4, mass=0.0)
    mats_o, mg_o, mats, mg = _mg_pair(h, ctx, (O.SMOOTH_RICHARDSON, 8, 0.1), 3, True)
    b = h.finest.rhs
    ref = O.solve_gmres(mats_o[-1], b, 1e-8, M=mg_o)
    s = IterativeSolver(ctx=ctx)
    x = s.solvePGMRES(mats[-1], mg, b, 1e-8)
    assert s.last.status == N.OK
    assert s.iterations < 10 and s.iterations == ref.iterations
    assert rel(x, ref.x) < REL


def test_bicgstab_fe_matches_oracle(ctx):
    sp, sy = fe_system(1, 20)
    tol = 1e-10 * np.linalg.norm(sy.rhs)
    ref = O.solve_bicgstab(coo_oracle(sy), sy.rhs, tol)
    s = IterativeSolver(ctx=ctx)
    x = s.solveBiCGStab(dev(sy, ctx), sy.rhs, tol)
    assert rel(x, ref.x) < REL
    # |rho| < tol ends BiCGStab in a GMRES fallback here (IterativeSolver.java:293-294)
    assert ref.status == O.BREAKDOWN
    assert abs(s.iterations - ref.iterations) <= 3


def test_pbicgstab_mg(ctx):
    h = mg_levels(2, 4, 3)
    mats_o, mg_o, mats, mg = _mg_pair(h, ctx, (O.SMOOTH_JACOBI, 2, 2.0 / 3.0), 1, False)
    b = h.finest.rhs
    tol = 1e-9 * np.linalg.norm(b)
    ref = O.solve_pbicgstab(mats_o[-1], mg_o, b, tol)
    s = IterativeSolver(ctx=ctx)
    x = s.solvePBiCGStab(mats[-1], mg, b, tol)
    assert rel(x, ref.x) < 1e-7
    assert abs(s.iterations - ref.iterations) <= 1


def test_nonfinite_rhs_status(ctx):
    sp, sy = fe_system(1, 8)
    b = sy.rhs.copy()
    b[5] = np.nan
    s = IterativeSolver(ctx=ctx)
    s.solveCG(dev(sy, ctx), b, 1e-10)
    assert s.last.status == N.NONFINITE


def test_not_pd_flag(ctx):
    a = np.diag([1.0, -2.0, 3.0])
    r, c = np.nonzero(a)
    A = SparseMatrix.from_coo(3, 3, r, c, a[r, c], ctx)
    s = IterativeSolver(ctx=ctx)
    s.solveCG(A, np.array([1.0, 1.0, 1.0]), 1e-12)
    assert s.last.not_pd


def test_iteration_cap(ctx):
    sp, sy = fe_system(1, 32)
    s = IterativeSolver(ctx=ctx)
    A = dev(sy, ctx)
    s._run(N.CG, A, None, sy.rhs, 1e-30, s._start(sy.n), maxit=7)
    assert s.last.status == N.NOT_CONVERGED and s.iterations == 7


def test_pcg_mg_full_size(ctx):
    """Q2 512x512 (1,050,625 dofs), 8 levels, Jacobi 2/2 omega=2/3: FP64 and
    mixed PCG reach the 1e-8 relative FP64 true residual and agree."""
    h = mg_levels(2, 4, 8, modes=16, seed=0)
    mats = [dev(s, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(7)]
    sm = JacobiSmoother(2, 2.0 / 3.0)
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [sm] * 7, cycles=1, use_fmg=False, precision="mixed",
                          ctx=ctx)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    s = IterativeSolver(ctx=ctx)
    x64 = s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK and s.last.final_residual <= tol
    it64 = s.iterations
    for mode in ("mixed", "mixed-precond"):
        s2 = IterativeSolver(ctx=ctx)
        s2.precision = mode
        x32 = s2.solvePCG(mats[-1], mg, b, tol)
        assert s2.last.status == N.OK and s2.last.final_residual <= tol, mode
        assert rel(x32, x64) < 1e-7, mode
    assert it64 <= 20


@pytest.mark.parametrize("precision", ["mixed-bf16", "mixed-fp16"])
def test_pcg_bf16_vcycle(ctx, precision):
    """FP64 PCG with the FP32 V-cycle reading BF16 or scaled-FP16 matrices
    (hierarchy precision "mixed-bf16" / "mixed-fp16"): same FP64 true
    residual, at most one extra iteration over the FP64 preconditioner."""
    h = mg_levels(2, 4, 6, modes=16, seed=3)    # Q2 128x128
    mats_o, mg_o, mats, mg = _mg_pair(h, ctx, (O.SMOOTH_JACOBI, 2, 2.0 / 3.0), 1, False, precision=precision)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_pcg(mats_o[-1], mg_o, b, tol)
    s = IterativeSolver(ctx=ctx)
    s.precision = "mixed-precond"
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK and s.last.final_residual <= tol
    assert rel(x, ref.x) < 1e-7
    assert s.iterations <= ref.iterations + 1
    if precision == "mixed-fp16":
        assert s.iterations == ref.iterations


def _fp16_rounded(dev_matrix):
    """The oracle matrix of the merged values rounded as the FP16 hierarchy
    stores them: fp16(a 2^k) / 2^k with max |a| 2^k in [2^14, 2^15)."""
    ri, ci, v = dev_matrix.coo()
    k = 15 - int(np.frexp(np.abs(v).max())[1])
    vh = (v * 2.0 ** k).astype(np.float16).astype(np.float64) / 2.0 ** k
    assert np.count_nonzero(vh) == np.count_nonzero(v)          # no entry flushed to zero
    return O.CooMatrix(dev_matrix.rows, dev_matrix.cols, ri, ci, vh)


def test_fp16_vcycle_matches_rounded_oracle(ctx):
    """Mixed PCG with the FP16 hierarchy against the oracle PCG whose V-cycle
    runs in FP64 on the same FP16-rounded matrices: same iterations, residual
    histories within 10 % (the GPU keeps the Jacobi diagonal and the coarsest
    inverse in full precision, the oracle's V-cycle takes them from the
    rounded matrices)."""
    h = mg_levels(2, 4, 5, modes=8, seed=2)
    mats_o, mg_o, mats, mg = _mg_pair(h, ctx, (O.SMOOTH_JACOBI, 2, 2.0 / 3.0), 1, False, precision="mixed-fp16")
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(len(h.systems) - 1)]
    mg_r = O.MGPreconditioner([_fp16_rounded(m) for m in mats], [_fp16_rounded(p) for p in prol], h.boundary,
                              [None] + [(O.SMOOTH_JACOBI, 2, 2.0 / 3.0)] * (len(mats) - 1), cycles=1, use_fmg=False)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_pcg(mats_o[-1], mg_r, b, tol)
    s = IterativeSolver(ctx=ctx)
    s.precision = "mixed-precond"
    s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK and s.iterations == ref.iterations
    assert len(s.last.history) == len(ref.history)
    np.testing.assert_allclose(s.last.history, ref.history, rtol=0.1)


def test_start_modes(ctx):
    """opts.start = 1 (e0) and 2 (zero) give the same solve as passing that
    start vector in x (start = 0)."""
    import ctypes as C
    sp, sy = fe_system(1, 24)
    A = dev(sy, ctx)
    b = sy.rhs
    n = sy.n
    for start, x0 in ((1, np.eye(1, n, 0)[0]), (2, np.zeros(n))):
        outs = []
        for mode in (0, start):
            o = N.SolverOpts()
            N.load().jfg_solver_opts_default(C.byref(o))
            o.tol = 1e-10 * np.linalg.norm(b)
            o.start = mode
            x = x0.copy() if mode == 0 else np.full(n, np.nan)
            info = N.SolveInfo()
            ctx.check(N.load().jfg_solve(ctx.handle, N.CG, A.handle, N.PREC_NONE, None, N.dptr(N.f64(b)),
                                         N.dptr(x), C.byref(o), C.byref(info)))
            outs.append((x, info.iterations))
        assert outs[0][1] == outs[1][1]
        assert np.array_equal(outs[0][0], outs[1][0])


@pytest.mark.parametrize("p,cells", [(1, 64), (2, 40), (1, 127)])
def test_cg_small_cluster_path(ctx, monkeypatch, p, cells):
    """Unpreconditioned CG of systems up to 16,384 rows runs in one cluster
    launch: same iterations as the oracle (+-2) and as the multi-kernel loop,
    solutions equal to rounding, the first residuals equal; the maxit and
    zero-iteration exits."""
    sp, sy = fe_system(p, cells)
    A = dev(sy, ctx)
    b = sy.rhs
    tol = 1e-10 * np.linalg.norm(b)
    ref = O.solve_cg(coo_oracle(sy), b, tol)
    out = {}
    for flag, smem in (("1", "1"), ("1", "0"), ("0", "1")):     # shared-memory variant, global variant, loop
        monkeypatch.setenv("JFEM_SMALL_CG", flag)
        monkeypatch.setenv("JFEM_SMALL_CG_SMEM", smem)
        s = IterativeSolver(ctx=ctx)
        x = s.solveCG(A, b, tol)
        out[flag + smem] = (x, s.iterations, s.last.status, s.last.history)
    x0, it0, st0, h0 = out["01"]
    assert st0 == N.OK
    for key in ("11", "10"):
        x1, it1, st1, h1 = out[key]
        assert st1 == N.OK
        assert abs(it1 - ref.iterations) <= 2 and abs(it1 - it0) <= 2
        assert rel(x1, ref.x) < 1e-8 and rel(x1, x0) < 1e-8
        # histories agree until rounding differences are amplified (as for the oracle)
        np.testing.assert_allclose(h1[:5], h0[:5], rtol=1e-7)
    monkeypatch.setenv("JFEM_SMALL_CG_SMEM", "1")
    monkeypatch.setenv("JFEM_SMALL_CG", "1")
    s = IterativeSolver(ctx=ctx)
    s._run(N.CG, A, None, b, 1e-30, s._start(len(b)), maxit=5)
    assert s.last.status == N.NOT_CONVERGED and s.iterations == 5
    s._run(N.CG, A, None, b, 1e300, s._start(len(b)))
    assert s.last.status == N.OK and s.iterations == 0
