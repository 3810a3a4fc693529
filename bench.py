"""Benchmark: time to a 1e-8 FP64 residual and SpMV GB/s on one B200.

Default workload (one "step" = one solve): -div(kappa grad u) = f on the unit
square, Q1 elements on a 1024x1024 cell grid (1,050,625 unknowns), kappa =
exp(g) with g a seeded Gaussian random field (squared-exponential
covariance, length 0.05, variance 1), zero Dirichlet data, f from 4x4 seeded
sine modes; 9-level geometric multigrid (coarse levels rediscretised with
2x2-averaged kappa), 2+2 damped-Jacobi sweeps (omega = 2/3), coarsest 4x4
cells solved by a dense FP64 inverse.  Arms, each a whole solve to
||b - A x|| <= 1e-8 ||b|| in FP64:

  fp64      plain FP64 GMG-PCG from e0 (the drop-in; the judge)
  mixed     FP64 PCG + FP32 V-cycle preconditioner
  fp16      FP64 PCG + V-cycle reading scaled-FP16 matrices (FP32 vectors)
  fgmres    FGMRES(30) + FP32 V-cycle
  learned   FGMRES(30) + FP32 V-cycle + learned smoother (the headline value)

The working set (FP64 finest matrix, hierarchy, vectors) is larger than L2,
so solves run back to back without a flush.  The Q2 512x512 -Lap u + 5u = f
GMG-PCG (the Q2 multigrid case, 8 levels) is timed too and reported as extra keys.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Under torchrun every rank solves its own replica (no data-path collective;
"replicas only"); the step time is the max over ranks.

The other configurations are measured with --workload (one JSON line each,
1 GPU, no reference arm): gmg-pcg (the Q2 512x512 case alone), cg-small,
batch-heat (256 uneven Q1 heat systems, 50 implicit-Euler steps in one
persistent launch), stokes (Taylor-Hood Q2/Q1 on 256x256 cells, GMRES(50)
with the block-diagonal preconditioner), galerkin, gs-pcg, assemble.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-8 residual (s) & SpMV GB/s: mixed+learned vs plain FP64 GMG-PCG, 1 B200"
WORKLOAD = "Q2 512x512 -Lap u + 5u = f, GMG-PCG to 1e-8 relative FP64 residual"
CELLS, P, LEVELS, MODES, SEED = 512, 2, 8, 16, 0
RTOL = 1e-8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=CELLS)
    ap.add_argument("--levels", type=int, default=LEVELS)
    ap.add_argument("--vcycle", default="fp32", choices=["fp32", "fp16", "bf16"],
                    help="storage of the V-cycle matrices of the mixed solve (FP32 vectors and sums in every case)")
    ap.add_argument("--workload", default="kappa",
                    choices=["kappa", "gmg-pcg", "cg-small", "batch-heat", "stokes", "learned", "galerkin", "gs-pcg",
                             "assemble"])
    ap.add_argument("--no-q2", action="store_true", help="kappa workload: skip the Q2 512x512 extra keys")
    ap.add_argument("--batch-systems", type=int, default=256,
                    help="batch-heat: number of systems (the configuration has 256; fewer only for profiling)")
    ap.add_argument("--heat-steps", type=int, default=50,
                    help="batch-heat: implicit-Euler steps (the configuration has 50; fewer only for profiling)")
    ap.add_argument("--profile", default=None,
                    choices=["solve-fp64", "solve-mixed", "solve-mixed-nograph", "gs-mixed-nograph", "spmv64", "spmv32",
                             "solve-learned", "solve-learned-nograph", "solve-fp64-nograph", "precond-apply"],
                    help="set up, run the named operation --warmup + 1 times and exit (for ncu captures)")
    return ap.parse_args()


def dist_env():
    from jfem_b200.replicas import dist_env as de
    return de()


class ClockSampler:
    """SM clocks and throttle reasons of the benchmarked GPU sampled every
    10 ms by NVML (the library behind nvidia-smi; read-only queries) on a
    background thread; summary() keeps the samples taken between
    mark_start() and mark_end().  When the timed region is shorter than a
    few sampling periods, extend() keeps the same work running (untimed)
    until three samples exist after mark_start().  Without NVML the clocks
    are reported as unavailable."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device):
        self.device = device
        self.samples = []          # (time, sm_mhz, max_mhz, power_w, reasons_mask)
        self.t0 = self.t1 = None
        self.extended = False
        self.source = None
        self._stop = None
        self._thread = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading
        try:
            nv, h = self._handle()
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._stop = threading.Event()

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append((time.time(), nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                             nv.nvmlDeviceGetPowerUsage(h) / 1000.0, int(reasons(h))))
                    except Exception:
                        pass
                    self._stop.wait(0.01)

            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
            self.source = "nvml"
        except Exception:
            self.source = None
        return self

    def __exit__(self, *a):
        if self._thread:
            self._stop.set()
            self._thread.join()

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def _inside(self):
        t0 = self.t0 if self.t0 is not None else 0.0
        t1 = self.t1 if self.t1 is not None else time.time()
        return [r for r in list(self.samples) if t0 - 0.005 <= r[0] <= t1 + 0.005]

    def extend(self, fn, min_samples=3, max_s=5.0):
        if not self.source or self.t0 is None:
            return
        t_stop = time.time() + max_s
        self.t1 = None
        while time.time() < t_stop and len(self._inside()) < min_samples:
            fn()
            self.extended = True
        self.t1 = time.time()

    def summary(self):
        if not self.source:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        rows = self._inside()
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        reasons = sorted({name for r in rows for name, bit in self.REASONS if r[4] & bit})
        out = {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows),
               "reasons": reasons, "samples": len(rows), "power_w_median": statistics.median(r[3] for r in rows),
               "source": self.source}
        if self.extended:
            out["note"] = "timed region shorter than the sampling period: the same solve kept running untimed"
        return out


def build_problem(cells, levels):
    from jfem_b200 import problems
    return problems.hierarchy(P, cells >> (levels - 1), levels, mass=5.0, modes=MODES, seed=SEED)


# DRAM bytes (read + write) of one cold launch of the FP32 finest-level SpMV of
# Q2 512x512 (n = 1,050,625, nnz = 16,707,665), 16-bit column offsets, from one
# ncu capture; it applies only to that matrix.
SPMV32_TRAFFIC_CASE = (1050625, 16707665)
SPMV32_TRAFFIC_BYTES = 109.13e6 + 4.55e6


def spmv_bytes(n, nnz, sval, sx):
    """Algorithmic CSR bytes: values + column indices + row pointers + x + y."""
    return nnz * (sval + 4) + (n + 1) * 4 + n * sx + n * sx


def run_ours(args):
    import torch
    from jfem_b200.replicas import Replicas
    reps = Replicas(timeout_s=120)
    rank, world, local = reps.rank, reps.world, reps.local
    torch.cuda.set_device(local)
    os.environ["JFEM_DEVICE"] = str(local)
    from jfem_b200 import IterativeSolver, JacobiSmoother, MGPreconditioner
    from jfem_b200 import _native as N
    from jfem_b200.linalg import DeviceMatrix
    import ctypes as C

    ctx = N.Context(local)
    HEADLINE = N.MIXED_PRECOND
    t0 = time.time()
    h = build_problem(args.cells, args.levels)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(args.levels - 1)]
    if args.profile == "gs-mixed-nograph":      # forward-backward Gauss-Seidel (1 run), multicolour
        from jfem_b200 import ForwardBackwardGaussSeidelSmoother
        sms = [None] + [ForwardBackwardGaussSeidelSmoother(1, mats[l], "multicolour") for l in range(1, args.levels)]
    else:
        sms = [None] + [JacobiSmoother(2, 2.0 / 3.0)] * (args.levels - 1)
    hier = {"fp32": "mixed", "fp16": "mixed-fp16", "bf16": "mixed-bf16"}[args.vcycle]
    mg = MGPreconditioner(mats, prol, h.boundary, sms, cycles=1, use_fmg=False, precision=hier, ctx=ctx)
    A = mats[-1]
    n = A.rows
    b_host = h.finest.rhs.copy()
    bnorm = float(np.linalg.norm(b_host))
    tol = RTOL * bnorm
    setup_s = time.time() - t0

    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    db = torch.from_numpy(b_host).to(f"cuda:{local}")
    e0 = torch.zeros(n, dtype=torch.float64, device=f"cuda:{local}")
    e0[0] = 1.0
    dx = torch.empty_like(e0)
    torch.cuda.synchronize()

    def opts(precision):
        o = N.SolverOpts()
        N.load().jfg_solver_opts_default(C.byref(o))
        o.tol = tol
        o.precision = precision
        o.inner_rtol = 1e-4
        return o

    info = N.SolveInfo()

    def solve_dev(precision, hierarchy=None):
        with torch.cuda.stream(stream):
            dx.copy_(e0)           # the reference's start vector e0
        o = opts(precision)
        if args.profile in ("solve-mixed-nograph", "gs-mixed-nograph"):
            o.use_graph = 0        # plain launches: every kernel of the solve is visible to a profiler
        g = mg if hierarchy is None else hierarchy
        st = N.load().jfg_solve_dev(ctx.handle, N.PCG, A.handle, N.PREC_MG, g.handle, C.c_void_p(db.data_ptr()),
                                    C.c_void_p(dx.data_ptr()), C.byref(o), C.byref(info))
        ctx.check(st)
        return info.iterations, info.final_residual, info.outer_iterations

    def barrier():
        reps.barrier()

    def max_over_ranks(v):
        return reps.max(v)

    def timed(fn, steps, warmup, clk=None):
        for _ in range(warmup):
            fn()
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if clk:
            clk.mark_start()
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        if clk:
            clk.mark_end()
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1) / steps)

    if args.profile:
        for _ in range(args.warmup + 1):
            if args.profile == "solve-fp64":
                solve_dev(N.FP64)
            elif args.profile in ("solve-mixed", "solve-mixed-nograph", "gs-mixed-nograph"):
                solve_dev(HEADLINE)
            else:
                A.time_spmv(precision=1 if args.profile == "spmv32" else 0, iters=1)
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "iterations": info.iterations}))
        return

    # FP64 judge (the plain drop-in) and the mixed-precision headline
    ms64 = timed(lambda: solve_dev(N.FP64), max(2, args.steps // 2), max(3, args.warmup))
    it64, res64, _ = solve_dev(N.FP64)
    x64 = dx.cpu().numpy().copy()
    # the other mixed mode (defect correction around FP32 inner PCG), reported beside
    ms_dc = timed(lambda: solve_dev(N.MIXED), max(2, args.steps // 2), max(3, args.warmup))
    it_dc, res_dc, outer_dc = solve_dev(N.MIXED)
    l0 = N.kernel_launches()
    with ClockSampler(local) as clk:
        ms = timed(lambda: solve_dev(HEADLINE), args.steps, args.warmup, clk)
        launches = (N.kernel_launches() - l0) / (args.steps + args.warmup)
        clk.extend(lambda: solve_dev(HEADLINE))
    itm, resm, outer = solve_dev(HEADLINE)
    xm = dx.cpu().numpy().copy()
    rel_err = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))
    # the same mixed solve with the V-cycle matrices stored as scaled FP16
    # (reported beside; FP32 vectors and sums, the same FP64 stopping test)
    alt = None
    if args.vcycle == "fp32":
        mg16 = MGPreconditioner(mats, prol, h.boundary, sms, cycles=1, use_fmg=False, precision="mixed-fp16",
                                ctx=ctx)
        ms16 = timed(lambda: solve_dev(HEADLINE, mg16), args.steps, args.warmup)
        it16, res16, _ = solve_dev(HEADLINE, mg16)
        x16 = dx.cpu().numpy().copy()
        alt = {"time_s": ms16 / 1e3, "iterations": it16, "final_rel_residual": res16 / bnorm,
               "rel_error_vs_fp64": float(np.linalg.norm(x16 - x64) / np.linalg.norm(x64)),
               "mode": "FP64 PCG + FP32 V-cycle reading scaled-FP16 matrices"}
        del mg16

    # end to end through the C ABI with host buffers (pinned), copies timed
    hb = torch.from_numpy(b_host).pin_memory()
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()

    def solve_host():
        o = opts(HEADLINE)
        o.start = 1                # e0, the reference's start vector, made on the device
        st = N.load().jfg_solve(ctx.handle, N.PCG, A.handle, N.PREC_MG, mg.handle,
                                C.cast(hb.data_ptr(), C.POINTER(C.c_double)),
                                C.cast(hx.data_ptr(), C.POINTER(C.c_double)), C.byref(o), C.byref(info))
        ctx.check(st)

    for _ in range(args.warmup):
        solve_host()
    barrier()
    t_e2e = time.perf_counter()
    for _ in range(args.steps):
        solve_host()
    e2e_s = (time.perf_counter() - t_e2e) / args.steps
    e2e_s = max_over_ranks(e2e_s)

    # dominant kernel: the finest-level SELL-32 SpMV (FP32 in the mixed solve),
    # timed with the L2 flushed before every launch
    nnz = A.nnz
    ms_spmv32 = A.time_spmv(precision=1, iters=50)
    ms_spmv64 = A.time_spmv(precision=0, iters=50)
    b32 = spmv_bytes(n, nnz, 4, 4)
    b64 = spmv_bytes(n, nnz, 8, 8)
    gbs32 = b32 / (ms_spmv32 * 1e-3) / 1e9
    gbs64 = b64 / (ms_spmv64 * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    cpu = None
    if rank == 0 and world == 1 and os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        cpu = cpu_baseline(h, tol)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": ms / 1e3,
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64",
            "data": "synthetic (seeded sine-mode source, assembled Q2 system)",
            "config": {"workload": WORKLOAD, "dofs": n, "nnz": int(nnz), "levels": args.levels,
                       "smoother": "Jacobi 2+2 omega=2/3", "coarse": "dense FP64 inverse 81x81",
                       "l2": "solve working set larger than L2 (FP64 finest matrix 167 MB + FP32 hierarchy); "
                             "roofline SpMV timed with the L2 flushed before each launch", "parallelism": f"replicas{world}"},
            "iterations": itm,
            "outer_iterations": outer,
            "final_rel_residual": resm / bnorm,
            "rel_error_vs_fp64": rel_err,
            "fp64_time_s": ms64 / 1e3,
            "fp64_iterations": it64,
            "fp64_final_rel_residual": res64 / bnorm,
            "speedup_vs_fp64": ms64 / ms,
            "mode": "FP64 PCG + FP32 V-cycle preconditioner" + {"fp32": "", "fp16": " (matrices stored as scaled FP16)",
                                                                   "bf16": " (matrices stored as BF16)"}[args.vcycle],
            "defect_correction": {"time_s": ms_dc / 1e3, "inner_iterations": it_dc, "outer_iterations": outer_dc,
                                  "final_rel_residual": res_dc / bnorm},
            "fp16_vcycle": alt,
            "spmv_gbs": {"fp64": gbs64, "fp32": gbs32},
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "path": "jfg_solve (C ABI) with pinned host rhs in and solution out; start e0 (opts.start=1)"},
            "gpu_launches": int(round(launches)),
            "roofline": {"bound": "hbm", "achieved": gbs32, "peak": peak, "unit": "GB/s", "frac": gbs32 / peak,
                         "traffic": SPMV32_TRAFFIC_BYTES if (n, nnz) == SPMV32_TRAFFIC_CASE else None,
                         "traffic_source": "constant from an earlier ncu capture of this kernel on this matrix "
                                           "(dram__bytes_read.sum + dram__bytes_write.sum, one cold launch); "
                                           "not measured in this run",
                         "kernel": "k_spmv_pipe<float> finest level", "peak_source": peak_src,
                         "bytes_per_launch": b32, "ms_per_launch": ms_spmv32},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "setup_s": setup_s,
        }
        print(json.dumps(line))
    reps.close()


KAPPA_CELLS, KAPPA_LEVELS, KAPPA_SEED = 1024, 9, 0
KAPPA_WORKLOAD = ("Q1 1024x1024 -div(kappa grad u) = f, kappa = exp(GRF l=0.05 var=1), 9-level GMG, "
                  "Jacobi 2+2, to 1e-8 relative FP64 residual")


def kappa_size(args):
    """(cells, levels) of the kappa workload: 1024^2 cells and 9 levels unless
    --cells / --levels are given (the coarsest grid stays 4x4 cells)."""
    if args.cells != CELLS:
        return args.cells, int(round(np.log2(args.cells // 4))) + 1
    return KAPPA_CELLS, KAPPA_LEVELS


def layout_bytes(A, sval, sx):
    """Algorithmic bytes of one product in the layout the library picked:
    values-only stencil rows (9 values, no indices) + CSR rows (values,
    columns, row list and pointers) + x read once + y written once; the CSR
    formula when the matrix has no stencil layout."""
    lay = A.layout()
    n = A.rows
    if not lay["stencil"]:
        return spmv_bytes(n, A.nnz, sval, sx), lay
    b = 9 * lay["regular_rows"] * sval + lay["other_nnz"] * (sval + 4) + lay["other_rows"] * 4 \
        + (lay["other_rows"] + 1) * 4 + n * sx + n * sx
    return b, lay


def run_kappa(args):
    import ctypes as C
    import torch
    from jfem_b200.replicas import Replicas
    reps = Replicas(timeout_s=120)
    rank, world, local = reps.rank, reps.world, reps.local
    torch.cuda.set_device(local)
    os.environ["JFEM_DEVICE"] = str(local)
    from jfem_b200 import _native as N
    from jfem_b200.cnn import LearnedSmoother
    from jfem_b200.learned import WEIGHTS, KappaSystem
    from jfem_b200.multigrid import JacobiSmoother, MGPreconditioner

    ctx = N.Context(local)
    t0 = time.time()
    ks = KappaSystem(ctx, kappa_size(args)[0], kseed=KAPPA_SEED)
    L = len(ks.mats)
    mg16 = MGPreconditioner(ks.mats, ks._prol, ks.h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (L - 1),
                            cycles=1, use_fmg=False, precision="mixed-fp16", ctx=ctx)
    net = LearnedSmoother(ctx, weights=np.load(WEIGHTS))
    pc_v = ks.preconditioner(net, use_net=False)
    pc_net = ks.preconditioner(net, use_net=True)
    A = ks.A
    n = ks.n
    b_host = ks.b.copy()
    bnorm = float(np.linalg.norm(b_host))
    tol = RTOL * bnorm
    setup_s = time.time() - t0

    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    dev = f"cuda:{local}"
    db = torch.from_numpy(b_host).to(dev)
    e0 = torch.zeros(n, dtype=torch.float64, device=dev)
    e0[0] = 1.0
    z0 = torch.zeros(n, dtype=torch.float64, device=dev)
    dx = torch.empty_like(e0)
    torch.cuda.synchronize()
    info = N.SolveInfo()
    arms = {
        "fp64": (N.PCG, N.PREC_MG, ks.mg, N.FP64, e0, "FP64 GMG-PCG from e0 (the plain drop-in)"),
        "mixed": (N.PCG, N.PREC_MG, ks.mg, N.MIXED_PRECOND, e0, "FP64 PCG + FP32 V-cycle, from e0"),
        "fp16": (N.PCG, N.PREC_MG, mg16, N.MIXED_PRECOND, e0,
                 "FP64 PCG + V-cycle reading scaled-FP16 matrices (FP32 vectors and sums), from e0"),
        "fgmres": (N.FGMRES, N.PREC_MG_CNN, pc_v, N.FP64, z0, "FGMRES(30) + FP32 V-cycle, from zero"),
        "learned": (N.FGMRES, N.PREC_MG_CNN, pc_net, N.FP64, z0,
                    "FGMRES(30) + FP32 V-cycle + learned smoother (BF16 network), from zero"),
    }
    HEAD = "learned"

    def opts(precision, graph=True):
        o = N.SolverOpts()
        N.load().jfg_solver_opts_default(C.byref(o))
        o.tol = tol
        o.precision = precision
        o.inner_rtol = 1e-4
        o.restart = 30
        o.use_graph = 1 if graph else 0
        return o

    def solve_dev(arm, graph=True):
        kind, pk, pc, prec, start, _ = arms[arm]
        with torch.cuda.stream(stream):
            dx.copy_(start)
        st = N.load().jfg_solve_dev(ctx.handle, kind, A.handle, pk, pc.handle, C.c_void_p(db.data_ptr()),
                                    C.c_void_p(dx.data_ptr()), C.byref(opts(prec, graph)), C.byref(info))
        ctx.check(st)
        return info.iterations

    def timed(fn, steps, warmup, clk=None):
        for _ in range(warmup):
            fn()
        reps.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if clk:
            clk.mark_start()
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        if clk:
            clk.mark_end()
        reps.barrier()
        return reps.max(ev0.elapsed_time(ev1) / steps)

    if args.profile:
        name = {"solve-learned": ("learned", True), "solve-learned-nograph": ("learned", False),
                "solve-fp64": ("fp64", True), "solve-fp64-nograph": ("fp64", False),
                "solve-mixed": ("mixed", True), "solve-mixed-nograph": ("mixed", False)}.get(args.profile)
        for _ in range(args.warmup + 1):
            if name:
                solve_dev(name[0], name[1])
            else:
                A.time_spmv(precision=1 if args.profile == "spmv32" else 0, iters=1)
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "iterations": info.iterations}))
        reps.close()
        return

    out = {}
    x64 = None
    for arm in ("fp64", "mixed", "fp16", "fgmres"):
        ms_a = timed(lambda a=arm: solve_dev(a), max(2, args.steps // 2), max(3, args.warmup))
        it = solve_dev(arm)
        x = dx.cpu().numpy().copy()
        r = float(np.linalg.norm(b_host - A.spmv(x)))
        if arm == "fp64":
            x64 = x
        out[arm] = {"time_s": ms_a / 1e3, "iterations": it, "true_rel_residual": r / bnorm,
                    "rel_error_vs_fp64": float(np.linalg.norm(x - x64) / np.linalg.norm(x64)),
                    "mode": arms[arm][5]}
    l0 = N.kernel_launches()
    with ClockSampler(local) as clk:
        ms = timed(lambda: solve_dev(HEAD), args.steps, args.warmup, clk)
        launches = (N.kernel_launches() - l0) / (args.steps + args.warmup)
        clk.extend(lambda: solve_dev(HEAD))
    it_h = solve_dev(HEAD)
    xh = dx.cpu().numpy().copy()
    out[HEAD] = {"time_s": ms / 1e3, "iterations": it_h,
                 "true_rel_residual": float(np.linalg.norm(b_host - A.spmv(xh))) / bnorm,
                 "rel_error_vs_fp64": float(np.linalg.norm(xh - x64) / np.linalg.norm(x64)), "mode": arms[HEAD][5]}
    for a in out:
        out[a]["speedup_vs_fp64"] = out["fp64"]["time_s"] / out[a]["time_s"]

    # end to end through the C ABI with host buffers (pinned): rhs in, solution out
    hb = torch.from_numpy(b_host).pin_memory()
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()
    kind, pk, pc, prec, _, _ = arms[HEAD]

    def solve_host():
        o = opts(prec)
        o.start = 2                 # zero start, made on the device (FGMRES starts from zero)
        st = N.load().jfg_solve(ctx.handle, kind, A.handle, pk, pc.handle, C.cast(hb.data_ptr(), C.POINTER(C.c_double)),
                                C.cast(hx.data_ptr(), C.POINTER(C.c_double)), C.byref(o), C.byref(info))
        ctx.check(st)

    for _ in range(args.warmup):
        solve_host()
    reps.barrier()
    t_e2e = time.perf_counter()
    for _ in range(args.steps):
        solve_host()
    e2e_s = reps.max((time.perf_counter() - t_e2e) / args.steps)

    # dominant kernel: the finest-level product with FP32 values (the V-cycle's
    # smoothing sweeps and residuals).  Timed two ways: back to back over four
    # copies of the finest matrix taken in turn (185 MB of FP32 layout bytes,
    # more than the L2, so every launch reads its matrix from HBM; the launches
    # overlap their ramps as in a solve), and one launch at a time with the L2
    # flushed before it and events around it.
    from jfem_b200.linalg import DeviceMatrix
    sy = ks.h.finest
    copies = [A] + [DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx) for _ in range(3)]
    ms_spmv32 = DeviceMatrix.time_spmv_rotating(copies, precision=1, iters=20)
    ms_spmv64 = DeviceMatrix.time_spmv_rotating(copies, precision=0, iters=20)
    del copies
    ms_cold32 = A.time_spmv(precision=1, iters=50)
    ms_cold64 = A.time_spmv(precision=0, iters=50)
    b32, lay = layout_bytes(A, 4, 4)
    b64, _ = layout_bytes(A, 8, 8)
    gbs32 = b32 / (ms_spmv32 * 1e-3) / 1e9
    gbs64 = b64 / (ms_spmv64 * 1e-3) / 1e9
    csr32 = spmv_bytes(n, A.nnz, 4, 4) / (ms_spmv32 * 1e-3) / 1e9
    csr64 = spmv_bytes(n, A.nnz, 8, 8) / (ms_spmv64 * 1e-3) / 1e9
    cold = {"fp32_gbs": b32 / (ms_cold32 * 1e-3) / 1e9, "fp64_gbs": b64 / (ms_cold64 * 1e-3) / 1e9,
            "fp32_ms": ms_cold32, "fp64_ms": ms_cold64,
            "timing": "one launch between CUDA events, L2 flushed (256 MB read) before each"}
    peaks = _peaks()
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    q2 = None
    if not args.no_q2:
        q2 = q2_extra(ctx, reps, stream, args)

    cpu = None
    if rank == 0 and world == 1 and os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        cpu = cpu_baseline(ks.h, tol)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": ms / 1e3,
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "bf16+f32+f64",
            "data": "synthetic (seeded GRF kappa and sine-mode source, assembled Q1 system)",
            "config": {"workload": KAPPA_WORKLOAD, "dofs": n, "nnz": int(A.nnz), "levels": L,
                       "smoother": "Jacobi 2+2 omega=2/3", "coarse": "dense FP64 inverse 25x25",
                       "network": "6-layer 3x3 conv, 32 channels, BF16 weights, FP32 accumulation",
                       "l2": "solve working set larger than L2 (FP64 finest matrix + hierarchy + vectors); "
                             "roofline SpMV over four copies of the finest matrix taken in turn (inputs larger "
                             "than L2)",
                       "parallelism": f"replicas{world}"},
            "iterations": it_h,
            "final_rel_residual": out[HEAD]["true_rel_residual"],
            "rel_error_vs_fp64": out[HEAD]["rel_error_vs_fp64"],
            "mode": arms[HEAD][5],
            "speedup_vs_fp64": out["fp64"]["time_s"] / (ms / 1e3),
            "fp64_time_s": out["fp64"]["time_s"],
            "arms": out,
            "spmv_gbs": {"fp64": gbs64, "fp32": gbs32, "fp64_csr_equivalent": csr64, "fp32_csr_equivalent": csr32,
                         "layout": lay, "cold_single_launch": cold},
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "path": "jfg_solve (C ABI), FGMRES + V-cycle + network, pinned host rhs in and solution out"},
            "gpu_launches": int(round(launches)),
            "roofline": {"bound": "hbm", "achieved": gbs32, "peak": peak, "unit": "GB/s", "frac": gbs32 / peak,
                         "traffic": None,
                         "kernel": "k_spmv_st<float> (values-only 9-point layout), finest level",
                         "timing": "20 rounds of 4 back-to-back launches over 4 matrix copies, one event pair",
                         "peak_source": peak_src, "bytes_per_launch": b32, "ms_per_launch": ms_spmv32},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "q2_512_gmg_pcg": q2,
            "setup_s": setup_s,
        }
        if KAPPA_TRAFFIC.get("case") == (n, int(A.nnz)):
            line["roofline"]["traffic"] = KAPPA_TRAFFIC["bytes"]
            line["roofline"]["traffic_source"] = KAPPA_TRAFFIC["source"]
        print(json.dumps(line))
    reps.close()


# DRAM bytes (read + write) of one cold launch of the FP32 finest-level product
# of the kappa workload (k_spmv_st), from an ncu capture of that launch: a
# constant of an earlier capture, not measured by this script.
KAPPA_TRAFFIC = {"case": (1050625, 9410585), "bytes": 42063360,
                 "source": "ncu capture of one cold k_spmv_st<float> launch on this matrix "
                           "(dram__bytes_read.sum 42.058 MB + dram__bytes_write.sum 5 KB); a constant, "
                           "not measured in this run"}


def q2_extra(ctx, reps, stream, args):
    """The Q2 512x512 -Lap u + 5u = f GMG-PCG (FP64, FP64 PCG + FP32
    V-cycle, and FP64 PCG + V-cycle reading scaled-FP16 matrices, from e0),
    timed like the arms of the main line."""
    import ctypes as C
    import torch
    from jfem_b200 import _native as N
    from jfem_b200.linalg import DeviceMatrix
    from jfem_b200.multigrid import JacobiSmoother, MGPreconditioner
    h = build_problem(CELLS, LEVELS)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(LEVELS - 1)]
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (LEVELS - 1), cycles=1,
                          use_fmg=False, precision="mixed", ctx=ctx)
    mg16 = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (LEVELS - 1), cycles=1,
                            use_fmg=False, precision="mixed-fp16", ctx=ctx)
    A = mats[-1]
    n = A.rows
    b = torch.from_numpy(h.finest.rhs).cuda()
    tol = RTOL * float(np.linalg.norm(h.finest.rhs))
    e0 = torch.zeros(n, dtype=torch.float64, device="cuda")
    e0[0] = 1.0
    dx = torch.empty_like(e0)
    info = N.SolveInfo()
    res = {}
    for name, prec, pm in (("fp64", N.FP64, mg), ("mixed", N.MIXED_PRECOND, mg), ("fp16", N.MIXED_PRECOND, mg16)):
        def once():
            with torch.cuda.stream(stream):
                dx.copy_(e0)
            o = N.SolverOpts()
            N.load().jfg_solver_opts_default(C.byref(o))
            o.tol = tol
            o.precision = prec
            ctx.check(N.load().jfg_solve_dev(ctx.handle, N.PCG, A.handle, N.PREC_MG, pm.handle,
                                             C.c_void_p(b.data_ptr()), C.c_void_p(dx.data_ptr()), C.byref(o),
                                             C.byref(info)))
        for _ in range(max(3, args.warmup)):
            once()
        reps.barrier()
        torch.cuda.synchronize()
        e_0 = torch.cuda.Event(enable_timing=True)
        e_1 = torch.cuda.Event(enable_timing=True)
        k = max(2, args.steps // 2)
        e_0.record(stream)
        for _ in range(k):
            once()
        e_1.record(stream)
        e_1.synchronize()
        res[name] = {"time_s": reps.max(e_0.elapsed_time(e_1) / k) / 1e3, "iterations": info.iterations,
                     "final_rel_residual": info.final_residual / float(np.linalg.norm(h.finest.rhs))}
    ms32 = A.time_spmv(precision=1, iters=20)
    res["workload"] = WORKLOAD
    res["speedup_mixed_vs_fp64"] = res["fp64"]["time_s"] / res["mixed"]["time_s"]
    res["speedup_fp16_vs_fp64"] = res["fp64"]["time_s"] / res["fp16"]["time_s"]
    res["spmv_fp32_gbs"] = spmv_bytes(n, A.nnz, 4, 4) / (ms32 * 1e-3) / 1e9
    return res


def oracle_threads():
    """All host threads this process may use, for the oracle loops the
    reference runs as parallel streams (restriction, GMRES factors, Schwarz
    patches of a colour); the COO SpMV and the vector updates stay serial as
    in the reference."""
    import oracle as O
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        n = os.cpu_count() or 1
    return O.set_threads(n)


def oracle_gmg(h):
    import oracle as O
    mats = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    mg = O.MGPreconditioner(mats, prol, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2.0 / 3.0)] * (len(mats) - 1),
                            cycles=1, use_fmg=False)
    return mats, mg


def cpu_baseline(h, tol):
    """The oracle (C restatement of the reference's FP64 PCG + GMG V-cycle)
    timed on one whole solve from e0, on all host threads for the loops the
    reference runs as parallel streams."""
    import oracle as O
    mats, mg = oracle_gmg(h)
    cores = oracle_threads()
    t0 = time.perf_counter()
    ref = O.solve_pcg(mats[-1], mg, h.finest.rhs, tol)
    t = time.perf_counter() - t0
    return {"value": t, "unit": "s", "cores": cores, "kind": "port",
            "sample": f"one whole FP64 GMG-PCG solve ({ref.iterations} iterations) of the same system"}


def run_reference(args):
    """The reference arm: the oracle (C restatement of the reference's Java
    FP64 GMG-PCG: COO scatter SpMV, the V-cycle with Jacobi 2+2, PCG from e0)
    on the host cores, one whole solve per step, on the same system as the
    default line (Q1 1024^2 kappa-GRF), or on Q2 512^2 with --workload gmg-pcg."""
    rank, world, local = dist_env()
    if world > 1 and rank != 0:
        return
    import oracle as O
    if args.workload == "gmg-pcg":
        h = build_problem(args.cells, args.levels)
        workload, data = WORKLOAD, "synthetic (seeded sine-mode source, assembled Q2 system)"
    else:
        from jfem_b200 import problems
        kc, kl = kappa_size(args)
        h, _ = problems.kappa_hierarchy(1, kc >> (kl - 1), kl, 0.05, 1.0, kseed=KAPPA_SEED)
        workload, data = KAPPA_WORKLOAD, "synthetic (seeded GRF kappa and sine-mode source, assembled Q1 system)"
    mats, mg = oracle_gmg(h)
    b = h.finest.rhs
    tol = RTOL * float(np.linalg.norm(b))
    cores = oracle_threads()
    # each step is one whole FP64 GMG-PCG solve from e0 (the COO scatter SpMV
    # serial as in the reference, the restriction on all cores)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        full = O.solve_pcg(mats[-1], mg, b, tol)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    val = statistics.mean(times)
    line = {"metric": METRIC, "value": val, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": val * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": data,
            "config": {"workload": workload, "dofs": int(h.finest.n), "parallelism": "cpu"},
            "impl": "reference",
            "iterations": full.iterations,
            "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "port",
                             "sample": f"one whole solve per step ({full.iterations} PCG iterations)"},
            "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def run_cg_small(args):
    """-Lap u + 5u = f, Q1 on 64 x 64 cells (4,225 unknowns), 4 x 4 seeded sine
    modes, unpreconditioned CG to 1e-10 * ||b|| from e0, FP64; the oracle CG
    is timed on the whole solve beside it."""
    import torch
    from jfem_b200 import _native as N
    from jfem_b200.linalg import DeviceMatrix, IterativeSolver
    ctx = N.default_context()
    h = problems_hierarchy(1, 64, 1, modes=4)
    s = h.finest
    A = DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx)
    b = torch.tensor(s.rhs, device="cuda")
    tol = 1e-10 * float(np.linalg.norm(s.rhs))
    e0 = torch.zeros_like(b)
    e0[0] = 1.0
    solver = IterativeSolver(ctx=ctx)
    ms = []
    with ClockSampler(0) as clk:
        for i in range(max(3, args.warmup) + args.steps):
            x = e0.clone()
            torch.cuda.synchronize()
            if i == max(3, args.warmup):
                clk.mark_start()
            t0 = time.perf_counter()
            solver.solve_device(N.CG, A, None, b, x, tol)
            torch.cuda.synchronize()
            if i >= max(3, args.warmup):
                ms.append((time.perf_counter() - t0) * 1e3)
        clk.mark_end()
    it = solver.iterations
    res = float(np.linalg.norm(s.rhs - A.spmv(x.cpu().numpy())))
    cpu = None
    if os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        import oracle as O
        Ao = O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals)
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            ref = O.solve_cg(Ao, s.rhs, tol)
            ts.append(time.perf_counter() - t0)
        cpu = {"value": statistics.median(ts), "unit": "s", "cores": 1, "kind": "port",
               "sample": "the whole CG solve (median of 5); serial: the reference's CG has no parallel loop",
               "iterations": ref.iterations}
    line = {"metric": "time-to-1e-10 residual (s), unpreconditioned CG", "value": statistics.median(ms) / 1e3,
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median(ms), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 4x4 sine-mode source)",
            "config": {"workload": "cg-small: -Lap u + 5u = f, Q1 64x64 cells, CG to 1e-10 ||b|| from e0",
                       "dofs": s.n, "nnz": int(A.nnz)},
            "iterations": it, "final_rel_residual": res / float(np.linalg.norm(s.rhs)),
            "clocks": clk.summary(), "cpu_baseline": cpu}
    print(json.dumps(line))


def run_galerkin(args):
    """Set-up of an AMG-from-matrix hierarchy: the Galerkin coarse systems
    (P^T A) P of the Q2 512x512 finest matrix down 8 levels on the GPU
    (AMGFromMatrix), timed per hierarchy; the oracle builds the same chain on
    the host.  A check: on interior nodes the Galerkin operator of nested
    conforming spaces equals the assembled coarse operator."""
    import torch
    from jfem_b200 import _native as N
    from jfem_b200.linalg import DeviceMatrix
    ctx = N.default_context()
    h = build_problem(args.cells, args.levels)
    L = len(h.systems)
    fine = h.finest
    A = DeviceMatrix(fine.n, fine.n, fine.rows, fine.cols, fine.vals, ctx)
    P = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]

    def chain():
        out, M = [], A
        for l in range(L - 2, -1, -1):
            M = M.galerkin(P[l])
            out.append(M)
        return out

    for _ in range(max(1, args.warmup)):
        chain()
    ts = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        levels = chain()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    # interior rows and columns of the first coarse level against the assembled matrix
    C = levels[0]
    sc = h.systems[L - 2]
    Ac = DeviceMatrix(sc.n, sc.n, sc.rows, sc.cols, sc.vals, ctx)
    inner = np.ones(sc.n, bool)
    inner[np.asarray(h.boundary[L - 2], dtype=np.int64)] = False
    x = np.where(inner, np.random.default_rng(0).standard_normal(sc.n), 0.0)
    d = np.where(inner, C.spmv(x) - Ac.spmv(x), 0.0)
    rel = float(np.linalg.norm(d) / np.linalg.norm(np.where(inner, Ac.spmv(x), 0.0)))
    cpu = None
    if os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        import oracle as O
        Ao = O.CooMatrix(fine.n, fine.n, *A.coo())
        Po = [O.CooMatrix(p.rows, p.cols, *p.coo()) for p in P]
        t0 = time.perf_counter()
        M = Ao
        for l in range(L - 2, -1, -1):
            M = Po[l].tmmul(M).mmmul(Po[l])
        t = time.perf_counter() - t0
        cpu = {"value": t, "unit": "s", "cores": 1, "kind": "port",
               "sample": "the whole chain, Gustavson restatement of SparseMatrix.mmMul (the reference's own "
                         "mmMul loops over every column of B for every row of A)"}
    line = {"metric": "time to build the Galerkin coarse systems (s)", "value": statistics.median(ts), "unit": "s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (assembled Q2 system)",
            "config": {"workload": f"galerkin: (P^T A) P, Q2 {args.cells}x{args.cells}, {L} levels",
                       "dofs": fine.n, "nnz": int(A.nnz)},
            "coarse_nnz": [int(m.nnz) for m in levels],
            "interior_rel_diff_vs_assembled": rel, "cpu_baseline": cpu}
    print(json.dumps(line))


def run_gs_pcg(args):
    """The GMG-PCG solve of the Q2 512x512 system with forward-backward
    Gauss-Seidel smoothing (1 run pre and post) in the multicolour and the
    natural ordering, against Jacobi 2 + 2; FP64 and mixed (FP32 V-cycle)."""
    import torch
    from jfem_b200 import _native as N
    from jfem_b200.linalg import DeviceMatrix, IterativeSolver
    from jfem_b200.multigrid import ForwardBackwardGaussSeidelSmoother, JacobiSmoother, MGPreconditioner
    ctx = N.default_context()
    h = build_problem(args.cells, args.levels)
    L = len(h.systems)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    b = torch.tensor(h.finest.rhs, device="cuda")
    tol = RTOL * float(np.linalg.norm(h.finest.rhs))
    out = {}
    variants = [("jacobi_2_2", lambda A: JacobiSmoother(2, 2 / 3)),
                ("fbgs_1_multicolour", lambda A: ForwardBackwardGaussSeidelSmoother(1, A, "multicolour")),
                ("fbgs_1_natural", lambda A: ForwardBackwardGaussSeidelSmoother(1, A, "natural"))]
    for name, make in variants:
        t0 = time.perf_counter()
        sms = [None] + [make(mats[l]) for l in range(1, L)]
        setup = time.perf_counter() - t0
        mg = MGPreconditioner(mats, prol, h.boundary, sms, cycles=1, use_fmg=False, precision="mixed", ctx=ctx)
        info = sms[-1].info() if hasattr(sms[-1], "info") else None
        for prec in ("fp64", "mixed-precond"):
            s = IterativeSolver(ctx=ctx)
            s.precision = prec
            best = None
            for _ in range(max(1, args.warmup) + max(1, args.steps // 3)):
                x = torch.zeros_like(b)
                x[0] = 1.0
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                s.solve_device(N.PCG, mats[-1], mg, b, x, tol)
                torch.cuda.synchronize()
                dt = time.perf_counter() - t1
                best = dt if best is None else min(best, dt)
            r = float(torch.linalg.vector_norm(b - mats[-1].spmv_dev(x)).item())
            out[f"{name}/{prec}"] = {"time_s": best, "iterations": s.iterations, "status": N.STATUS_NAMES[s.last.status],
                                     "true_rel_residual": r / float(torch.linalg.vector_norm(b).item()),
                                     "smoother_setup_s": setup, "finest_levels_fwd_bwd_colours": info}
    line = {"metric": "time-to-1e-8 residual (s), GMG-PCG with Gauss-Seidel smoothing",
            "value": out["fbgs_1_multicolour/mixed-precond"]["time_s"], "unit": "s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic (seeded sine-mode source, assembled Q2 system)",
            "config": {"workload": f"gs-pcg: Q2 {args.cells}x{args.cells}, {L} levels, FBGS(1) vs Jacobi 2+2",
                       "dofs": int(h.finest.n)},
            "variants": out}
    print(json.dumps(line))


def run_assemble(args):
    """Assembly of the Q2 512x512 system (GRAD_GRAD + 5 VALUE_VALUE, 16 x 16
    sine-mode source, zero Dirichlet data) on the GPU (jfg_assemble_tp: host
    source values at the Gauss points in, device matrix and host rhs out)
    against the host numpy assembler of the same system."""
    import ctypes as C
    import torch
    from jfem_b200 import _native as N
    from jfem_b200.assembly import Space, assemble
    from jfem_b200.problems import modes_source
    ctx = N.default_context()
    sp = Space(P, args.cells, args.cells)
    f, _ = modes_source(MODES, SEED)
    X, Y = sp.quadrature_points()
    fq = np.ascontiguousarray(f(X, Y))
    d = N.TPDesc(P, args.cells, args.cells, 0.0, 1.0, 0.0, 1.0, 1.0, 5.0, 1)
    n = sp.nx * sp.ny
    rhs = np.empty(n)

    def once():
        h = C.c_void_p()
        ctx.check(N.load().jfg_assemble_tp(ctx.handle, C.byref(d), None, N.dptr(fq), C.byref(h), N.dptr(rhs),
                                           None, None))
        N.load().jfg_matrix_free(h)

    for _ in range(max(1, args.warmup)):
        once()
    ts = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        once()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    cpu = None
    if os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        t0 = time.perf_counter()
        assemble(sp, 1.0, 5.0, source=lambda X, Y: fq)
        cpu = {"value": time.perf_counter() - t0, "unit": "s", "cores": 1, "kind": "port",
               "sample": "the whole host numpy assembly of the same system, the same source values at the Gauss "
                         "points given"}
    line = {"metric": "time to assemble the system (s)", "value": statistics.median(ts), "unit": "s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (16 x 16 seeded sine modes)",
            "config": {"workload": f"assemble: Q{P} {args.cells}x{args.cells}, GRAD_GRAD + 5 VALUE_VALUE",
                       "dofs": n, "cell_triples": args.cells * args.cells * (P + 1) ** 4},
            "note": "GPU time: source values at the Gauss points already on the host (52 MB copied in), the "
                    "matrix merged on the device, the rhs copied out", "cpu_baseline": cpu}
    print(json.dumps(line))


def problems_hierarchy(p, cells, levels, modes):
    from jfem_b200 import problems
    return problems.hierarchy(p, cells >> (levels - 1), levels, mass=5.0, modes=modes, seed=SEED)


def run_batch_heat(args):
    """256 Q1 heat systems, cells drawn from {32, 48, ..., 256}^2,
    dt = 1e-3, 50 implicit-Euler steps, FP32 PCG + FP64 refinement to 1e-10."""
    import torch
    from jfem_b200 import _native as N
    from jfem_b200 import problems
    from jfem_b200.batch import BatchedParabolicIntegrator
    from jfem_b200.linalg import DeviceMatrix
    ctx = N.default_context()
    batch = problems.heat_batch(nsys=args.batch_systems, dt=1e-3, seed=0)
    K = [DeviceMatrix(s.K.n, s.K.n, s.K.rows, s.K.cols, s.K.vals, ctx) for s in batch]
    M = [DeviceMatrix(s.M.n, s.M.n, s.M.rows, s.M.cols, s.M.vals, ctx) for s in batch]
    B = BatchedParabolicIntegrator(K, M, ctx)
    u0 = B.pack([s.u0 for s in batch])
    steps = args.heat_steps
    for _ in range(max(3, args.warmup)):
        B.timeSteps(u0, steps)
    ms = []
    with ClockSampler(0) as clk:
        clk.mark_start()
        for _ in range(args.steps):
            t0 = time.perf_counter()
            B.timeSteps(u0, steps)
            ms.append((time.perf_counter() - t0) * 1e3)
        clk.mark_end()
    last = B.last
    dofs = int(sum(s.K.n for s in batch))
    nnz = int(sum(s.K.nnz for s in batch))
    cpu = None
    if os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        import oracle as O
        pick = list(range(0, len(batch), 32))
        t0 = time.perf_counter()
        n_s = 0
        for i in pick:
            s = batch[i]
            Ko = O.CooMatrix(s.K.n, s.K.n, s.K.rows, s.K.cols, s.K.vals)
            Mo = O.CooMatrix(s.M.n, s.M.n, s.M.rows, s.M.cols, s.M.vals)
            rhs = Mo.mvmul(s.u0)
            O.solve_cg(Ko, rhs, 1e-10 * np.linalg.norm(rhs), x0=s.u0)
            n_s += s.K.n
        t = time.perf_counter() - t0
        cpu = {"value": t / n_s * dofs * steps, "unit": "s", "cores": 1, "kind": "port",
               "sample": f"one CG step (1e-10) of {len(pick)} systems, scaled by unknowns to {len(batch)} systems x "
                         f"{steps} steps; "
                         "serial: the reference's CG has no parallel loop"}
    line = {"metric": f"time for {steps} implicit-Euler steps of {len(batch)} uneven Q1 heat systems (s)",
            "value": statistics.median(ms) / 1e3, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.median(ms), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded bumps)",
            "config": {"workload": f"batch-heat: {len(batch)} Q1 systems, cells {{32..256 step 16}}^2, dt=1e-3, "
                                   f"{steps} steps",
                                   "systems": len(batch), "steps": steps, "dofs": dofs, "nnz": nnz},
            "kernel_ms": last.ms, "total_inner_iterations": last.total_inner_iterations,
            "max_rel_residual": last.max_rel_residual, "failed": last.failed,
            "cluster": last.cluster, "threads": last.threads, "rows_per_thread": last.rows_per_thread, "clocks": clk.summary(), "cpu_baseline": cpu}
    print(json.dumps(line))


def stokes_cpu_sample(cells=64):
    """The oracle (GMRES(50) + block-diagonal preconditioner with the coloured
    Schwarz-smoothed velocity V-cycle, one host thread) solved whole on a
    smaller Taylor-Hood grid; the per-iteration time is scaled by unknowns to
    the full grid.  The Schwarz patches and colours come from the GPU solver's
    own decomposition of that grid."""
    import oracle as O
    from jfem_b200 import _native as N
    from jfem_b200.stokes import StokesSolver, stokes_problem
    prob = stokes_problem(cells, 4, seed=0, pin_pressure=False)
    sol = StokesSolver(N.default_context(), prob)
    L = len(prob.spaces)
    t0 = time.perf_counter()
    mats = [O.CooMatrix(t.nv, t.nv, *prob.velocity_blocks[l]) for l, t in enumerate(prob.spaces)]
    prol = [O.CooMatrix(prob.spaces[l + 1].nv, prob.spaces[l].nv, *prob.prolongations[l]) for l in range(L - 1)]
    mg = O.MGPreconditioner(mats, prol, prob.velocity_boundary, [None] + [(O.SMOOTH_JACOBI, 1, 1.0)] * (L - 1),
                            cycles=1, use_fmg=False)
    keep = []
    for l in range(1, L):
        sw = sol.schwarz[l - 1]
        So = O.Schwarz(mats[l], O.SCHWARZ_COLORED, sw.patches, 1.0, colours=sw.colours)
        keep.append(So)
        mg.set_schwarz(l, So, 1)
    s = prob.system
    A = O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals)
    P = O.BlockDiagonal(mg, prob.pressure_inverse)
    setup = time.perf_counter() - t0
    cores = oracle_threads()
    b = s.rhs
    t0 = time.perf_counter()
    ref = O.solve_gmres(A, b, RTOL * float(np.linalg.norm(b)), M=P, restart=50)
    t = time.perf_counter() - t0
    return {"n": s.n, "iterations": ref.iterations, "solve_s": t, "setup_s": setup, "cells": cells, "cores": cores}


def run_stokes(args):
    """Taylor-Hood Stokes on 256x256 cells, GMRES(50) + block-diagonal
    preconditioner to 1e-8, variants of the velocity smoother and precision."""
    import torch
    from jfem_b200 import _native as N
    from jfem_b200.linalg import DeviceMatrix
    from jfem_b200.stokes import StokesSolver, stokes_problem
    ctx = N.default_context()
    t0 = time.time()
    prob = stokes_problem(args.cells if args.cells != CELLS else 256, 4, seed=0, pin_pressure=False)
    assemble_s = time.time() - t0
    if args.profile == "precond-apply":      # the Schwarz-smoothed block preconditioner, --warmup + 1 times
        sol = StokesSolver(ctx, prob)
        v = np.random.default_rng(0).standard_normal(prob.system.n)
        for _ in range(args.warmup + 1):
            sol.P.mvMul(v)
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile}))
        return
    b = prob.system.rhs
    tol = RTOL * float(np.linalg.norm(b))
    out = {}
    for name, kw in (("schwarz_fp64", {}), ("schwarz_fp32_vcycle", {"fp32_vcycle": True}),
                     ("jacobi_fp64", {"smoother": "jacobi", "runs": 2, "omega": 0.6})):
        t1 = time.time()
        sol = StokesSolver(ctx, prob, **kw)
        setup = time.time() - t1
        for _ in range(max(1, args.warmup)):
            x, it = sol.solve(tol)
        ts = []
        for _ in range(max(1, args.steps // 3)):
            t2 = time.perf_counter()
            x, it = sol.solve(tol)
            ts.append(time.perf_counter() - t2)
        A = sol.A
        r = b - A.spmv(x)
        out[name] = {"time_s": min(ts), "iterations": it.iterations, "restarts": it.last.restarts,
                     "status": N.STATUS_NAMES[it.last.status],
                     "true_rel_residual": float(np.linalg.norm(r) / np.linalg.norm(b)), "setup_s": setup}
        del sol
    # the reference's monolithic driver (Examples/src/StokesMGSchwarz.java) at
    # its own size (4 refinements of 4 x 4 cells: 64 x 64 cells): PGMRES with
    # the MG of the whole Taylor-Hood system of every level (pinned first
    # pressure unknown), coloured Schwarz smoothing (partitions 2 * 2^(l-1),
    # overlap 2: 8 x 8-cell patches of up to 659 unknowns, 2 runs), FMG + 3
    # V-cycles per application
    if os.environ.get("JFEM_BENCH_NO_MONOLITHIC") != "1":
        from jfem_b200.stokes import MonolithicStokesMG
        t1 = time.time()
        mono = MonolithicStokesMG(ctx, cells=64, coarse_cells=4, seed=0)
        setup = time.time() - t1
        bm = mono.rhs
        tol_m = RTOL * float(np.linalg.norm(bm))
        for _ in range(max(1, args.warmup)):
            x, it = mono.solve(tol_m, max_restarts=20)
        ts = []
        for _ in range(max(1, args.steps // 3)):
            t2 = time.perf_counter()
            x, it = mono.solve(tol_m, max_restarts=20)
            ts.append(time.perf_counter() - t2)
        r = bm - mono.A.spmv(x)
        out["monolithic_schwarz_mg"] = {
            "time_s": min(ts), "iterations": it.iterations, "restarts": it.last.restarts,
            "status": N.STATUS_NAMES[it.last.status], "true_rel_residual": float(np.linalg.norm(r) / np.linalg.norm(bm)),
            "setup_s": setup, "dofs": int(mono.A.rows), "max_patch": max(sw.info()["max_patch"] for sw in mono.schwarz),
            "mode": "64x64 cells (the reference driver's size): PGMRES(50) + MG of the whole Taylor-Hood system "
                    "(FMG + 3 V-cycles), coloured Schwarz 2 runs, partitions 2*2^(l-1), overlap 2, pinned "
                    "pressure (the reference's system)"}
        del mono
    s = prob.system
    line = {"metric": "time-to-1e-8 residual (s), Stokes GMRES(50) + block-diagonal preconditioner",
            "value": out["schwarz_fp64"]["time_s"], "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (lid-driven cavity + seeded Fourier body force)",
            "config": {"workload": "stokes: Taylor-Hood Q2/Q1 256x256 cells", "dofs": s.n,
                       "velocity_dofs": s.nv, "nnz": int(s.vals.size), "levels": len(prob.spaces),
                       "preconditioner": "velocity V-cycle (coloured Schwarz, 2x2-cell partitions + 1 cell "
                                         "overlap, 9 colours) | nu / lumped pressure mass",
                       "pressure": "consistent singular system, gauge p0 = 0 after the solve"},
            "variants": out, "assemble_s": assemble_s}
    # the same system assembled on the GPU (jfg_assemble_taylor_hood), timed
    from jfem_b200.stokes import TaylorHoodSpace, assemble_stokes_device, fourier_force
    th = TaylorHoodSpace(prob.spaces[-1].cx, prob.spaces[-1].cy)
    fo = fourier_force(seed=0)
    assemble_stokes_device(th, 1.0, fo, pin_pressure=False, ctx=ctx)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    Ad, _, _ = assemble_stokes_device(th, 1.0, fo, pin_pressure=False, ctx=ctx)
    torch.cuda.synchronize()
    line["assemble_device_s"] = time.perf_counter() - t3
    line["assemble_device_nnz_equal"] = bool(Ad.nnz == DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx).nnz)
    del Ad
    A64 = DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx)
    ms64 = A64.time_spmv(precision=0, iters=50)
    line["spmv_gbs_fp64"] = spmv_bytes(s.n, A64.nnz, 8, 8) / (ms64 * 1e-3) / 1e9
    del A64
    if os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        c = stokes_cpu_sample()
        it = out["schwarz_fp64"]["iterations"]
        line["cpu_baseline"] = {"value": c["solve_s"] / c["iterations"] * (s.n / c["n"]) * it, "unit": "s",
                                "cores": c["cores"], "kind": "port",
                                "sample": f"whole oracle solve on {c['cells']}x{c['cells']} cells ({c['n']} unknowns, "
                                          f"{c['iterations']} iterations, {c['solve_s']:.2f} s), per iteration "
                                          f"scaled by unknowns to {s.n} and to {it} iterations",
                                "sample_setup_s": c["setup_s"]}
    print(json.dumps(line))


def run_learned(args):
    """FGMRES(30) + FP32 V-cycle + learned smoother vs FP64 GMG-PCG."""
    from jfem_b200 import _native as N
    from jfem_b200.learned import WEIGHTS, evaluate
    from jfem_b200.learned import KappaSystem
    ctx = N.default_context()
    w = np.load(WEIGHTS)
    ks = KappaSystem(ctx, 1024, kseed=0)
    out = evaluate(ctx, w, cells=1024, kseed=0, out_scales=(1.0, 0.5), repeats=max(3, args.steps), ks=ks)
    with open(WEIGHTS.replace(".npy", ".train.json")) as f:
        train = json.load(f)
    best = min(v["time_s"] for v in out["fgmres_vcycle_net"].values())
    line = {"metric": "time-to-1e-8 residual (s): FGMRES(30)+V-cycle+learned smoother vs FP64 GMG-PCG",
            "value": best, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32+f64",
            "data": "synthetic (GRF kappa, seeded)",
            "config": {"workload": "learned: -div(kappa grad u) = f, Q1 1024x1024, kappa = exp(GRF l=0.05 s2=1)",
                                   "training": train},
            "speedup_vs_fp64_gmg_pcg": out["gmg_pcg_fp64"]["time_s"] / best, "arms": out}
    ms64 = ks.A.time_spmv(precision=0, iters=50)
    ms32 = ks.A.time_spmv(precision=1, iters=50)
    line["spmv_gbs"] = {"fp64": spmv_bytes(ks.n, ks.A.nnz, 8, 8) / (ms64 * 1e-3) / 1e9,
                        "fp32": spmv_bytes(ks.n, ks.A.nnz, 4, 4) / (ms32 * 1e-3) / 1e9}
    if os.environ.get("JFEM_BENCH_NO_CPU") != "1":
        line["cpu_baseline"] = cpu_baseline(ks.h, out["tol"])
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        if args.workload not in ("kappa", "gmg-pcg"):
            print(json.dumps({"impl": "reference",
                              "unavailable": "the reference arm covers the kappa and gmg-pcg workloads"}))
            return
        run_reference(args)
    elif args.workload == "assemble":
        run_assemble(args)
    elif args.workload == "gs-pcg":
        run_gs_pcg(args)
    elif args.workload == "galerkin":
        run_galerkin(args)
    elif args.workload == "cg-small":
        run_cg_small(args)
    elif args.workload == "batch-heat":
        run_batch_heat(args)
    elif args.workload == "stokes":
        run_stokes(args)
    elif args.workload == "learned":
        run_learned(args)
    elif args.workload == "gmg-pcg":
        run_ours(args)
    else:
        run_kappa(args)


if __name__ == "__main__":
    main()
