"""Benchmark: time to a 1e-8 relative FP64 residual and SpMV GB/s on one B200.

Workload (one "step" = one solve): -Laplace u + 5u = f on the unit square,
Q2 elements on a 512x512 cell grid (1,050,625 dofs, 8-level geometric
multigrid, 2+2 damped-Jacobi sweeps with omega = 2/3, coarsest 4x4 cells
solved by a dense FP64 inverse), f from 16x16 seeded sine modes.  The headline
solve is the mixed-precision GMG-PCG (FP64 defect correction around FP32
V-cycle-preconditioned CG); the plain FP64 GMG-PCG on the same GPU is timed
beside it.  The matrix (202 MB FP64 / 134 MB FP32 values + indices) is larger
than L2, so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Under torchrun every rank solves its own replica (no data-path collective;
"replicas only"); the step time is the max over ranks.

The other configurations are measured with --workload (one JSON line each,
1 GPU, no reference arm): batch-heat (256 uneven Q1 heat systems, 50
implicit-Euler steps in one persistent launch), stokes (Taylor-Hood Q2/Q1
on 256x256 cells, GMRES(50) with the block-diagonal preconditioner) and
learned (-div(kappa grad u) = f on Q1 1024x1024: FGMRES(30) with the
V-cycle + learned smoother against FP64 GMG-PCG).
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
    ap.add_argument("--workload", default="gmg-pcg", choices=["gmg-pcg", "cg-small", "batch-heat", "stokes", "learned", "galerkin", "gs-pcg",
                                                        "assemble"])
    ap.add_argument("--profile", default=None,
                    choices=["solve-fp64", "solve-mixed", "solve-mixed-nograph", "gs-mixed-nograph", "spmv64", "spmv32"],
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
        cpu = cpu_baseline(h, tol, it64)

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
                         "traffic": SPMV32_TRAFFIC_BYTES if (n, nnz) == SPMV32_TRAFFIC_CASE else None, "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                         "one cold launch (profiles/k_spmv_sell_fp32_q2_512.md)",
                         "kernel": "k_spmv_pipe<float> finest level", "peak_source": peak_src,
                         "bytes_per_launch": b32, "ms_per_launch": ms_spmv32},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "setup_s": setup_s,
        }
        print(json.dumps(line))
    reps.close()


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


def cpu_baseline(h, tol, iters_hint):
    """The oracle (C restatement of the reference's FP64 PCG + GMG V-cycle),
    one host thread, on a bounded sample: 2 PCG iterations, scaled to the
    FP64 GPU iteration count."""
    import oracle as O
    mats = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    mg = O.MGPreconditioner(mats, prol, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2.0 / 3.0)] * (len(mats) - 1),
                            cycles=1, use_fmg=False)
    b = h.finest.rhs
    sample = 2
    cores = oracle_threads()
    t0 = time.perf_counter()
    O.solve_pcg(mats[-1], mg, b, tol, maxit=sample)
    t = time.perf_counter() - t0
    per_it = t / sample
    return {"value": per_it * max(iters_hint, 1), "unit": "s", "cores": cores, "kind": "port",
            "sample": f"{sample} PCG iterations (incl. setup residual) scaled to {iters_hint} iterations",
            "sample_s": t}


def run_reference(args):
    rank, world, local = dist_env()
    if world > 1 and rank != 0:
        return
    h = build_problem(args.cells, args.levels)
    import oracle as O
    mats = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(h.systems) - 1)]
    mg = O.MGPreconditioner(mats, prol, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2.0 / 3.0)] * (len(mats) - 1),
                            cycles=1, use_fmg=False)
    b = h.finest.rhs
    tol = RTOL * float(np.linalg.norm(b))
    cores = oracle_threads()
    # each step is one whole FP64 GMG-PCG solve from e0 (about 3 s on one
    # host core for the SpMV, all cores for the restriction)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        full = O.solve_pcg(mats[-1], mg, b, tol)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    val = statistics.mean(times)
    line = {"metric": METRIC, "value": val, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": val * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sine-mode source, assembled Q2 system)",
            "config": {"workload": WORKLOAD, "dofs": int(h.finest.n), "parallelism": "cpu"},
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
    batch = problems.heat_batch(nsys=256, dt=1e-3, seed=0)
    K = [DeviceMatrix(s.K.n, s.K.n, s.K.rows, s.K.cols, s.K.vals, ctx) for s in batch]
    M = [DeviceMatrix(s.M.n, s.M.n, s.M.rows, s.M.cols, s.M.vals, ctx) for s in batch]
    B = BatchedParabolicIntegrator(K, M, ctx)
    u0 = B.pack([s.u0 for s in batch])
    steps = 50
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
        pick = list(range(0, 256, 32))
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
               "sample": f"one CG step (1e-10) of {len(pick)} systems, scaled by unknowns to 256 systems x 50 steps; "
                         "serial: the reference's CG has no parallel loop"}
    line = {"metric": "time for 50 implicit-Euler steps of 256 uneven Q1 heat systems (s)",
            "value": statistics.median(ms) / 1e3, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.median(ms), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded bumps)",
            "config": {"workload": "batch-heat: 256 Q1 systems, cells {32..256 step 16}^2, dt=1e-3, 50 steps",
                                   "systems": 256, "dofs": dofs, "nnz": nnz},
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
        line["cpu_baseline"] = cpu_baseline(ks.h, out["tol"], out["gmg_pcg_fp64"]["iterations"])
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        if args.workload != "gmg-pcg":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm covers the gmg-pcg workload"}))
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
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
