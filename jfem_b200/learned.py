"""Training and evaluation of the learned smoother on -div(kappa grad u) = f
(Q1, kappa = exp(g), g a Gaussian random field).  No counterpart in the
reference (JFEM has no neural-network code).

Training data are made on the GPU from independently seeded kappa fields:

    v        a random vector of mixed spectrum (zero on Dirichlet nodes, unit norm)
    r'       = v - A V(v)                 the residual left by one FP32 V-cycle
    q        = D^-1 r',  s = rms(q)       the network input is q / s

The default loss is the residual left after the network's correction,
||r' - A s net(q / s)||^2 on the full node grid, so the network learns a
local smoother for what the V-cycle leaves behind.  The alternative loss
fits e' / s with e' = A^-1 r' (FP64 PCG with the same hierarchy) on random
square crops.  The trained network is used by
MGCNNPreconditioner inside FGMRES(30) and compared with plain FP64 GMG-PCG.

Command line:

    python -m jfem_b200.learned train --out WEIGHTS.npy [--cells 1024 --fields 16 --pairs 125 --steps 4000]
    python -m jfem_b200.learned eval --weights WEIGHTS.npy [--cells 1024]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np
import torch

from . import _native as N
from . import problems
from .cnn import LearnedSmoother, MGCNNPreconditioner, he_init, pixel_map
from .linalg import DeviceMatrix, IterativeSolver
from .multigrid import JacobiSmoother, MGPreconditioner

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "smoother_kappa_q1.npy")
COARSE_CELLS = 4          # the hierarchy ends at 4 x 4 cells
LENGTH, VARIANCE = 0.05, 1.0


class KappaSystem:
    """One kappa field: the Q1 hierarchy on the GPU, the FP64 V-cycle (for
    GMG-PCG and for exact error targets) and the FP32 one (for the network
    preconditioner), with Jacobi 2 + 2 sweeps (omega = 2/3)."""

    def __init__(self, ctx, cells: int, kseed: int, fseed: int = 0, modes: int = 4):
        levels = int(round(math.log2(cells // COARSE_CELLS))) + 1
        if COARSE_CELLS << (levels - 1) != cells:
            raise ValueError("cells must be 4 * 2^k")
        h, self.kappa = problems.kappa_hierarchy(1, COARSE_CELLS, levels, LENGTH, VARIANCE, kseed=kseed,
                                                 modes=modes, fseed=fseed)
        self.h = h
        self.ctx = ctx
        self.mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
        prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(levels - 1)]
        self.mg = MGPreconditioner(self.mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (levels - 1),
                                   cycles=1, use_fmg=False, precision="mixed", ctx=ctx)
        self._prol = prol
        self.A = self.mats[-1]
        self.n = self.A.rows
        self.H, self.W, self.dof = pixel_map(h.spaces[-1])
        self.bd = h.boundary[-1]
        self.b = h.finest.rhs
        dev = torch.device("cuda")
        self.diag_t = torch.tensor(self.A.diag(), device=dev)
        self.dof_t = torch.tensor(self.dof, dtype=torch.long, device=dev)
        self.bd_t = torch.tensor(np.asarray(self.bd, dtype=np.int64), device=dev)

    def preconditioner(self, net, out_scale=1.0, use_net=True):
        return MGCNNPreconditioner(self.mg, net, self.A, self.H, self.W, self.dof, self.bd, out_scale=out_scale,
                                   use_net=use_net)


def random_vectors(ks: KappaSystem, count: int, gen: torch.Generator) -> torch.Tensor:
    """count unit vectors: white noise filtered by a Gaussian of random width
    (0 to 64 node spacings, log-uniform above 0.5), zero on Dirichlet nodes."""
    H, W = ks.H, ks.W
    out = torch.empty(count, ks.n, dtype=torch.float64, device="cuda")
    fy = torch.fft.fftfreq(H, device="cuda", dtype=torch.float64)
    fx = torch.fft.fftfreq(W, device="cuda", dtype=torch.float64)
    k2 = (fy[:, None] ** 2 + fx[None, :] ** 2) * (2 * math.pi) ** 2
    for i in range(count):
        z = torch.randn(H, W, generator=gen, device="cuda", dtype=torch.float64)
        u = torch.rand(1, generator=gen, device="cuda").item()
        if u > 0.2:
            ell = 0.5 * 128.0 ** ((u - 0.2) / 0.8)
            z = torch.fft.ifft2(torch.fft.fft2(z) * torch.exp(-0.5 * k2 * ell * ell)).real
        v = torch.empty(ks.n, dtype=torch.float64, device="cuda")
        v[ks.dof_t] = z.reshape(-1)
        v[ks.bd_t] = 0.0
        out[i] = v / torch.linalg.vector_norm(v)
    return out


def make_pairs(ks: KappaSystem, count: int, crops: int, crop: int, gen: torch.Generator, net=None):
    """(inputs, targets): (count * crops, crop, crop) float32 CUDA tensors."""
    if net is None:
        net = LearnedSmoother(ks.ctx, weights=he_init(0))
    pc = ks.preconditioner(net, use_net=False)
    solver = IterativeSolver(ctx=ks.ctx)
    solver.precision = "mixed-precond"
    X = torch.empty(count * crops, crop, crop, dtype=torch.float32, device="cuda")
    T = torch.empty_like(X)
    vs = random_vectors(ks, count, gen)
    k = 0
    for i in range(count):
        v = vs[i].contiguous()
        z0 = pc.apply_dev(v)
        rp = v - ks.A.spmv_dev(z0)
        q = rp / ks.diag_t
        s = torch.sqrt(torch.mean(q * q)).item()
        e = torch.zeros_like(rp)
        tol = 1e-10 * torch.linalg.vector_norm(rp).item()
        solver.solve_device(N.PCG, ks.A, ks.mg, rp.contiguous(), e, tol)
        qi = (q[ks.dof_t] / s).reshape(ks.H, ks.W)
        ei = (e[ks.dof_t] / s).reshape(ks.H, ks.W)
        for _ in range(crops):
            y0 = int(torch.randint(0, ks.H - crop + 1, (1,), generator=gen, device="cuda").item())
            x0 = int(torch.randint(0, ks.W - crop + 1, (1,), generator=gen, device="cuda").item())
            X[k] = qi[y0:y0 + crop, x0:x0 + crop].float()
            T[k] = ei[y0:y0 + crop, x0:x0 + crop].float()
            k += 1
    return X, T


def make_residuals(ks: KappaSystem, count: int, gen: torch.Generator, net):
    """count (network input, residual, scale) triples on the full node grid:
    q / s as (count, H, W) float32, r' as (count, n) float64, s as (count,)."""
    pc = ks.preconditioner(net, use_net=False)
    X = torch.empty(count, ks.H, ks.W, dtype=torch.float32, device="cuda")
    RP = torch.empty(count, ks.n, dtype=torch.float64, device="cuda")
    S = torch.empty(count, dtype=torch.float64, device="cuda")
    vs = random_vectors(ks, count, gen)
    for i in range(count):
        v = vs[i].contiguous()
        rp = v - ks.A.spmv_dev(pc.apply_dev(v))
        q = rp / ks.diag_t
        s = torch.sqrt(torch.mean(q * q))
        X[i] = (q[ks.dof_t] / s).reshape(ks.H, ks.W).float()
        RP[i] = rp
        S[i] = s
    return X, RP, S


def residual_step(net, A, dof_t, bd_t, X, RP, S, lr):
    """One Adam step on L = sum_b ||r'_b - A z_b||^2 / (B n) with
    z_b = s_b * scatter(net(x_b)) (zero on Dirichlet nodes).  The network
    kernels train on mean((y - t)^2); the pseudo-target
    t = y - dL/dy * (B H W) / 2 gives them exactly dL/dy.  Returns
    sum ||r' - A z||^2 / sum ||r'||^2."""
    B, H, W = X.shape
    n = RP.shape[1]
    y = net.forward(X)
    z = torch.zeros(B, n, dtype=torch.float64, device="cuda")
    z[:, dof_t] = y.reshape(B, -1).double() * S[:, None]
    z[:, bd_t] = 0.0
    g = torch.empty_like(z)
    num = den = 0.0
    for b in range(B):
        res = RP[b] - A.spmv_dev(z[b].contiguous())
        num += float((res * res).sum())
        den += float((RP[b] * RP[b]).sum())
        g[b] = A.spmv_t_dev(res.contiguous()) * (-2.0 / (B * n))
    g[:, bd_t] = 0.0
    gy = (g[:, dof_t] * S[:, None]).reshape(B, H, W)
    t = (y.double() - gy * (B * H * W / 2.0)).float().contiguous()
    net.train_step(X, t, lr=lr)
    return num / den


def train(ctx, cells=1024, fields=16, pairs=125, crops=4, crop=128, steps=4000, batch=16, lr=1e-3, seed=0,
          log=print, loss="residual"):
    """Trains from scratch; returns (weights, report).  loss="residual"
    minimises the residual left after the network's correction on full node
    grids (batch images of one field per step); loss="error" fits the
    normalised error e'/s on random crops."""
    if loss == "residual":
        return _train_residual(ctx, cells, fields, pairs, steps, min(batch, 4), lr, seed, log)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    t0 = time.time()
    net = LearnedSmoother(ctx, weights=he_init(seed, gain_last=0.1))
    Xs, Ts = [], []
    for f in range(fields):
        ks = KappaSystem(ctx, cells, kseed=1000 + f)
        X, T = make_pairs(ks, pairs, crops, crop, gen, net)
        Xs.append(X)
        Ts.append(T)
        log(f"field {f}: {X.shape[0]} crops, {time.time() - t0:.1f} s")
        del ks
    X = torch.cat(Xs)
    T = torch.cat(Ts)
    t_data = time.time() - t0
    m = X.shape[0]
    t1 = time.time()
    losses = []
    for it in range(steps):
        idx = torch.randint(0, m, (batch,), generator=gen, device="cuda")
        x = X[idx].contiguous()
        t = T[idx].contiguous()
        cur = lr * 0.5 * (1 + math.cos(math.pi * it / steps))
        losses.append(net.train_step(x, t, lr=cur))
        if it % 500 == 0 or it == steps - 1:
            log(f"step {it}: loss {np.mean(losses[-100:]):.4e}")
    t_train = time.time() - t1
    report = {"pairs": fields * pairs, "fields": fields, "crops": int(m), "crop": crop, "steps": steps,
              "batch": batch, "data_s": round(t_data, 1), "train_s": round(t_train, 1),
              "final_loss": float(np.mean(losses[-100:])), "first_loss": float(np.mean(losses[:100]))}
    return net.get_weights(), report


def _train_residual(ctx, cells, fields, pairs, steps, batch, lr, seed, log):
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    t0 = time.time()
    net = LearnedSmoother(ctx, weights=he_init(seed, gain_last=0.1))
    sets = []
    for f in range(fields):
        ks = KappaSystem(ctx, cells, kseed=1000 + f)
        X, RP, S = make_residuals(ks, pairs, gen, net)
        sets.append((ks.A, ks.dof_t, ks.bd_t, X, RP, S))
        log(f"field {f}: {pairs} residuals, {time.time() - t0:.1f} s")
        del ks
    t_data = time.time() - t0
    t1 = time.time()
    ratios = []
    for it in range(steps):
        f = int(torch.randint(0, fields, (1,), generator=gen, device="cuda").item())
        A, dof_t, bd_t, X, RP, S = sets[f]
        idx = torch.randint(0, X.shape[0], (batch,), generator=gen, device="cuda")
        cur = lr * 0.5 * (1 + math.cos(math.pi * it / steps))
        ratios.append(residual_step(net, A, dof_t, bd_t, X[idx].contiguous(), RP[idx].contiguous(),
                                    S[idx].contiguous(), cur))
        if it % 250 == 0 or it == steps - 1:
            log(f"step {it}: residual ratio {np.mean(ratios[-50:]):.4f}")
    t_train = time.time() - t1
    report = {"loss": "residual", "pairs": fields * pairs, "fields": fields, "grid": [cells + 1, cells + 1],
              "steps": steps, "batch": batch, "data_s": round(t_data, 1), "train_s": round(t_train, 1),
              "first_ratio": float(np.mean(ratios[:50])), "final_ratio": float(np.mean(ratios[-50:]))}
    return net.get_weights(), report


def evaluate(ctx, weights, cells=1024, kseed=0, tol_rel=1e-8, restart=30, out_scales=(1.0,), repeats=3, ks=None):
    """Time-to-tolerance on one kappa field: FP64 GMG-PCG, FGMRES(restart)
    with the FP32 V-cycle alone, and with the V-cycle + network; the solve is
    repeated and the best time kept (the first run also captures graphs).
    ks: an already built KappaSystem of that field (built here if None)."""
    if ks is None:
        ks = KappaSystem(ctx, cells, kseed=kseed)
    b = torch.tensor(ks.b, device="cuda")
    tol = tol_rel * float(np.linalg.norm(ks.b))
    net = LearnedSmoother(ctx, weights=weights)
    out = {"workload": f"kappa-grf Q1 {cells}x{cells}", "dofs": ks.n, "tol": tol, "kappa_seed": kseed}

    def timed(kind, prec, precision="fp64", rs=None):
        s = IterativeSolver(ctx=ctx)
        s.precision = precision
        best = None
        for _ in range(repeats):
            x = torch.zeros_like(b)
            torch.cuda.synchronize()
            t = time.perf_counter()
            s.solve_device(kind, ks.A, prec, b, x, tol, restart=rs)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t
            best = dt if best is None else min(best, dt)
        r = b - ks.A.spmv_dev(x)
        return {"time_s": best, "iterations": s.iterations, "status": N.STATUS_NAMES[s.last.status],
                "true_residual": float(torch.linalg.vector_norm(r).item())}

    out["gmg_pcg_fp64"] = timed(N.PCG, ks.mg)
    out["gmg_pcg_fp32_vcycle"] = timed(N.PCG, ks.mg, precision="mixed-precond")
    pc = ks.preconditioner(net, use_net=False)
    out["fgmres_vcycle"] = timed(N.FGMRES, pc, rs=restart)
    res = {}
    for sc in out_scales:
        pc.set(sc, use_net=True)
        res[str(sc)] = timed(N.FGMRES, pc, rs=restart)
    out["fgmres_vcycle_net"] = res
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m jfem_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--cells", type=int, default=1024)
    t.add_argument("--fields", type=int, default=16)
    t.add_argument("--pairs", type=int, default=125)
    t.add_argument("--crops", type=int, default=4)
    t.add_argument("--crop", type=int, default=128)
    t.add_argument("--steps", type=int, default=4000)
    t.add_argument("--batch", type=int, default=16)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--report", default=None)
    t.add_argument("--loss", choices=("residual", "error"), default="residual")
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--cells", type=int, default=1024)
    e.add_argument("--kseed", type=int, default=0)
    e.add_argument("--scales", default="1.0")
    a = ap.parse_args(argv)
    ctx = N.default_context()
    if a.cmd == "train":
        w, rep = train(ctx, a.cells, a.fields, a.pairs, a.crops, a.crop, a.steps, a.batch, a.lr, a.seed, loss=a.loss)
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        np.save(a.out, w)
        print(json.dumps(rep))
        if a.report:
            with open(a.report, "w") as f:
                json.dump(rep, f, indent=1)
    else:
        w = np.load(a.weights)
        scales = tuple(float(s) for s in a.scales.split(","))
        print(json.dumps(evaluate(ctx, w, a.cells, a.kseed, out_scales=scales)))


if __name__ == "__main__":
    main()
