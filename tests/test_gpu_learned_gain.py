"""What the trained network gains over the method without it, on the
learned-preconditioner workload (Q1 1024 x 1024, kappa = exp(GRF), a kappa
field the network was not trained on).

Stated relation (measured; the numbers are printed):
* one application of "FP32 V-cycle + network" leaves a smaller residual
  than the V-cycle alone: mean ||v - A M(v)|| / ||v - A V(v)|| below 0.95
  over seeded random vectors of mixed spectrum;
* FGMRES(30) with the network needs no more iterations than without it to
  reach the 1e-8 FP64 true residual.
The network does not make the solve faster (it costs one forward pass per
iteration); the times are printed, not asserted."""
import json
import time

import numpy as np
import pytest
import torch

from jfem_b200 import IterativeSolver
from jfem_b200 import _native as N
from jfem_b200.cnn import LearnedSmoother
from jfem_b200.learned import WEIGHTS, KappaSystem, random_vectors

pytestmark = pytest.mark.gpu


def test_network_gain_on_unseen_kappa(ctx):
    ks = KappaSystem(ctx, 1024, kseed=0)                  # training used kappa seeds 1000..1015
    net = LearnedSmoother(ctx, weights=np.load(WEIGHTS))
    pv = ks.preconditioner(net, use_net=False)
    pn = ks.preconditioner(net, use_net=True)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(123)
    vs = random_vectors(ks, 8, gen)
    ratios = []
    for i in range(vs.shape[0]):
        v = vs[i].contiguous()
        r1 = torch.linalg.vector_norm(v - ks.A.spmv_dev(pv.apply_dev(v))).item()
        r2 = torch.linalg.vector_norm(v - ks.A.spmv_dev(pn.apply_dev(v))).item()
        ratios.append(r2 / r1)
    b = torch.tensor(ks.b, device="cuda")
    tol = 1e-8 * float(np.linalg.norm(ks.b))
    out = {}
    for name, pc in (("vcycle", pv), ("vcycle+net", pn)):
        s = IterativeSolver(ctx=ctx)
        best = None
        for _ in range(3):
            x = torch.zeros_like(b)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.solve_device(N.FGMRES, ks.A, pc, b, x, tol, restart=30)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        res = torch.linalg.vector_norm(b - ks.A.spmv_dev(x)).item()
        assert s.last.status == N.OK and res <= tol * 1.0001
        out[name] = {"iterations": s.iterations, "time_s": best}
    print(json.dumps({"residual_ratio_mean": float(np.mean(ratios)), "residual_ratios": ratios, "fgmres": out}))
    assert float(np.mean(ratios)) < 0.95
    assert out["vcycle+net"]["iterations"] <= out["vcycle"]["iterations"]
