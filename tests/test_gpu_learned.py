"""Training of the learned smoother through the real operator (small grid)."""
import numpy as np
import pytest

from jfem_b200 import _native as N
from jfem_b200.learned import evaluate, train

pytestmark = pytest.mark.gpu


def test_residual_training_reduces_the_residual(ctx):
    w, rep = train(ctx, cells=32, fields=2, pairs=8, steps=300, batch=2, lr=2e-3, log=lambda *_: None)
    assert rep["final_ratio"] < rep["first_ratio"]
    assert rep["final_ratio"] < 0.9
    assert w.shape == (37440,) and np.all(np.isfinite(w))


def test_evaluate_runs_all_arms(ctx):
    w, _ = train(ctx, cells=32, fields=1, pairs=4, steps=50, batch=2, log=lambda *_: None)
    out = evaluate(ctx, w, cells=32, kseed=0, out_scales=(1.0,), repeats=1)
    for arm in ("gmg_pcg_fp64", "gmg_pcg_fp32_vcycle", "fgmres_vcycle"):
        assert out[arm]["status"] == "OK"
        assert out[arm]["true_residual"] <= out["tol"] * 1.0001
    assert out["fgmres_vcycle_net"]["1.0"]["status"] in ("OK", "NOT_CONVERGED")
