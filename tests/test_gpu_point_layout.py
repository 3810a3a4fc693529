"""The values-only point layouts and the staged product kernel.

* 9-point layout of Q1 level matrices: the register kernel (k_spmv_st, the
  default) and the staged kernel (k_spmv_pt: value streams by bulk copies
  into shared memory, JFEM_ST_STAGED=1) give the SELL kernels' bits
  (products in FP64, FP32, BF16 and scaled FP16);
* transfer layouts of Q1 prolongations (4 values per fine row) and
  restrictions (9 values per coarse row), built by the multigrid set-up when
  the level matrices carry the 9-point layout with strides S and 2 S - 1: the
  V-cycle in every hierarchy precision agrees with the one with SELL-32
  transfers (JFEM_MG_TRANSFER=0) and the oracle's, and the prolongation's
  products equal the oracle's COO scatter (SparseMatrix.mvMul / tvMul,
  linalg/SparseMatrix.java:480-501) to 1e-12.
"""
import numpy as np
import pytest
import torch

import oracle as O
from jfem_b200 import JacobiSmoother, MGPreconditioner, problems
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q1_512():
    h, _ = problems.kappa_hierarchy(1, 4, 8, 0.05, 1.0, kseed=3)          # Q1 512^2, kappa-GRF
    return h


def _mg(h, ctx, precision):
    L = len(h.systems)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (L - 1), cycles=1,
                          use_fmg=False, precision=precision, ctx=ctx)
    return mats, prol, mg


@pytest.mark.parametrize("values", ["fp64", "fp32", "bf16", "fp16"])
def test_staged_equals_register_stencil_kernel(ctx, q1_512, monkeypatch, values):
    sy = q1_512.finest
    monkeypatch.setenv("JFEM_ST_STAGED", "1")
    A_pt = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    monkeypatch.setenv("JFEM_ST_STAGED", "0")
    A_reg = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    monkeypatch.setenv("JFEM_STENCIL", "0")
    A_sell = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    assert A_pt.layout()["kind"] == "stencil" and A_sell.layout()["kind"] == "sell"
    x = np.random.default_rng(21).standard_normal(sy.n)
    if values == "fp64":
        ys = [A.spmv(x) for A in (A_pt, A_reg, A_sell)]
        zs = [A.spmv_t(x) for A in (A_pt, A_reg, A_sell)]
        assert np.array_equal(ys[0], ys[2]) and np.array_equal(ys[1], ys[2])
        assert np.array_equal(zs[0], zs[2]) and np.array_equal(zs[1], zs[2])
    else:
        xd = torch.from_numpy(x.astype(np.float32)).cuda()
        ys = [A.spmv_lowp_dev(xd, values).cpu().numpy() for A in (A_pt, A_reg, A_sell)]
        assert np.array_equal(ys[0], ys[2]) and np.array_equal(ys[1], ys[2])


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed-bf16", "mixed-fp16"])
def test_transfer_layouts_vcycle(ctx, q1_512, monkeypatch, precision):
    """The V-cycle with the transfer layouts against the same V-cycle with
    SELL-32 transfers (JFEM_MG_TRANSFER=0): the products on levels below
    262,144 rows split SELL rows over 4-8 lanes, so the two agree to rounding
    (1e-12 in FP64, 1e-5 with FP32 sums); the FP64 one also matches the
    oracle's V-cycle to 1e-10, and the finest prolongation (one thread per
    row in both layouts) gives identical bits."""
    h = q1_512
    b = h.finest.rhs
    _, prol, mg = _mg(h, ctx, precision)
    lay = prol[-1].layout()
    assert lay["kind"] == "prolongation" and lay["stride"] == 513
    assert lay["regular_rows"] > 0.98 * h.finest.n
    v_pt = mg.vCycle(np.zeros(b.size), b)
    monkeypatch.setenv("JFEM_MG_TRANSFER", "0")
    _, prol0, mg0 = _mg(h, ctx, precision)
    assert prol0[-1].layout()["kind"] == "sell"
    v_sell = mg0.vCycle(np.zeros(b.size), b)
    tol = 1e-12 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(v_pt, v_sell, rtol=tol, atol=tol * np.abs(v_sell).max())
    xc = torch.from_numpy(np.random.default_rng(23).standard_normal(h.systems[-2].n).astype(np.float32)).cuda()
    for vals in ("fp32", "bf16", "fp16"):
        assert np.array_equal(prol[-1].spmv_lowp_dev(xc, vals).cpu().numpy(),
                              prol0[-1].spmv_lowp_dev(xc, vals).cpu().numpy())
    if precision == "fp64":
        L = len(h.systems)
        mats_o = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in h.systems]
        prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
        mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2 / 3)] * (L - 1),
                                  cycles=1, use_fmg=False)
        ref = mg_o.vcycle(np.zeros(b.size), b)
        np.testing.assert_allclose(v_pt, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_prolongation_layout_vs_oracle(ctx, q1_512):
    """FP64 products of the prolongations (SELL-32 for FP64 values) to
    1e-12 and the FP32 products of the transfer layout within the classical
    summation bound 2 (k + 1) u (|P| |x|) of the oracle's product of the same
    FP32-rounded values and vector."""
    h = q1_512
    _, prol, _ = _mg(h, ctx, "mixed")
    rng = np.random.default_rng(22)
    u32 = 2.0 ** -24
    for l in (len(prol) - 1, len(prol) - 3):
        P = prol[l]
        nf, nc = h.systems[l + 1].n, h.systems[l].n
        assert P.layout()["kind"] == "prolongation"
        ref = O.CooMatrix(nf, nc, *h.prolong[l])
        x = rng.standard_normal(nc)
        yr = ref.mvmul(x)
        np.testing.assert_allclose(P.spmv(x), yr, rtol=1e-12, atol=1e-12 * np.abs(yr).max())
        z = rng.standard_normal(nf)
        zr = ref.tvmul(z)
        np.testing.assert_allclose(P.spmv_t(z), zr, rtol=1e-12, atol=1e-12 * np.abs(zr).max())
        x32 = x.astype(np.float32)
        y32 = P.spmv_lowp_dev(torch.from_numpy(x32).cuda(), "fp32").cpu().numpy().astype(np.float64)
        r, c, v = h.prolong[l]
        v32 = np.asarray(v).astype(np.float32).astype(np.float64)
        exact = O.CooMatrix(nf, nc, r, c, v32).mvmul(x32.astype(np.float64))
        absr = O.CooMatrix(nf, nc, r, c, np.abs(v32)).mvmul(np.abs(x32).astype(np.float64))
        assert np.all(np.abs(y32 - exact) <= 2 * 5 * u32 * absr + 1e-30)
