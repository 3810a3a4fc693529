"""Parity at the benchmark sizes: the products and solves that the timed
workloads run, against the oracle on the same seeded inputs.

* Q2 on 512 x 512 cells (1,050,625 rows, 16.7 M nonzeros): the finest level
  of the multigrid-PCG workload, whose products take the staged SELL kernel
  (k_spmv_pipe, one thread per row from 262,144 rows);
* Q1 on 1024 x 1024 cells with kappa = exp(Gaussian random field) (1,050,625
  rows, 9.4 M nonzeros): the learned-preconditioner workload, whose level
  matrices take the values-only 9-point stencil layout.

FP64 products equal the oracle's COO scatter (SparseMatrix.mvMul /
tvMul, linalg/SparseMatrix.java:480-501) to 1e-12 relative (absolute floor
1e-12 * max |y|: the sums run in another order).  Reduced-precision products
(FP32, BF16, scaled FP16 values; FP32 vectors and sums) are compared with the
oracle's product of the same rounded values and vectors within the classical
summation bound |y - y_exact| <= 2 (k + 1) u (|A| |x|) per row, k the row
length, u = 2^-24 the FP32 unit roundoff (the value rounding itself is part of
the inputs).  Whole solves: FP64 GMG-PCG (IterativeSolver.solvePCG,
linalg/IterativeSolver.java:102-162, one V-cycle per application) against the
oracle's solve -- same iteration count, relative solution error <= 1e-8,
residual histories within 1e-6 -- and FGMRES(30) with the FP64 V-cycle against
the FGMRES oracle.
"""
import numpy as np
import pytest
import scipy.sparse as sps
import torch

import oracle as O
from jfem_b200 import IterativeSolver, JacobiSmoother, MGPreconditioner, problems
from jfem_b200 import _native as N
from jfem_b200.linalg import DeviceMatrix
from oracle.fgmres import solve_fgmres

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


@pytest.fixture(scope="module")
def cfg1():
    return problems.hierarchy(2, 4, 8, mass=5.0, modes=16, seed=0)          # Q2 512^2


@pytest.fixture(scope="module")
def cfg4():
    h, _ = problems.kappa_hierarchy(1, 4, 9, 0.05, 1.0, kseed=0)              # Q1 1024^2, kappa-GRF
    return h


def merged(sy):
    A = sps.csr_matrix((sy.vals, (sy.rows, sy.cols)), shape=(sy.n, sy.n))
    A.sum_duplicates()
    A.eliminate_zeros()
    A.sort_indices()
    return A


def _case(request, name):
    return request.getfixturevalue(name)


@pytest.mark.parametrize("name,stencil", [("cfg1", False), ("cfg4", True)])
def test_fp64_mvmul_tvmul_vs_oracle(ctx, request, name, stencil):
    sy = _case(request, name).finest
    A = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    assert A.layout()["stencil"] == stencil
    ref = O.CooMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals)
    rng = np.random.default_rng(11)
    for x in (rng.standard_normal(sy.n), np.cos(np.arange(sy.n) * 0.37)):
        yr = ref.mvmul(x)
        np.testing.assert_allclose(A.spmv(x), yr, rtol=1e-12, atol=1e-12 * np.abs(yr).max())
        zr = ref.tvmul(x)
        np.testing.assert_allclose(A.spmv_t(x), zr, rtol=1e-12, atol=1e-12 * np.abs(zr).max())


@pytest.mark.parametrize("name", ["cfg1", "cfg4"])
@pytest.mark.parametrize("values", ["fp32", "bf16", "fp16"])
def test_reduced_precision_mvmul_vs_oracle(ctx, request, name, values):
    sy = _case(request, name).finest
    A = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    M = merged(sy)
    x = np.random.default_rng(12).standard_normal(sy.n).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    y = A.spmv_lowp_dev(xd, values).cpu().numpy().astype(np.float64)
    lay = A.layout()
    # the values the kernel reads, rounded from the merged FP64 values
    if values == "fp32":
        v = M.data.astype(np.float32).astype(np.float64)
    elif values == "bf16":
        v = torch.from_numpy(M.data.astype(np.float32)).to(torch.bfloat16).to(torch.float64).numpy()
    else:
        s = 1.0 / lay["fp16_scale_inv"]
        v = (M.data * s).astype(np.float16).astype(np.float64) / s
    rows = np.repeat(np.arange(sy.n, dtype=np.int32), np.diff(M.indptr))
    ref = O.CooMatrix(sy.n, sy.n, rows, M.indices.astype(np.int32), v)
    y_exact = ref.mvmul(x.astype(np.float64))
    absr = O.CooMatrix(sy.n, sy.n, rows, M.indices.astype(np.int32), np.abs(v)).mvmul(np.abs(x).astype(np.float64))
    k = np.diff(M.indptr)
    bound = 2.0 * (k + 1) * U32 * absr + 1e-30
    err = np.abs(y - y_exact)
    assert np.all(err <= bound), (float(np.max(err / bound)), values)


@pytest.mark.parametrize("values", ["fp64", "fp32", "fp16"])
def test_stencil_layout_equals_sell_bitwise(ctx, cfg4, monkeypatch, values):
    """The values-only stencil kernel sums each row in the SELL kernels'
    order with the same multiply-adds: identical bits on the Q1 kappa matrix
    (JFEM_STENCIL=0 builds the same matrix without the stencil layout)."""
    sy = cfg4.finest
    A_st = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    monkeypatch.setenv("JFEM_STENCIL", "0")
    A_sell = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    assert A_st.layout()["stencil"] and not A_sell.layout()["stencil"]
    x = np.random.default_rng(13).standard_normal(sy.n)
    if values == "fp64":
        assert np.array_equal(A_st.spmv(x), A_sell.spmv(x))
        assert np.array_equal(A_st.spmv_t(x), A_sell.spmv_t(x))
    else:
        xd = torch.from_numpy(x.astype(np.float32)).cuda()
        assert np.array_equal(A_st.spmv_lowp_dev(xd, values).cpu().numpy(),
                              A_sell.spmv_lowp_dev(xd, values).cpu().numpy())


def _mg(h, ctx, precision="fp64"):
    L = len(h.systems)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (L - 1), cycles=1,
                          use_fmg=False, precision=precision, ctx=ctx)
    return mats, prol, mg


def _mg_oracle(h):
    L = len(h.systems)
    mats = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in h.systems]
    prol = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
    mg = O.MGPreconditioner(mats, prol, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2 / 3)] * (L - 1), cycles=1,
                            use_fmg=False)
    return mats, mg


@pytest.mark.parametrize("name", ["cfg1", "cfg4"])
def test_fp64_gmg_pcg_vs_oracle(ctx, request, name):
    """The plain FP64 GMG-PCG drop-in on the whole benchmark system, from e0."""
    h = _case(request, name)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    mats_o, mg_o = _mg_oracle(h)
    ref = O.solve_pcg(mats_o[-1], mg_o, b, tol)
    mats, prol, mg = _mg(h, ctx)
    s = IterativeSolver(ctx=ctx)
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert ref.status == O.OK and s.last.status == N.OK
    assert s.iterations == ref.iterations
    assert np.linalg.norm(x - ref.x) / np.linalg.norm(ref.x) < 1e-8
    np.testing.assert_allclose(s.last.history, ref.history, rtol=1e-6)
    assert np.linalg.norm(b - mats_o[-1].mvmul(x)) <= tol
    # the mixed solve (FP32 V-cycle) reaches the same FP64 tolerance and agrees with the oracle's solution
    s32 = IterativeSolver(ctx=ctx)
    s32.precision = "mixed-precond"
    _, _, mg32 = _mg(h, ctx, "mixed")
    x32 = s32.solvePCG(mats[-1], mg32, b, tol)
    assert s32.last.status == N.OK
    assert np.linalg.norm(b - mats_o[-1].mvmul(x32)) <= tol
    assert abs(s32.iterations - ref.iterations) <= 1
    assert np.linalg.norm(x32 - ref.x) / np.linalg.norm(ref.x) < 1e-6


def test_cfg4_fgmres_vcycle_vs_oracle(ctx, cfg4):
    """FGMRES(30) preconditioned by the FP64 V-cycle on the kappa system
    against the FGMRES oracle with the oracle's V-cycle."""
    h = cfg4
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    mats_o, mg_o = _mg_oracle(h)
    x_o, it_o, _, st_o, hist_o = solve_fgmres(mats_o[-1].mvmul, mg_o.mvmul, b, tol, restart=30)
    mats, prol, mg = _mg(h, ctx)
    s = IterativeSolver(ctx=ctx)
    x = s.solveFGMRES(mats[-1], mg, b, tol, restart=30)
    assert st_o == O.OK and s.last.status == N.OK
    assert s.iterations == it_o
    np.testing.assert_allclose(s.last.history[:it_o], hist_o[:it_o], rtol=1e-6)
    assert np.linalg.norm(x - x_o) / np.linalg.norm(x_o) < 1e-8
    assert np.linalg.norm(b - mats_o[-1].mvmul(x)) <= tol
