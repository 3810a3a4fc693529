"""The allocation-free CG entry point, jfg_cg_noalloc, through the C ABI.

Callers that must not allocate device memory while they solve (a framework
that owns the device heap, a loop that cannot take cudaMalloc's latency and
implicit synchronisation) solve with jfg_cg_noalloc, whose work memory is a
fixed array inside the library.  Its result must agree with the allocating
entry point jfg_solve_dev(JFG_CG) on the same system, call after call: the
array keeps the previous call's contents, so two calls in a row are checked,
and the device's free memory must not change across a call.  This file is
collected last so that a stop-at-first-failure run has run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sps
import torch

from fixtures import fe_system
from jfem_b200 import _native as N
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu

NOALLOC_MAX_ROWS = 1 << 18


def _vp(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_cg_matches_solve_dev(ctx):
    space, sy = fe_system(1, 96, modes=4, seed=3)           # Q1 96x96: 9,409 unknowns
    A = sps.csr_matrix((sy.vals, (sy.rows, sy.cols)), shape=(sy.n, sy.n))
    A.sum_duplicates()
    A.eliminate_zeros()
    A.sort_indices()
    dev = torch.device("cuda", ctx.device)
    rowptr = torch.from_numpy(A.indptr.astype(np.int32)).to(dev)
    col = torch.from_numpy(A.indices.astype(np.int32)).to(dev)
    val = torch.from_numpy(A.data.astype(np.float64)).to(dev)
    b = torch.from_numpy(sy.rhs).to(dev)
    x0 = torch.zeros(sy.n, dtype=torch.float64, device=dev)
    x0[0] = 1.0                                              # the reference's start vector e0
    tol = 1e-10 * float(np.linalg.norm(sy.rhs))

    # the allocating entry point
    M = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    x_ref = x0.clone()
    torch.cuda.synchronize()
    opts = N.SolverOpts()
    N.load().jfg_solver_opts_default(C.byref(opts))
    opts.tol = tol
    info = N.SolveInfo()
    st = N.load().jfg_solve_dev(ctx.handle, N.CG, M.handle, N.PREC_NONE, None, _vp(b), _vp(x_ref), C.byref(opts),
                                C.byref(info))
    assert st == N.OK
    ref = x_ref.cpu().numpy()

    for call in range(2):
        x = x0.clone()
        torch.cuda.synchronize()
        it = C.c_int(-1)
        rn = C.c_double(-1.0)
        free_before = torch.cuda.mem_get_info(dev)[0]
        st = N.load().jfg_cg_noalloc(ctx.handle, sy.n, _vp(rowptr), _vp(col), _vp(val), _vp(b), _vp(x), tol, 0,
                                     C.byref(it), C.byref(rn))
        free_after = torch.cuda.mem_get_info(dev)[0]
        assert st == N.OK, (call, N.load().jfg_last_error(ctx.handle))
        if call == 1:      # the first call may load the library's kernels; the second allocates nothing at all
            assert free_after == free_before, (free_before, free_after)
        got = x.cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-8, call
        assert abs(it.value - info.iterations) <= 1, (call, it.value, info.iterations)
        assert 0 <= rn.value <= tol
        r = sy.rhs - A @ got
        assert np.linalg.norm(r) <= tol * 1.01


def test_noalloc_rejects_oversize(ctx):
    dev = torch.device("cuda", ctx.device)
    dummy_i = torch.zeros(4, dtype=torch.int32, device=dev)
    dummy_d = torch.zeros(4, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it = C.c_int()
    rn = C.c_double()
    st = N.load().jfg_cg_noalloc(ctx.handle, NOALLOC_MAX_ROWS + 1, _vp(dummy_i), _vp(dummy_i), _vp(dummy_d),
                                 _vp(dummy_d), _vp(dummy_d), 1e-8, 0, C.byref(it), C.byref(rn))
    assert st == N.ERR_BAD_ARG
    assert b"exceeds the fixed scratch limit" in N.load().jfg_last_error(ctx.handle)


def test_noalloc_reports_indefinite(ctx):
    """An indefinite matrix (diag(1, -1)) meets p.Ap <= 0; the call says so
    through jfg_last_error, as jfg_solve_dev does through info.not_pd."""
    dev = torch.device("cuda", ctx.device)
    rowptr = torch.tensor([0, 1, 2], dtype=torch.int32, device=dev)
    col = torch.tensor([0, 1], dtype=torch.int32, device=dev)
    val = torch.tensor([1.0, -1.0], dtype=torch.float64, device=dev)
    b = torch.tensor([0.0, 1.0], dtype=torch.float64, device=dev)
    x = torch.zeros(2, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it = C.c_int()
    rn = C.c_double()
    st = N.load().jfg_cg_noalloc(ctx.handle, 2, _vp(rowptr), _vp(col), _vp(val), _vp(b), _vp(x), 1e-12, 4,
                                 C.byref(it), C.byref(rn))
    assert st != N.ERR_CUDA
    assert b"not positive definite" in N.load().jfg_last_error(ctx.handle)
