"""ctypes binding of libjfem_gpu.so (the C ABI declared in include/jfem_gpu.h).

The library is the only compute path: if it is missing or no CUDA device is
present, every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libjfem_gpu.so")

# jfg_status
OK, NOT_CONVERGED, BREAKDOWN, NONFINITE, ERR_BAD_ARG, ERR_SINGULAR, ERR_CUDA, ERR_NO_DEVICE, ERR_UNSUPPORTED = range(9)
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "BREAKDOWN", 3: "NONFINITE", 4: "BAD_ARG", 5: "SINGULAR",
                6: "CUDA", 7: "NO_DEVICE", 8: "UNSUPPORTED"}
# jfg_solver_kind
CG, PCG, BICGSTAB, PBICGSTAB, GMRES, PGMRES, GMRES2, FGMRES = range(8)
# jfg_precond_kind
PREC_NONE, PREC_MG, PREC_JACOBI, PREC_MATRIX, PREC_MG_CNN, PREC_SCHWARZ, PREC_BLOCKDIAG = range(7)
# jfg_precision
FP64, MIXED, MIXED_PRECOND = 0, 1, 2
SMOOTH_JACOBI, SMOOTH_RICHARDSON, SMOOTH_SCHWARZ, SMOOTH_FBGS, SMOOTH_GS = 0, 1, 2, 3, 4
GS_NATURAL, GS_MULTICOLOR = 0, 1
SCHWARZ_MULTIPLICATIVE, SCHWARZ_COLORED, SCHWARZ_ADDITIVE = 0, 1, 2

# Every symbol include/jfem_gpu.h declares.
EXPORTED = [
    "jfg_create", "jfg_destroy", "jfg_last_error", "jfg_synchronize", "jfg_release_scratch", "jfg_stream",
    "jfg_version",
    "jfg_kernel_launches",
    "jfg_matrix_from_coo", "jfg_matrix_free", "jfg_matrix_info", "jfg_spmv", "jfg_spmv_t", "jfg_spmv_dev",
    "jfg_spmv_t_dev", "jfg_spmv_f32_dev", "jfg_spmv_lowp_dev", "jfg_matrix_layout", "jfg_matrix_diag", "jfg_spmv_time", "jfg_spmv_time_rotating", "jfg_smooth",
    "jfg_matrix_csr", "jfg_matrix_mmmul", "jfg_matrix_tmmul", "jfg_matrix_galerkin",
    "jfg_gs_create", "jfg_gs_free", "jfg_gs_info", "jfg_gs_ranks", "jfg_assemble_tp",
    "jfg_assemble_taylor_hood",
    "jfg_mg_create", "jfg_mg_free", "jfg_mg_apply", "jfg_mg_vcycle", "jfg_mg_wcycle", "jfg_mg_fmg",
    "jfg_solver_opts_default", "jfg_solve", "jfg_solve_dev",
    "jfg_dense_solve", "jfg_dense_inverse", "jfg_sparse_solve", "jfg_cg_noalloc",
    "jfg_batch_opts_default", "jfg_batch_create", "jfg_batch_free", "jfg_batch_layout", "jfg_batch_heat",
    "jfg_cnn_num_params", "jfg_cnn_create", "jfg_cnn_free", "jfg_cnn_set_weights", "jfg_cnn_get_weights",
    "jfg_cnn_forward_dev", "jfg_cnn_loss_grad_dev", "jfg_cnn_adam_step", "jfg_cnn_time_forward",
    "jfg_mgcnn_create", "jfg_mgcnn_set", "jfg_mgcnn_apply_dev", "jfg_mgcnn_free",
    "jfg_schwarz_create", "jfg_schwarz_free", "jfg_schwarz_info", "jfg_schwarz_apply", "jfg_schwarz_solve",
    "jfg_schwarz_smooth", "jfg_schwarz_smooth_dev", "jfg_schwarz_local_inverse", "jfg_schwarz_time",
    "jfg_blockdiag_create", "jfg_blockdiag_apply", "jfg_blockdiag_free",
    "jfg_schur_create", "jfg_schur_apply", "jfg_schur_solve", "jfg_schur_free",
]


class SmootherDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("runs", C.c_int), ("omega", C.c_double), ("schwarz", C.c_void_p),
                ("gs", C.c_void_p)]


class TPDesc(C.Structure):
    _fields_ = [("p", C.c_int), ("cx", C.c_int), ("cy", C.c_int), ("x0", C.c_double), ("x1", C.c_double),
                ("y0", C.c_double), ("y1", C.c_double), ("grad_coef", C.c_double), ("mass_coef", C.c_double),
                ("dirichlet", C.c_int)]


class MGDesc(C.Structure):
    _fields_ = [("cycles", C.c_int), ("use_fmg", C.c_int), ("precision", C.c_int), ("cycle", C.c_int)]


class SolverOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("maxit", C.c_int), ("restart", C.c_int), ("max_restarts", C.c_int),
                ("precision", C.c_int), ("inner_rtol", C.c_double), ("use_graph", C.c_int),
                ("graph_chunk", C.c_int), ("h_history", C.POINTER(C.c_double)), ("history_cap", C.c_int),
                ("start", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("restarts", C.c_int), ("status", C.c_int),
                ("outer_iterations", C.c_int), ("final_residual", C.c_double), ("final_norm", C.c_double),
                ("history_len", C.c_int), ("not_pd", C.c_int)]


class BatchOpts(C.Structure):
    _fields_ = [("cluster", C.c_int), ("threads", C.c_int), ("rtol", C.c_double), ("inner_rtol", C.c_double),
                ("inner_max", C.c_int), ("max_refine", C.c_int), ("rows_per_thread", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [("total_inner_iterations", C.c_int), ("max_refine_used", C.c_int),
                ("max_rel_residual", C.c_double), ("failed", C.c_int), ("cluster", C.c_int),
                ("threads", C.c_int), ("ms", C.c_double), ("rows_per_thread", C.c_int)]


class JfgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)


def load():
    """Loads the CUDA library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library missing: {LIB_PATH} (run python -m jfem_b200.build)")
    L = C.CDLL(LIB_PATH)
    L.jfg_create.argtypes = [C.c_int, C.POINTER(_P)]
    L.jfg_destroy.argtypes = [_P]
    L.jfg_last_error.restype = C.c_char_p
    L.jfg_last_error.argtypes = [_P]
    L.jfg_synchronize.argtypes = [_P]
    L.jfg_release_scratch.argtypes = [_P]
    L.jfg_stream.restype = _P
    L.jfg_stream.argtypes = [_P]
    L.jfg_version.restype = C.c_char_p
    L.jfg_kernel_launches.argtypes = [C.POINTER(C.c_uint64)]
    L.jfg_matrix_from_coo.argtypes = [_P, C.c_int, C.c_int, C.c_int64, _I, _I, _D, C.POINTER(_P)]
    L.jfg_matrix_free.argtypes = [_P]
    L.jfg_matrix_info.argtypes = [_P, _I, _I, C.POINTER(C.c_int64)]
    for f in ("jfg_spmv", "jfg_spmv_t"):
        getattr(L, f).argtypes = [_P, _D, _D]
    for f in ("jfg_spmv_dev", "jfg_spmv_t_dev", "jfg_spmv_f32_dev"):
        getattr(L, f).argtypes = [_P, _P, _P]
    L.jfg_spmv_lowp_dev.argtypes = [_P, C.c_int, _P, _P]
    L.jfg_matrix_layout.argtypes = [_P, _I, _I, _I, _I, C.POINTER(C.c_int64), _D]
    L.jfg_matrix_diag.argtypes = [_P, _D]
    L.jfg_spmv_time.argtypes = [_P, C.c_int, C.c_int, _D]
    L.jfg_spmv_time_rotating.argtypes = [C.POINTER(_P), C.c_int, C.c_int, C.c_int, _D]
    L.jfg_matrix_csr.argtypes = [_P, _I, _I, _D]
    for f in ("jfg_matrix_mmmul", "jfg_matrix_tmmul"):
        getattr(L, f).argtypes = [_P, _P, C.POINTER(_P)]
    L.jfg_matrix_galerkin.argtypes = [_P, _P, _P, C.POINTER(_P)]
    L.jfg_gs_create.argtypes = [_P, _P, C.c_int, C.POINTER(_P)]
    L.jfg_gs_free.argtypes = [_P]
    L.jfg_gs_info.argtypes = [_P, _I, _I, _I]
    L.jfg_gs_ranks.argtypes = [_P, _I]
    L.jfg_assemble_tp.argtypes = [_P, C.POINTER(TPDesc), _D, _D, C.POINTER(_P), _D, _I, _I]
    L.jfg_assemble_taylor_hood.argtypes = [_P, C.c_int, C.c_int, C.c_double, _D, C.c_int, C.c_int, C.POINTER(_P),
                                           _D, _I]
    L.jfg_smooth.argtypes = [_P, C.POINTER(SmootherDesc), _D, _D]
    L.jfg_mg_create.argtypes = [_P, C.c_int, C.POINTER(_P), C.POINTER(_P), C.POINTER(_I), _I,
                                C.POINTER(SmootherDesc), C.POINTER(MGDesc), C.POINTER(_P)]
    L.jfg_mg_free.argtypes = [_P]
    L.jfg_mg_apply.argtypes = [_P, _D, _D]
    L.jfg_mg_vcycle.argtypes = [_P, _D, _D, _D]
    L.jfg_mg_wcycle.argtypes = [_P, _D, _D, _D]
    L.jfg_mg_fmg.argtypes = [_P, _D, _D]
    L.jfg_solver_opts_default.restype = None
    L.jfg_solver_opts_default.argtypes = [C.POINTER(SolverOpts)]
    L.jfg_solve.argtypes = [_P, C.c_int, _P, C.c_int, _P, _D, _D, C.POINTER(SolverOpts), C.POINTER(SolveInfo)]
    L.jfg_solve_dev.argtypes = [_P, C.c_int, _P, C.c_int, _P, _P, _P, C.POINTER(SolverOpts),
                                C.POINTER(SolveInfo)]
    L.jfg_dense_solve.argtypes = [_P, C.c_int, _D, _D, _D]
    L.jfg_dense_inverse.argtypes = [_P, C.c_int, _D, _D]
    L.jfg_sparse_solve.argtypes = [_P, C.c_int, C.c_int64, _I, _I, _D, _D, _D]
    L.jfg_cg_noalloc.argtypes = [_P, C.c_int, _P, _P, _P, _P, _P, C.c_double, C.c_int, _I, _D]
    L.jfg_batch_opts_default.restype = None
    L.jfg_batch_opts_default.argtypes = [C.POINTER(BatchOpts)]
    L.jfg_batch_create.argtypes = [_P, C.c_int, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
    L.jfg_batch_free.argtypes = [_P]
    L.jfg_batch_layout.argtypes = [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.jfg_batch_heat.argtypes = [_P, C.c_int, _D, _D, C.POINTER(BatchOpts), C.POINTER(BatchInfo)]
    L.jfg_cnn_num_params.argtypes = [_I]
    L.jfg_cnn_create.argtypes = [_P, C.POINTER(_P)]
    L.jfg_cnn_free.argtypes = [_P]
    L.jfg_cnn_set_weights.argtypes = [_P, _F]
    L.jfg_cnn_get_weights.argtypes = [_P, _F]
    L.jfg_cnn_forward_dev.argtypes = [_P, C.c_int, C.c_int, C.c_int, _P, _P]
    L.jfg_cnn_loss_grad_dev.argtypes = [_P, C.c_int, C.c_int, C.c_int, _P, _P, _D, _F]
    L.jfg_cnn_adam_step.argtypes = [_P, C.c_double, C.c_double, C.c_double, C.c_double]
    L.jfg_cnn_time_forward.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_int, _D, _D]
    L.jfg_mgcnn_create.argtypes = [_P, _P, _P, _P, C.c_int, C.c_int, _I, _I, C.c_int, C.c_double, C.c_int,
                                   C.POINTER(_P)]
    L.jfg_mgcnn_set.argtypes = [_P, C.c_double, C.c_int]
    L.jfg_mgcnn_apply_dev.argtypes = [_P, _P, _P]
    L.jfg_mgcnn_free.argtypes = [_P]
    L.jfg_schwarz_create.argtypes = [_P, _P, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int64), _I, C.c_int, _I,
                                     _I, C.POINTER(_P)]
    L.jfg_schwarz_free.argtypes = [_P]
    L.jfg_schwarz_info.argtypes = [_P, _I, C.POINTER(C.c_int64), _I]
    L.jfg_schwarz_apply.argtypes = [_P, _D, _D]
    L.jfg_schwarz_solve.argtypes = [_P, _D, _D]
    L.jfg_schwarz_smooth.argtypes = [_P, C.c_int, _D, _D]
    L.jfg_schwarz_smooth_dev.argtypes = [_P, C.c_int, _P, _P]
    L.jfg_schwarz_local_inverse.argtypes = [_P, C.c_int, _I, _I, _D]
    L.jfg_schwarz_time.argtypes = [_P, C.c_int, _D]
    L.jfg_blockdiag_create.argtypes = [_P, _P, C.c_int, C.c_int, _D, C.c_int, C.POINTER(_P)]
    L.jfg_blockdiag_apply.argtypes = [_P, _D, _D]
    L.jfg_blockdiag_free.argtypes = [_P]
    L.jfg_schur_create.argtypes = [_P, _P, C.c_int, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
    L.jfg_schur_apply.argtypes = [_P, _D, _D]
    L.jfg_schur_solve.argtypes = [_P, C.c_int, C.c_int, _P, _D, _D, C.POINTER(SolverOpts), C.POINTER(SolveInfo)]
    L.jfg_schur_free.argtypes = [_P]
    _lib = L
    return L


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_I)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One CUDA stream on one device (jfg_ctx)."""

    def __init__(self, device: int = 0):
        L = load()
        h = _P()
        st = L.jfg_create(device, C.byref(h))
        if st != OK:
            raise JfgError(st, f"cannot create a context on device {device}")
        self._h = h
        self.device = device

    def check(self, st, allow=(OK,)):
        if st not in allow:
            msg = load().jfg_last_error(self._h)
            raise JfgError(st, msg.decode() if msg else "")
        return st

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        self.check(load().jfg_synchronize(self._h))

    def stream_ptr(self) -> int:
        return load().jfg_stream(self._h) or 0

    def close(self):
        if getattr(self, "_h", None):
            load().jfg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launches() -> int:
    c = C.c_uint64()
    load().jfg_kernel_launches(C.byref(c))
    return c.value


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("JFEM_DEVICE", "0")))
    return _default_ctx
