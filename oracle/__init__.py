"""CPU oracle for JFEM's linear-solve path (test infrastructure only).

This package wraps ``jfem_oracle.c`` -- a plain-C FP64 restatement of the
reference's Java solver routines (each C function cites the Java file:line it
follows).  It is the parity checker for the CUDA library and the timed CPU
baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg import it; the product package ``jfem_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "jfem_oracle.c")
_LIB = os.path.join(_HERE, "libjfem_oracle.so")

OK, MAXITER, BREAKDOWN, NONFINITE, BADARG, SINGULAR = range(6)
SMOOTH_JACOBI, SMOOTH_RICHARDSON, SMOOTH_FBGS, SMOOTH_GS = 0, 1, 3, 4


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (recipe also in oracle/Makefile)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-shared", "-o", _LIB, _SRC,
                               "-lm"])
    return _LIB


def set_threads(n: int) -> int:
    """Threads of the loops the reference runs as parallel streams; returns
    the count in effect."""
    lib().or_set_threads(int(n))
    return lib().or_threads()


def threads() -> int:
    return lib().or_threads()


class _Info(C.Structure):
    _fields_ = [("iterations", C.c_int), ("restarts", C.c_int), ("status", C.c_int),
                ("final_norm", C.c_double), ("hist_len", C.c_int)]


_lib = None
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        L.or_mat_new.restype = _P
        L.or_mat_new.argtypes = [C.c_int, C.c_int, C.c_longlong, _I, _I, _D]
        L.or_mat_free.argtypes = [_P]
        for f in ("or_mat_mvmul", "or_mat_tvmul", "or_mat_mvmul_rows", "or_mat_tvmul_cols"):
            getattr(L, f).argtypes = [_P, _D, _D]
        L.or_mat_nnz.restype = C.c_longlong
        L.or_mat_nnz.argtypes = [_P]
        L.or_mat_coo.argtypes = [_P, _I, _I, _D]
        L.or_mat_mmmul.restype = _P
        L.or_mat_mmmul.argtypes = [_P, _P]
        L.or_gs_smooth.argtypes = [_P, C.c_int, C.c_int, _I, _D, _D]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_threads.restype = C.c_int
        L.or_mat_diag.argtypes = [_P, _D]
        L.or_mat_dense.argtypes = [_P, _D]
        L.or_jrandom_doubles.argtypes = [C.c_longlong, C.c_longlong, _D]
        L.or_dense_solve.argtypes = [C.c_int, _D, _D, _D]
        L.or_dense_inverse.argtypes = [C.c_int, _D, _D]
        L.or_op_matrix.restype = _P
        L.or_op_matrix.argtypes = [_P]
        L.or_op_identity.restype = _P
        L.or_op_identity.argtypes = [C.c_int]
        L.or_op_free.argtypes = [_P]
        L.or_op_apply.argtypes = [_P, _D, _D]
        L.or_solve_cg.argtypes = [_P, _D, _D, C.c_double, C.c_int, C.POINTER(_Info), _D, C.c_int]
        L.or_solve_pcg.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, C.POINTER(_Info), _D, C.c_int]
        L.or_solve_bicgstab.argtypes = [_P, _D, _D, C.c_double, C.c_int, C.POINTER(_Info), _D, C.c_int]
        L.or_solve_pbicgstab.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, C.POINTER(_Info), _D, C.c_int]
        L.or_solve_gmres.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, C.c_int, C.POINTER(_Info), _D, C.c_int]
        L.or_solve_gmres2.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, C.c_int, C.POINTER(_Info), _D, C.c_int]
        L.or_smooth.argtypes = [_P, C.c_int, C.c_int, C.c_double, _D, _D]
        L.or_mg_new.restype = _P
        L.or_mg_new.argtypes = [C.c_int, C.POINTER(_P), C.POINTER(_P), C.POINTER(_I), _I, _I, _I, _D, C.c_int]
        L.or_mg_free.argtypes = [_P]
        L.or_mg_vcycle.argtypes = [_P, _D, _D, _D]
        L.or_mg_fmg.argtypes = [_P, _D, _D]
        L.or_mg_apply.argtypes = [_P, _D, _D]
        L.or_mg_apply_ex.argtypes = [_P, C.c_int, C.c_int, _D, _D]
        L.or_mg_apply_kind.argtypes = [_P, C.c_int, C.c_int, C.c_int, _D, _D]
        L.or_mg_wcycle.argtypes = [_P, _D, _D, _D]
        L.or_op_mg.restype = _P
        L.or_op_mg.argtypes = [_P, C.c_int, C.c_int]
        L.or_op_mg_kind.restype = _P
        L.or_op_mg_kind.argtypes = [_P, C.c_int, C.c_int, C.c_int]
        L.or_op_mg_free.argtypes = [_P]
        L.or_mg_coarse_status.argtypes = [_P]
        L.or_mg_set_schwarz.argtypes = [_P, C.c_int, _P, C.c_int]
        L.or_op_blockdiag.restype = _P
        L.or_op_blockdiag.argtypes = [_P, C.c_int, _D]
        L.or_schwarz_new.restype = _P
        L.or_schwarz_new.argtypes = [_P, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_longlong), _I, C.c_int, _I,
                                     _I]
        L.or_schwarz_status.argtypes = [_P]
        L.or_schwarz_free.argtypes = [_P]
        L.or_schwarz_apply.argtypes = [_P, _D, _D]
        L.or_schwarz_solve.argtypes = [_P, _D, _D]
        L.or_schwarz_smooth.argtypes = [_P, C.c_int, _D, _D]
        L.or_schwarz_inverse.restype = _D
        L.or_schwarz_inverse.argtypes = [_P, C.c_int, _I]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def java_random_doubles(seed: int, count: int) -> np.ndarray:
    """``new java.util.Random(seed).nextDouble()`` repeated ``count`` times."""
    out = np.empty(count, dtype=np.float64)
    lib().or_jrandom_doubles(seed, count, _d(out))
    return out


class CooMatrix:
    """COO triples in storage order, SparseMatrix.java semantics."""

    def __init__(self, rows, cols, ri, ci, v):
        self.rows, self.cols = int(rows), int(cols)
        self.ri, self.ci, self.v = _i32(ri), _i32(ci), _f64(v)
        h = lib().or_mat_new(self.rows, self.cols, len(self.v), _i(self.ri), _i(self.ci), _d(self.v))
        if not h:
            raise ValueError("invalid COO triples")
        self._h = h
        self._op = lib().or_op_matrix(h)

    def __del__(self):
        try:
            lib().or_op_free(self._op)
            lib().or_mat_free(self._h)
        except Exception:
            pass

    def mvmul(self, x):
        x = _f64(x)
        y = np.empty(self.rows)
        lib().or_mat_mvmul(self._h, _d(x), _d(y))
        return y

    def tvmul(self, x):
        x = _f64(x)
        y = np.empty(self.cols)
        lib().or_mat_tvmul(self._h, _d(x), _d(y))
        return y

    def mvmul_rows(self, x):
        x = _f64(x)
        y = np.empty(self.rows)
        lib().or_mat_mvmul_rows(self._h, _d(x), _d(y))
        return y

    def tvmul_cols(self, x):
        x = _f64(x)
        y = np.empty(self.cols)
        lib().or_mat_tvmul_cols(self._h, _d(x), _d(y))
        return y

    def diag(self):
        d = np.empty(min(self.rows, self.cols))
        lib().or_mat_diag(self._h, _d(d))
        return d

    def dense(self):
        a = np.empty((self.rows, self.cols))
        lib().or_mat_dense(self._h, _d(a))
        return a

    def mmmul(self, other: "CooMatrix") -> "CooMatrix":
        """SparseMatrix.mmMul: self * other (row-major triples, zero sums dropped)."""
        h = lib().or_mat_mmmul(self._h, other._h)
        if not h:
            raise ValueError("Incompatible sizes")
        try:
            m = lib().or_mat_nnz(h)
            ri = np.empty(m, dtype=np.int32)
            ci = np.empty(m, dtype=np.int32)
            v = np.empty(m)
            lib().or_mat_coo(h, _i(ri), _i(ci), _d(v))
        finally:
            lib().or_mat_free(h)
        return CooMatrix(self.rows, other.cols, ri, ci, v)

    def transpose(self) -> "CooMatrix":
        """SparseMatrix.transpose (SparseMatrix.java:469-478): triples with rows and columns exchanged."""
        return CooMatrix(self.cols, self.rows, self.ci, self.ri, self.v)

    def tmmul(self, other: "CooMatrix") -> "CooMatrix":
        """Matrix.tmMul (Matrix.java:142-148): transpose().mmMul(other)."""
        return self.transpose().mmmul(other)


def dense_solve(a, b):
    a = _f64(a)
    b = _f64(b)
    x = np.empty(len(b))
    st = lib().or_dense_solve(a.shape[0], _d(a), _d(b), _d(x))
    if st != OK:
        raise np.linalg.LinAlgError("singular")
    return x


def dense_inverse(a):
    a = _f64(a)
    out = np.empty_like(a)
    st = lib().or_dense_inverse(a.shape[0], _d(a), _d(out))
    if st != OK:
        raise np.linalg.LinAlgError("singular")
    return out


class Result:
    def __init__(self, x, info, hist):
        self.x = x
        self.iterations = info.iterations
        self.restarts = info.restarts
        self.status = info.status
        self.final_norm = info.final_norm
        self.history = hist[: min(info.hist_len, len(hist))].copy()


def _op(M):
    if M is None:
        return None
    if isinstance(M, (CooMatrix, MGPreconditioner, BlockDiagonal)):
        return M._op
    raise TypeError(type(M))


class BlockDiagonal:
    """diag(velocity multigrid, pressure scaling) over velocity-first unknowns."""

    def __init__(self, mg: "MGPreconditioner", pinv):
        self.mg = mg
        self._pinv = _f64(pinv)
        self._op = lib().or_op_blockdiag(mg._op, self._pinv.size, _d(self._pinv))
        self.n = mg.n + self._pinv.size

    def mvmul(self, v):
        out = np.empty(self.n)
        lib().or_op_apply(self._op, _d(_f64(v)), _d(out))
        return out

    def __del__(self):
        try:
            lib().or_op_free(self._op)
        except Exception:
            pass


def _run(fn, *args, x0, hist_cap=100000):
    x = _f64(x0).copy()
    info = _Info()
    hist = np.zeros(hist_cap)
    fn(*args[:-1], _d(x), *args[-1], C.byref(info), _d(hist), hist_cap)
    return Result(x, info, hist)


def start_iterate(n):
    """The reference's default start vector e0 (IterativeSolver.java:69-70)."""
    x = np.zeros(n)
    x[0] = 1.0
    return x


def solve_cg(A: CooMatrix, b, tol, x0=None, maxit=0):
    b = _f64(b)
    x0 = start_iterate(len(b)) if x0 is None else x0
    return _run(lib().or_solve_cg, A._op, _d(b), (C.c_double(tol), maxit), x0=x0)


def solve_pcg(A, M, b, tol, x0=None, maxit=0):
    b = _f64(b)
    x0 = start_iterate(len(b)) if x0 is None else x0
    return _run(lib().or_solve_pcg, A._op, _op(M), _d(b), (C.c_double(tol), maxit), x0=x0)


def solve_bicgstab(A, b, tol, x0=None, maxit=0):
    b = _f64(b)
    x0 = start_iterate(len(b)) if x0 is None else x0
    return _run(lib().or_solve_bicgstab, A._op, _d(b), (C.c_double(tol), maxit), x0=x0)


def solve_pbicgstab(A, M, b, tol, x0=None, maxit=0):
    b = _f64(b)
    x0 = start_iterate(len(b)) if x0 is None else x0
    return _run(lib().or_solve_pbicgstab, A._op, _op(M), _d(b), (C.c_double(tol), maxit), x0=x0)


def solve_gmres(A, b, tol, M=None, x0=None, restart=150, max_restarts=200):
    """GMRES.solve: e0 start without a preconditioner, zero start with one
    (GMRES.java:40-62)."""
    b = _f64(b)
    if x0 is None:
        x0 = start_iterate(len(b)) if M is None else np.zeros(len(b))
    return _run(lib().or_solve_gmres, A._op, _op(M), _d(b), (C.c_double(tol), restart, max_restarts), x0=x0)


def solve_gmres2(A, b, tol, M=None, x0=None, maxit=0, max_restarts=200):
    b = _f64(b)
    x0 = start_iterate(len(b)) if x0 is None else x0
    return _run(lib().or_solve_gmres2, A._op, _op(M), _d(b), (C.c_double(tol), maxit, max_restarts), x0=x0)


def gs_smooth(A: CooMatrix, kind, runs, rhs, x, rank=None):
    """ForwardBackwardGaussSeidelSmoother (kind SMOOTH_FBGS) / GaussSeidelSmoother
    (SMOOTH_GS) in the ordering `rank` (natural when None)."""
    x = _f64(x).copy()
    rk = None if rank is None else _i32(rank)
    st = lib().or_gs_smooth(A._h, kind, runs, _i(rk) if rk is not None else None, _d(_f64(rhs)), _d(x))
    if st == SINGULAR:
        raise np.linalg.LinAlgError("Singular Matrix")
    return x


def smooth(A: CooMatrix, kind, runs, omega, rhs, x):
    x = _f64(x).copy()
    rhs = _f64(rhs)
    lib().or_smooth(A._h, kind, runs, omega, _d(rhs), _d(x))
    return x


class MGPreconditioner:
    """MGPreconditionerInterface over explicit level data.

    ``mats[l]`` is the system on level l (0 = coarsest), ``prolong[l]`` the
    n_{l+1} x n_l prolongation, ``bdry[l]`` the Dirichlet node list,
    ``smoothers[l]`` a (kind, runs, omega) triple for l >= 1.
    use_fmg/cycles select the reference mvMul (FMG + cycles V-cycles) or a
    single V-cycle (use_fmg=False, cycles=1); cycle="W" selects mvMulW
    (wCycle in place of vCycle, MGPreconditionerSpace.java:165-183).
    """

    def __init__(self, mats, prolong, bdry, smoothers, cycles=3, use_fmg=True, cycle="V"):
        L = len(mats)
        self.mats, self.prolong = mats, prolong
        self._bd = [_i32(b) for b in bdry]
        A = (_P * L)(*[m._h for m in mats])
        P = (_P * L)(*([p._h for p in prolong] + [None]))
        BD = (_I * L)(*[_i(b) for b in self._bd])
        NBD = np.array([len(b) for b in self._bd], dtype=np.int32)
        sm = list(smoothers) if len(smoothers) == L else [None] + list(smoothers)
        kind = np.array([0 if s is None else s[0] for s in sm], dtype=np.int32)
        runs = np.array([0 if s is None else s[1] for s in sm], dtype=np.int32)
        omg = np.array([0.0 if s is None else s[2] for s in sm], dtype=np.float64)
        self._h = lib().or_mg_new(L, A, P, BD, _i(NBD), _i(kind), _i(runs), _d(omg), cycles)
        if lib().or_mg_coarse_status(self._h) != OK:
            raise np.linalg.LinAlgError("coarsest matrix singular")
        if cycle not in ("V", "W"):
            raise ValueError("cycle must be 'V' or 'W'")
        self._op = lib().or_op_mg_kind(self._h, 1 if use_fmg else 0, cycles, 1 if cycle == "W" else 0)
        self.n = mats[-1].rows

    def __del__(self):
        try:
            lib().or_op_mg_free(self._op)
            lib().or_mg_free(self._h)
        except Exception:
            pass

    def vcycle(self, x0, rhs):
        out = np.empty(self.n)
        lib().or_mg_vcycle(self._h, _d(_f64(x0)), _d(_f64(rhs)), _d(out))
        return out

    def wcycle(self, x0, rhs):
        out = np.empty(self.n)
        lib().or_mg_wcycle(self._h, _d(_f64(x0)), _d(_f64(rhs)), _d(out))
        return out

    def fmg(self, defect):
        out = np.empty(self.n)
        lib().or_mg_fmg(self._h, _d(_f64(defect)), _d(out))
        return out

    def apply(self, v, use_fmg=True, cycles=None, cycle="V"):
        out = np.empty(self.n)
        lib().or_mg_apply_kind(self._h, 1 if use_fmg else 0, 3 if cycles is None else cycles,
                               1 if cycle == "W" else 0, _d(_f64(v)), _d(out))
        return out

    def mvmul(self, v):
        out = np.empty(self.n)
        lib().or_op_apply(self._op, _d(_f64(v)), _d(out))
        return out

    def set_schwarz(self, level: int, schwarz: "Schwarz", runs: int):
        """Level ``level`` smooths with SchwarzSmoother(runs, schwarz)."""
        self._keep = getattr(self, "_keep", []) + [schwarz]
        lib().or_mg_set_schwarz(self._h, level, schwarz._h, runs)


SCHWARZ_MULTIPLICATIVE, SCHWARZ_COLORED, SCHWARZ_ADDITIVE = 0, 1, 2


class Schwarz:
    """UpFrontSchwarz + DirectSolver + one SubspaceCorrection over explicit
    patch DOF lists (and colours for the coloured correction)."""

    def __init__(self, A: CooMatrix, kind: int, patches, omega: float = 1.0, colours=None):
        self.A = A
        self.n = A.rows
        ptr = np.zeros(len(patches) + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([len(p) for p in patches])
        dofs = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int32) for p in patches]),
                                    dtype=np.int32)
        if colours is None:
            colours = []
        cptr = np.zeros(len(colours) + 1, dtype=np.int32)
        cptr[1:] = np.cumsum([len(c) for c in colours]) if colours else []
        cpat = np.ascontiguousarray(np.concatenate([np.asarray(c, dtype=np.int32) for c in colours])
                                    if colours else np.zeros(1, dtype=np.int32), dtype=np.int32)
        self._h = lib().or_schwarz_new(A._h, kind, omega, len(patches), ptr.ctypes.data_as(C.POINTER(C.c_longlong)),
                                       _i(dofs), len(colours), _i(cptr), _i(cpat))
        if lib().or_schwarz_status(self._h) != OK:
            lib().or_schwarz_free(self._h)
            self._h = None
            raise np.linalg.LinAlgError("singular patch matrix")

    def __del__(self):
        try:
            if self._h:
                lib().or_schwarz_free(self._h)
        except Exception:
            pass

    def apply(self, x, rhs):
        x = _f64(x).copy()
        lib().or_schwarz_apply(self._h, _d(x), _d(_f64(rhs)))
        return x

    def solve(self, rhs):
        out = np.empty(self.n)
        lib().or_schwarz_solve(self._h, _d(_f64(rhs)), _d(out))
        return out

    def smooth(self, runs, rhs, x):
        x = _f64(x).copy()
        lib().or_schwarz_smooth(self._h, runs, _d(_f64(rhs)), _d(x))
        return x

    def inverse(self, p):
        m = C.c_int()
        ptr = lib().or_schwarz_inverse(self._h, p, C.byref(m))
        return np.ctypeslib.as_array(ptr, shape=(m.value * m.value,)).reshape(m.value, m.value).copy()
