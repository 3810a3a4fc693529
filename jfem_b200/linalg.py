"""Host-side mirror of JFEM's linalg API over the CUDA library.

Names, argument meaning and error behaviour follow the Java classes
(Core/src/main/java/linalg/...): ``SparseMatrix`` (COO triples with
duplicates, ``add``/``set``/``mvMul``/``tvMul``/``solve``), ``DenseMatrix``
(``solve``/``inverse``), ``IterativeSolver`` (``solveCG``, ``solvePCG``,
``solveGMRES``, ``solvePGMRES``, ``solveBiCGStab``, ``solvePBiCGStab`` with the
public fields ``iterations``, ``showProgress`` and the warm start
``lastSolution``) and ``GMRES`` (``ITERATIONS_BEFORE_RESTART``,
``MAX_RESTARTS``).  Vectors are numpy float64 arrays.  Every product and solve
runs in libjfem_gpu.so; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class IllegalArgumentException(ValueError):
    """Raised where the Java code throws IllegalArgumentException."""


class SingularMatrixException(ArithmeticError):
    """The dense solve failed (the JNI layer returns null, sparseSolver.cpp:43-52)."""


class VectorMultiplyable:
    """linalg/VectorMultiplyable.java:8-17."""

    def getVectorSize(self) -> int:
        raise NotImplementedError

    def getTVectorSize(self) -> int:
        raise NotImplementedError

    def mvMul(self, vector):
        raise NotImplementedError

    def tvMul(self, vector):
        raise NotImplementedError


class SparseMatrix(VectorMultiplyable):
    """COO matrix (linalg/SparseMatrix.java).  Triples are kept in storage
    order on the host as the reference keeps them; the device copy (merged,
    row-block CSR) is built on first use and rebuilt after a modification."""

    def __init__(self, rows: int, cols: int, ctx: N.Context | None = None):
        self.rows, self.cols = int(rows), int(cols)
        self._ri: list = []
        self._ci: list = []
        self._v: list = []
        self._arrays = None
        self._dev = None
        self._ctx = ctx

    # -- construction ------------------------------------------------------
    @classmethod
    def from_coo(cls, rows, cols, row_idx, col_idx, vals, ctx=None):
        m = cls(rows, cols, ctx)
        ri, ci, v = N.i32(row_idx), N.i32(col_idx), N.f64(vals)
        if not (ri.size == ci.size == v.size):
            raise IllegalArgumentException("COO arrays differ in length")
        if ri.size and (ri.min() < 0 or ri.max() >= rows or ci.min() < 0 or ci.max() >= cols):
            raise IllegalArgumentException("coordinate out of bounds")
        m._arrays = (ri, ci, v)
        return m

    @classmethod
    def identity(cls, n, ctx=None):
        i = np.arange(n, dtype=np.int32)
        return cls.from_coo(n, n, i, i, np.ones(n), ctx)

    def _flush(self):
        if self._ri:
            add = (np.array(self._ri, np.int32), np.array(self._ci, np.int32), np.array(self._v, np.float64))
            if self._arrays is None:
                self._arrays = add
            else:
                self._arrays = tuple(np.concatenate([a, b]) for a, b in zip(self._arrays, add))
            self._ri, self._ci, self._v = [], [], []
        if self._arrays is None:
            self._arrays = (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0))

    def coo(self):
        self._flush()
        return self._arrays

    def add(self, value, row, col):
        """SparseMatrix.add (SparseMatrix.java:274-294): appends a triple; zero values are skipped."""
        if not (0 <= row < self.rows):
            raise IllegalArgumentException(f"y coordinate out of bounds{row} with rows: {self.rows}")
        if not (0 <= col < self.cols):
            raise IllegalArgumentException("x coordinate out of bounds")
        if value == 0:
            return
        self._ri.append(row)
        self._ci.append(col)
        self._v.append(float(value))
        self._dev = None

    def at(self, row, col):
        ri, ci, v = self.coo()
        return float(v[(ri == row) & (ci == col)].sum())

    def set(self, value, row, col):
        """SparseMatrix.set (:260-271): appends value - at(row, col)."""
        d = value - self.at(row, col)
        self._ri.append(row)
        self._ci.append(col)
        self._v.append(float(d))
        self._dev = None

    def getRows(self):
        return self.rows

    def getCols(self):
        return self.cols

    def getVectorSize(self):
        return self.cols

    def getTVectorSize(self):
        return self.rows

    def getSparseEntryCount(self):
        return int(self.coo()[0].size)

    # -- device side ---------------------------------------------------------
    def device(self) -> "DeviceMatrix":
        if self._dev is None:
            ri, ci, v = self.coo()
            self._dev = DeviceMatrix(self.rows, self.cols, ri, ci, v, self._ctx)
        return self._dev

    def mvMul(self, vector):
        """SparseMatrix.mvMul (:480-489) -- IllegalArgumentException on size mismatch."""
        x = N.f64(vector)
        if x.shape != (self.cols,):
            raise IllegalArgumentException("Incompatible sizes")
        return self.device().spmv(x)

    def tvMul(self, vector):
        x = N.f64(vector)
        if x.shape != (self.rows,):
            raise IllegalArgumentException("Incompatible sizes")
        return self.device().spmv_t(x)

    def diag(self):
        return self.device().diag()

    def _from_device(self, d: "DeviceMatrix") -> "SparseMatrix":
        ri, ci, v = d.coo()
        out = SparseMatrix.from_coo(d.rows, d.cols, ri, ci, v, self._ctx)
        out._dev = d
        return out

    def mmMul(self, matrix: "SparseMatrix") -> "SparseMatrix":
        """SparseMatrix.mmMul (SparseMatrix.java:549-593): the product on the
        GPU, returned as a new SparseMatrix (merged triples, zero sums not stored)."""
        if self.cols != matrix.rows:
            raise IllegalArgumentException("Incompatible sizes")
        return self._from_device(self.device().mmMul(matrix.device()))

    def tmMul(self, matrix: "SparseMatrix") -> "SparseMatrix":
        """Matrix.tmMul (Matrix.java:142-148): self^T * matrix."""
        if self.rows != matrix.rows:
            raise IllegalArgumentException("Incompatible sizes")
        return self._from_device(self.device().tmMul(matrix.device()))

    def transpose(self) -> "SparseMatrix":
        """SparseMatrix.transpose (SparseMatrix.java:469-478): triples with rows and columns exchanged."""
        ri, ci, v = self.coo()
        return SparseMatrix.from_coo(self.cols, self.rows, ci, ri, v, self._ctx)

    def solve(self, rhs):
        """SparseMatrix.solve (:142-145): the drop-in direct solve.  n <= 4096:
        dense LU on the GPU (the reference densifies and factorises too);
        larger: GPU GMRES to a 1e-12 relative residual."""
        if self.rows != self.cols:
            raise IllegalArgumentException("matrix is not square")
        b = N.f64(rhs)
        if b.shape != (self.rows,):
            raise IllegalArgumentException("Incompatible sizes")
        ctx = self._ctx or N.default_context()
        ri, ci, v = self.coo()
        x = np.zeros(self.rows)
        st = N.load().jfg_sparse_solve(ctx.handle, self.rows, v.size, N.iptr(ri), N.iptr(ci), N.dptr(v),
                                       N.dptr(b), N.dptr(x))
        if st == N.ERR_SINGULAR:
            raise SingularMatrixException(N.load().jfg_last_error(ctx.handle).decode())
        ctx.check(st)
        return x


class DeviceMatrix:
    """A matrix resident on the GPU (jfg_mat)."""

    def __init__(self, rows, cols, ri, ci, v, ctx=None):
        self.ctx = ctx or N.default_context()
        self.rows, self.cols = int(rows), int(cols)
        ri, ci, v = N.i32(ri), N.i32(ci), N.f64(v)
        h = C.c_void_p()
        st = N.load().jfg_matrix_from_coo(self.ctx.handle, self.rows, self.cols, v.size, N.iptr(ri), N.iptr(ci),
                                          N.dptr(v), C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        self._h = h
        r, c, nz = C.c_int(), C.c_int(), C.c_int64()
        N.load().jfg_matrix_info(h, C.byref(r), C.byref(c), C.byref(nz))
        self.nnz = nz.value

    @classmethod
    def _adopt(cls, h, ctx):
        """A DeviceMatrix owning the library matrix handle h."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self._h = h
        r, c, nz = C.c_int(), C.c_int(), C.c_int64()
        N.load().jfg_matrix_info(h, C.byref(r), C.byref(c), C.byref(nz))
        self.rows, self.cols, self.nnz = r.value, c.value, nz.value
        return self

    @property
    def handle(self):
        return self._h

    def csr(self):
        """(row pointers, columns, values) of the merged matrix, rows sorted
        and columns ascending within a row."""
        ptr = np.empty(self.rows + 1, dtype=np.int32)
        col = np.empty(max(self.nnz, 1), dtype=np.int32)
        val = np.empty(max(self.nnz, 1))
        self.ctx.check(N.load().jfg_matrix_csr(self._h, N.iptr(ptr), N.iptr(col), N.dptr(val)))
        return ptr, col[: self.nnz], val[: self.nnz]

    def coo(self):
        ptr, col, val = self.csr()
        return np.repeat(np.arange(self.rows, dtype=np.int32), np.diff(ptr)), col, val

    def _product(self, fn, *others):
        h = C.c_void_p()
        st = fn(*[o.handle if o is not None else None for o in (self, *others)], C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        return DeviceMatrix._adopt(h, self.ctx)

    def mmMul(self, other: "DeviceMatrix") -> "DeviceMatrix":
        """SparseMatrix.mmMul (SparseMatrix.java:549-593) on the device."""
        return self._product(N.load().jfg_matrix_mmmul, other)

    def tmMul(self, other: "DeviceMatrix") -> "DeviceMatrix":
        """Matrix.tmMul (Matrix.java:142-148): self^T * other on the device."""
        return self._product(N.load().jfg_matrix_tmmul, other)

    def galerkin(self, prolongation: "DeviceMatrix", restriction: "DeviceMatrix | None" = None) -> "DeviceMatrix":
        """Coarse operator (R A) P, or (P^T A) P without R, with A = self
        (AMGSpace.java:60-78, MGPreconditionerInterface.java:397-402)."""
        h = C.c_void_p()
        st = N.load().jfg_matrix_galerkin(restriction.handle if restriction is not None else None, self._h,
                                          prolongation.handle, C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        return DeviceMatrix._adopt(h, self.ctx)

    def spmv(self, x):
        x = N.f64(x)
        y = np.empty(self.rows)
        self.ctx.check(N.load().jfg_spmv(self._h, N.dptr(x), N.dptr(y)))
        return y

    def spmv_dev(self, x, y=None):
        """y = A x for contiguous FP64 CUDA tensors (returns when y is written)."""
        import torch
        if y is None:
            y = torch.empty(self.rows, dtype=torch.float64, device=x.device)
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_spmv_dev(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())))
        self.ctx.check(N.load().jfg_synchronize(self.ctx.handle))
        return y

    def spmv_t_dev(self, x, y=None):
        """y = A^T x for contiguous FP64 CUDA tensors (returns when y is written)."""
        import torch
        if y is None:
            y = torch.empty(self.cols, dtype=torch.float64, device=x.device)
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_spmv_t_dev(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())))
        self.ctx.check(N.load().jfg_synchronize(self.ctx.handle))
        return y

    def spmv_t(self, x):
        x = N.f64(x)
        y = np.empty(self.cols)
        self.ctx.check(N.load().jfg_spmv_t(self._h, N.dptr(x), N.dptr(y)))
        return y

    def diag(self):
        d = np.empty(min(self.rows, self.cols))
        self.ctx.check(N.load().jfg_matrix_diag(self._h, N.dptr(d)))
        return d

    def spmv_lowp_dev(self, x, values="fp32", y=None):
        """y = A x on FP32 CUDA tensors with the matrix values read as FP32,
        BF16 or scaled FP16 (the formats of the mixed-precision levels)."""
        import torch
        fmt = {"fp32": 0, "bf16": 1, "fp16": 2}[values]
        if y is None:
            y = torch.empty(self.rows, dtype=torch.float32, device=x.device)
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_spmv_lowp_dev(self._h, fmt, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())))
        self.ctx.check(N.load().jfg_synchronize(self.ctx.handle))
        return y

    def layout(self) -> dict:
        """The product layout: {'stencil': bool (the 9-point layout), 'kind'
        ('sell', 'stencil', 'prolongation' or 'restriction'), 'stride',
        'regular_rows', 'other_rows', 'other_nnz', 'fp16_scale_inv'}."""
        st, S, nreg, noth = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        onnz = C.c_int64()
        hs = C.c_double()
        self.ctx.check(N.load().jfg_matrix_layout(self._h, C.byref(st), C.byref(S), C.byref(nreg), C.byref(noth),
                                                  C.byref(onnz), C.byref(hs)))
        return {"stencil": st.value == 1, "kind": ("sell", "stencil", "prolongation", "restriction")[st.value],
                "stride": S.value, "regular_rows": nreg.value, "other_rows": noth.value,
                "other_nnz": int(onnz.value), "fp16_scale_inv": hs.value}

    @staticmethod
    def time_spmv_rotating(mats, precision=0, iters=20):
        """Milliseconds per product over the matrices taken in turn, back to
        back (no L2 flush between launches: the matrices together should
        exceed the L2)."""
        arr = (C.c_void_p * len(mats))(*[m._h.value for m in mats])
        ms = C.c_double()
        mats[0].ctx.check(N.load().jfg_spmv_time_rotating(arr, len(mats), precision, iters, C.byref(ms)))
        return ms.value

    def time_spmv(self, precision=0, iters=50):
        ms = C.c_double()
        self.ctx.check(N.load().jfg_spmv_time(self._h, precision, iters, C.byref(ms)))
        return ms.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_matrix_free(self._h)
        except Exception:
            pass


class DenseMatrix:
    """linalg/DenseMatrix.java: dense solve and inverse (UJMP there, GPU LU here)."""

    def __init__(self, a, ctx=None):
        self.a = np.array(a, dtype=np.float64)
        if self.a.ndim != 2:
            raise IllegalArgumentException("not a matrix")
        self.ctx = ctx or N.default_context()

    @classmethod
    def squareMatrixFromValues(cls, *values):
        n = int(round(len(values) ** 0.5))
        if n * n != len(values):
            raise IllegalArgumentException("nope")
        return cls(np.array(values, dtype=np.float64).reshape(n, n))

    def mvMul(self, v):
        return self.a @ N.f64(v)

    def solve(self, rhs):
        n = self.a.shape[0]
        if self.a.shape != (n, n):
            raise IllegalArgumentException("matrix is not square")
        b = N.f64(rhs)
        x = np.empty(n)
        st = N.load().jfg_dense_solve(self.ctx.handle, n, N.dptr(N.f64(self.a)), N.dptr(b), N.dptr(x))
        if st == N.ERR_SINGULAR:
            raise SingularMatrixException("singular matrix")
        self.ctx.check(st)
        return x

    def inverse(self):
        n = self.a.shape[0]
        out = np.empty((n, n))
        st = N.load().jfg_dense_inverse(self.ctx.handle, n, N.dptr(N.f64(self.a)), N.dptr(out))
        if st == N.ERR_SINGULAR:
            raise SingularMatrixException("singular matrix")
        self.ctx.check(st)
        return out


class GMRES:
    """Public knobs of linalg/GMRES.java:16-19."""

    def __init__(self):
        self.MAX_RESTARTS = 200
        self.ITERATIONS_BEFORE_RESTART = 150


class GMRES2:
    """linalg/GMRES2.java: minimal residual along A-orthonormalised Krylov
    directions (Arnoldi.java).  As in the Java class, the iterate persists
    between calls (field ``iterate``, starting at e0)."""

    def __init__(self, tol: float, ctx: N.Context | None = None):
        self.tol = float(tol)
        self.iterate = None
        self.ctx = ctx
        self.last = None
        self.iterations = 0

    def solve(self, A, b_or_preconditioner, b=None):
        """solve(A, b) or solve(A, M, b) (GMRES2.java:34-58)."""
        if b is None:
            M, rhs = None, b_or_preconditioner
        else:
            M, rhs = b_or_preconditioner, b
        s = IterativeSolver(ctx=self.ctx)
        n = len(rhs)
        if self.iterate is None:
            self.iterate = np.zeros(n)
            self.iterate[0] = 1.0
        x = s._run(N.GMRES2, A, M, rhs, self.tol, self.iterate)
        self.iterate = x
        self.last = s.last
        self.iterations = s.iterations
        return x


class SolveResult:
    def __init__(self, info: N.SolveInfo, history: np.ndarray):
        self.iterations = info.iterations
        self.restarts = info.restarts
        self.status = info.status
        self.outer_iterations = info.outer_iterations
        self.final_residual = info.final_residual
        self.final_norm = info.final_norm
        self.not_pd = bool(info.not_pd)
        self.history = history[: info.history_len].copy()


def _as_device(op) -> DeviceMatrix:
    if isinstance(op, SparseMatrix):
        return op.device()
    if isinstance(op, DeviceMatrix):
        return op
    raise IllegalArgumentException(f"operator of type {type(op).__name__} is not a GPU matrix")


class IterativeSolver:
    """linalg/IterativeSolver.java.  ``precision`` ('fp64', 'mixed' = FP64
    defect correction around FP32 inner solves, or 'mixed-precond' = FP64
    iteration with an FP32 multigrid preconditioner),
    ``use_graph`` and ``history_cap`` select the GPU execution; the defaults
    reproduce the reference's FP64 semantics."""

    def __init__(self, showProgress: bool = False, ctx: N.Context | None = None):
        self.showProgress = showProgress
        self.iterations = 0
        self.lastSolution = None
        self.gm = GMRES()
        self.ctx = ctx
        self.precision = "fp64"
        self.inner_rtol = 1e-4
        self.use_graph = True
        self.history_cap = 4096
        self.last = None          # SolveResult of the last call

    def _run(self, kind, op, prec, rhs, tol, x0, maxit=0, restart=None, device=False):
        A = _as_device(op)
        ctx = A.ctx
        if device:      # FP64 CUDA tensors, x0 is updated in place
            b, x = rhs, x0
            if tuple(b.shape) != (A.rows,) or tuple(x.shape) != (A.rows,):
                raise IllegalArgumentException("Vectors are of different size")
        else:
            b = N.f64(rhs)
            if b.shape != (A.rows,):
                raise IllegalArgumentException("Vectors are of different size")
            x = N.f64(x0).copy()
        pk, ph = N.PREC_NONE, None
        if prec is not None:
            from .multigrid import MGPreconditioner
            from .cnn import MGCNNPreconditioner
            if isinstance(prec, MGPreconditioner):
                pk, ph = N.PREC_MG, prec.handle
            elif isinstance(prec, MGCNNPreconditioner):
                pk, ph = N.PREC_MG_CNN, prec.handle
            elif hasattr(prec, "correction") and hasattr(prec, "patches"):     # a Schwarz decomposition
                pk, ph = N.PREC_SCHWARZ, prec.handle
            elif type(prec).__name__ == "BlockDiagonalPreconditioner":
                pk, ph = N.PREC_BLOCKDIAG, prec.handle
            elif isinstance(prec, (SparseMatrix, DeviceMatrix)):
                pk, ph = N.PREC_MATRIX, _as_device(prec).handle
            elif prec == "jacobi":
                pk = N.PREC_JACOBI
            else:
                raise IllegalArgumentException(f"unsupported preconditioner {type(prec).__name__}")
        opts = N.SolverOpts()
        N.load().jfg_solver_opts_default(C.byref(opts))
        opts.tol = tol
        opts.maxit = maxit
        opts.restart = self.gm.ITERATIONS_BEFORE_RESTART if restart is None else restart
        opts.max_restarts = self.gm.MAX_RESTARTS
        modes = {"fp64": N.FP64, "mixed": N.MIXED, "mixed-precond": N.MIXED_PRECOND}
        if self.precision not in modes:
            raise IllegalArgumentException(f"unknown precision {self.precision!r}")
        opts.precision = modes[self.precision]
        opts.inner_rtol = self.inner_rtol
        opts.use_graph = 1 if self.use_graph else 0
        hist = np.zeros(max(self.history_cap, 1))
        opts.h_history = N.dptr(hist)
        opts.history_cap = self.history_cap
        info = N.SolveInfo()
        if device:
            import torch
            torch.cuda.synchronize()
            st = N.load().jfg_solve_dev(ctx.handle, kind, A.handle, pk, ph, C.c_void_p(b.data_ptr()),
                                        C.c_void_p(x.data_ptr()), C.byref(opts), C.byref(info))
        else:
            st = N.load().jfg_solve(ctx.handle, kind, A.handle, pk, ph, N.dptr(b), N.dptr(x), C.byref(opts),
                                    C.byref(info))
        ctx.check(st, allow=(N.OK, N.NOT_CONVERGED, N.NONFINITE))
        self.last = SolveResult(info, hist)
        self.iterations = info.iterations
        if self.showProgress:
            for i, r in enumerate(self.last.history):
                print(f"residuum norm {i}: {r}")
        self.lastSolution = x
        return x

    def _start(self, n, zero=False):
        if self.lastSolution is not None:
            return self.lastSolution
        x = np.zeros(n)
        if not zero:
            x[0] = 1.0      # iterate.set(1, 0)  (IterativeSolver.java:69-70)
        return x

    def solveCG(self, operator, rhs, tol):
        return self._run(N.CG, operator, None, rhs, tol, self._start(len(rhs)))

    def solvePCG(self, operator, preconditioner, rhs, tol):
        return self._run(N.PCG, operator, preconditioner, rhs, tol, self._start(len(rhs)))

    def solveGMRES(self, operator, rhs, tol):
        return self._run(N.GMRES, operator, None, rhs, tol, self._start(len(rhs)))

    def solvePGMRES(self, operator, preconditioner, rhs, tol):
        # GMRES.solve with a preconditioner starts from zero (GMRES.java:59-60)
        return self._run(N.PGMRES, operator, preconditioner, rhs, tol, self._start(len(rhs), zero=True))

    def solveFGMRES(self, operator, preconditioner, rhs, tol, restart: int = 30):
        """Flexible right-preconditioned GMRES(restart) from zero; no
        counterpart in the reference.  The preconditioner may change from one
        application to the next (the multigrid + learned smoother).  Same
        absolute tolerance and restart semantics as solveGMRES."""
        return self._run(N.FGMRES, operator, preconditioner, rhs, tol, self._start(len(rhs), zero=True),
                         restart=restart)

    def solve_device(self, kind: int, operator, preconditioner, b, x, tol, maxit=0, restart=None):
        """Any solver kind (``_native.CG`` ... ``_native.FGMRES``) on FP64 CUDA
        tensors; x holds the start iterate and receives the solution."""
        return self._run(kind, operator, preconditioner, b, tol, x, maxit=maxit, restart=restart, device=True)

    def solveBiCGStab(self, operator, rhs, tol):
        return self._run(N.BICGSTAB, operator, None, rhs, tol, self._start(len(rhs)))

    def solvePBiCGStab(self, operator, preconditioner, rhs, tol):
        return self._run(N.PBICGSTAB, operator, preconditioner, rhs, tol, self._start(len(rhs)))
