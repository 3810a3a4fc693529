"""Host-side mirror of JFEM's multigrid API over the CUDA library.

``JacobiSmoother`` / ``RichardsonSmoother`` (multigrid/JacobiSmoother.java,
multigrid/RichardsonSmoother.java) expose ``smooth(operator, rhs, iterate)``;
``MGPreconditioner`` is the preconditioner of
multigrid/MGPreconditionerInterface.java (``mvMul``, ``vCycle``,
``fullVCycleCorrection``, ``cycles``) over explicit level systems,
prolongation matrices and Dirichlet node lists, the data that
MGPreconditionerSpace builds (multigrid/MGPreconditionerSpace.java:28-57).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .linalg import DeviceMatrix, IllegalArgumentException, SparseMatrix, VectorMultiplyable, _as_device


class JacobiSmoother:
    def __init__(self, runs: int, omega: float, A=None):
        self.runs, self.omega = int(runs), float(omega)
        self.kind = N.SMOOTH_JACOBI

    def desc(self):
        return N.SmootherDesc(self.kind, self.runs, self.omega)

    def smooth(self, operator, rhs, iterate, verbose=False, prefix=""):
        A = _as_device(operator)
        x = N.f64(iterate).copy()
        b = N.f64(rhs)
        if b.shape != (A.rows,) or x.shape != (A.rows,):
            raise IllegalArgumentException("Incompatible sizes")
        d = self.desc()
        A.ctx.check(N.load().jfg_smooth(A.handle, C.byref(d), N.dptr(b), N.dptr(x)))
        return x


class RichardsonSmoother(JacobiSmoother):
    def __init__(self, omega: float, runs: int):
        self.runs, self.omega = int(runs), float(omega)
        self.kind = N.SMOOTH_RICHARDSON


class ForwardBackwardGaussSeidelSmoother(JacobiSmoother):
    """multigrid/ForwardBackwardGaussSeidelSmoother.java: runs x
    { x += L^-1 D U^-1 (b - A x) } with the triangles of A.  ordering
    "natural" is the reference's row order; "multicolour" applies the same
    smoother to A permuted colour by colour (one parallel step per colour)."""

    _kind = N.SMOOTH_FBGS

    def __init__(self, runs: int, A, ordering: str = "natural"):
        orders = {"natural": N.GS_NATURAL, "multicolour": N.GS_MULTICOLOR, "multicolor": N.GS_MULTICOLOR}
        if ordering not in orders:
            raise IllegalArgumentException(f"unknown ordering {ordering!r}")
        self.runs, self.omega, self.kind = int(runs), 1.0, self._kind
        self.A = _as_device(A)
        if self.A.rows != self.A.cols:
            raise IllegalArgumentException("must be square")
        h = C.c_void_p()
        st = N.load().jfg_gs_create(self.A.ctx.handle, self.A.handle, orders[ordering], C.byref(h))
        if st == N.ERR_SINGULAR:
            from .linalg import SingularMatrixException
            raise SingularMatrixException(N.load().jfg_last_error(self.A.ctx.handle).decode())
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.A.ctx.handle).decode())
        self.A.ctx.check(st)
        self._h = h
        self.ordering = ordering

    @property
    def handle(self):
        return self._h

    def desc(self):
        return N.SmootherDesc(self.kind, self.runs, self.omega, None, self._h)

    def info(self):
        """(forward levels, backward levels, colours)."""
        f, b, c = C.c_int(), C.c_int(), C.c_int()
        N.load().jfg_gs_info(self._h, C.byref(f), C.byref(b), C.byref(c))
        return f.value, b.value, c.value

    def ranks(self):
        r = np.empty(self.A.rows, dtype=np.int32)
        self.A.ctx.check(N.load().jfg_gs_ranks(self._h, N.iptr(r)))
        return r

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_gs_free(self._h)
        except Exception:
            pass


class GaussSeidelSmoother(ForwardBackwardGaussSeidelSmoother):
    """multigrid/GaussSeidelSmoother.java: runs x { x = (L + D)^-1 (b - R x) },
    R the strict upper triangle (the reference inverts L + D densely; here it
    is a forward substitution)."""

    _kind = N.SMOOTH_GS


class MGPreconditioner(VectorMultiplyable):
    """Geometric multigrid preconditioner on the GPU.

    systems[l]: level matrices (0 = coarsest); prolongations[l]: n_{l+1} x n_l;
    boundary[l]: Dirichlet node lists; smoothers[l] for l >= 1 (entry 0 may be
    None).  cycles / use_fmg follow MGPreconditionerInterface.mvMul; the plain
    one-V-cycle preconditioner is cycles=1, use_fmg=False.
    precision="mixed" also builds the FP32 hierarchy used by mixed solves;
    "mixed-bf16" builds it with BF16 matrix values (FP32 vectors and sums);
    "mixed-fp16" with FP16 matrix values scaled by a power of two per matrix.
    cycle="W" makes the application MGPreconditionerSpace.mvMulW (wCycle in
    place of vCycle, multigrid/MGPreconditionerSpace.java:165-183).
    """

    def __init__(self, systems, prolongations, boundary, smoothers, cycles=3, use_fmg=True, precision="fp64",
                 ctx=None, cycle="V"):
        L = len(systems)
        if len(prolongations) != L - 1 or len(boundary) != L:
            raise IllegalArgumentException("level data of inconsistent length")
        self._A = [_as_device(s) for s in systems]
        self._P = [_as_device(p) for p in prolongations]
        self.ctx = ctx or self._A[0].ctx
        self._bd = [N.i32(b) for b in boundary]
        sm = list(smoothers)
        if len(sm) == L - 1:
            sm = [None] + sm
        if len(sm) != L:
            raise IllegalArgumentException("one smoother per level above the coarsest")
        self._smoothers = sm        # Schwarz smoothers own device data the hierarchy points to
        descs = (N.SmootherDesc * L)()
        for l, s in enumerate(sm):
            if s is not None:
                descs[l] = s.desc()
        Ah = (C.c_void_p * L)(*[a.handle for a in self._A])
        Ph = (C.c_void_p * max(L, 1))(*([p.handle for p in self._P] + [None]))
        Bh = (C.POINTER(C.c_int) * L)(*[N.iptr(b) for b in self._bd])
        nb = np.array([b.size for b in self._bd], dtype=np.int32)
        levels = {"fp64": 0, "mixed": 1, "mixed-bf16": 2, "mixed-fp16": 3}
        if precision not in levels:
            raise IllegalArgumentException(f"unknown hierarchy precision {precision!r}")
        if cycle not in ("V", "W"):
            raise IllegalArgumentException(f"unknown cycle {cycle!r}")
        desc = N.MGDesc(int(cycles), 1 if use_fmg else 0, levels[precision], 1 if cycle == "W" else 0)
        h = C.c_void_p()
        st = N.load().jfg_mg_create(self.ctx.handle, L, Ah, Ph, Bh, N.iptr(nb), descs, C.byref(desc), C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        self._h = h
        self.n = self._A[-1].rows
        self.cycles = cycles
        self.use_fmg = use_fmg
        self.precision = precision
        self.cycle = cycle

    @property
    def handle(self):
        return self._h

    def getVectorSize(self):
        return self.n

    def getTVectorSize(self):
        return self.n

    def mvMul(self, vector):
        v = N.f64(vector)
        if v.shape != (self.n,):
            raise IllegalArgumentException("wrong size")
        out = np.empty(self.n)
        self.ctx.check(N.load().jfg_mg_apply(self._h, N.dptr(v), N.dptr(out)))
        return out

    def tvMul(self, vector):
        raise NotImplementedError("not implemented yet")   # MGPreconditionerInterface.java:381-385

    def getSystem(self, level: int):
        return self._A[level]

    def getProlongationMatrix(self, level: int):
        return self._P[level]

    def maxLevel(self) -> int:
        return len(self._A) - 1

    def AMGFromMatrix(self, mat, levelToSmoother, isVerbose: bool = False, cycles: int | None = None,
                      precision: str | None = None) -> "MGPreconditioner":
        """MGPreconditionerInterface.AMGFromMatrix (MGPreconditionerInterface.java:387-471):
        a hierarchy whose finest system is `mat` and whose coarser systems are
        the Galerkin products P^T A P of the next finer one (P.tmMul(A).mmMul(P),
        computed on the GPU), with this hierarchy's prolongations, boundary
        handling of the transfers and level count up to the level of `mat`'s
        size; levelToSmoother(l, A_l) gives the smoother of level l >= 1."""
        A = _as_device(mat)
        sizes = [a.rows for a in self._A]
        if A.rows not in sizes:
            raise IllegalArgumentException("Matrix needs to be of same shape as finest system")
        level = max(l for l, n in enumerate(sizes) if n == A.rows)     # levelFromSize
        if A.rows != self._A[level].rows or A.cols != self._A[level].cols:
            raise IllegalArgumentException("Matrix needs to be of same shape as finest system")
        systems = [A]
        for i in range(1, level + 1):
            systems.append(systems[-1].galerkin(self._P[level - i]))
        systems.reverse()
        self.ctx.check(N.load().jfg_release_scratch(self.ctx.handle))
        smoothers = [None] + [levelToSmoother(l, systems[l]) for l in range(1, level + 1)]
        return MGPreconditioner(systems, self._P[:level], self._bd[:level + 1], smoothers,
                                cycles=self.cycles if cycles is None else cycles, use_fmg=self.use_fmg,
                                precision=self.precision if precision is None else precision, ctx=self.ctx,
                                cycle=self.cycle)

    def vCycle(self, initialIterate, rhs):
        x0, b = N.f64(initialIterate), N.f64(rhs)
        if x0.shape != (self.n,) or b.shape != (self.n,):
            raise IllegalArgumentException("wrong size")
        out = np.empty(self.n)
        self.ctx.check(N.load().jfg_mg_vcycle(self._h, N.dptr(x0), N.dptr(b), N.dptr(out)))
        return out

    def wCycle(self, initialIterate, rhs):
        """MGPreconditionerInterface.wCycle (multigrid/MGPreconditionerInterface.java:300-305)."""
        x0, b = N.f64(initialIterate), N.f64(rhs)
        if x0.shape != (self.n,) or b.shape != (self.n,):
            raise IllegalArgumentException("wrong size")
        out = np.empty(self.n)
        self.ctx.check(N.load().jfg_mg_wcycle(self._h, N.dptr(x0), N.dptr(b), N.dptr(out)))
        return out

    def fullVCycleCorrection(self, defect):
        d = N.f64(defect)
        if d.shape != (self.n,):
            raise IllegalArgumentException("wrong size")
        out = np.empty(self.n)
        self.ctx.check(N.load().jfg_mg_fmg(self._h, N.dptr(d), N.dptr(out)))
        return out

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_mg_free(self._h)
        except Exception:
            pass
