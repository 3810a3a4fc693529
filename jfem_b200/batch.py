"""Batched implicit-Euler time stepping (many independent systems, one launch).

Host-side mirror of the time loop of JFEM's heat example
(Examples/src/HeatEquation.java:81-94) and of
FullyImplicitParabolicIntegrator.timeStep
(Core/src/main/java/basic/FullyImplicitParabolicIntegrator.java:41-53):
every step solves (M + dt A) u^{k+1} = M u^k + f for every system of the batch.
All systems run inside one persistent GPU launch (jfg_batch_heat).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .linalg import DeviceMatrix, IllegalArgumentException


class BatchResult:
    def __init__(self, info: N.BatchInfo, status: int):
        self.status = status
        self.total_inner_iterations = info.total_inner_iterations
        self.max_refine_used = info.max_refine_used
        self.max_rel_residual = info.max_rel_residual
        self.failed = info.failed
        self.cluster = info.cluster
        self.threads = info.threads
        self.rows_per_thread = info.rows_per_thread
        self.ms = info.ms


class BatchedParabolicIntegrator:
    """K[s] = M[s] + dt A[s] and M[s] per system (DeviceMatrix or COO triples)."""

    def __init__(self, K, M, ctx=None):
        if len(K) != len(M) or not K:
            raise IllegalArgumentException("K and M lists differ in length or are empty")
        self._K = [k for k in K]
        self._M = [m for m in M]
        self.ctx = ctx or self._K[0].ctx
        n = len(K)
        Kh = (C.c_void_p * n)(*[k.handle for k in self._K])
        Mh = (C.c_void_p * n)(*[m.handle for m in self._M])
        h = C.c_void_p()
        st = N.load().jfg_batch_create(self.ctx.handle, n, Kh, Mh, C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        self._h = h
        tot = C.c_int64()
        offs = np.zeros(n + 1, dtype=np.int64)
        N.load().jfg_batch_layout(h, C.byref(tot), offs.ctypes.data_as(C.POINTER(C.c_int64)))
        self.offsets = offs
        self.total = tot.value
        self.last = None

    def pack(self, vectors):
        return np.concatenate([N.f64(v) for v in vectors]) if vectors else np.zeros(0)

    def unpack(self, packed):
        return [packed[self.offsets[s]:self.offsets[s + 1]] for s in range(len(self._K))]

    def timeSteps(self, u0, steps, f=None, cluster=0, threads=0, rtol=1e-10, inner_rtol=1e-5, inner_max=500,
                  max_refine=6, rows_per_thread=0):
        """Advance every system `steps` steps; u0 / f: lists of vectors or packed arrays."""
        u = N.f64(u0 if isinstance(u0, np.ndarray) else self.pack(u0)).copy()
        if u.shape != (self.total,):
            raise IllegalArgumentException("packed state has the wrong length")
        fp = None
        if f is not None:
            fp = N.f64(f if isinstance(f, np.ndarray) else self.pack(f))
            if fp.shape != (self.total,):
                raise IllegalArgumentException("packed source has the wrong length")
        o = N.BatchOpts()
        N.load().jfg_batch_opts_default(C.byref(o))
        o.cluster, o.threads, o.rows_per_thread = cluster, threads, rows_per_thread
        o.rtol, o.inner_rtol, o.inner_max, o.max_refine = rtol, inner_rtol, inner_max, max_refine
        info = N.BatchInfo()
        st = N.load().jfg_batch_heat(self._h, int(steps), N.dptr(fp) if fp is not None else None, N.dptr(u),
                                     C.byref(o), C.byref(info))
        self.ctx.check(st, allow=(N.OK, N.NOT_CONVERGED, N.NONFINITE))
        self.last = BatchResult(info, st)
        return u

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_batch_free(self._h)
        except Exception:
            pass
