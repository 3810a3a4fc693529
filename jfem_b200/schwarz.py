"""Overlapping Schwarz decompositions (schwarz/*.java) on the GPU.

The patch builders run on the host (they only produce DOF lists): cell
blocks of a Cartesian grid (CartesianUpFrontSchwarz, ColoredCartesianSchwarz)
or pressure-node stencils (VankaSchwarz).  Everything numeric -- the local
operators R A R^T, their cached inverses (DirectSolver) and the subspace
corrections -- runs in libjfem_gpu.so (jfg_schwarz_*).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .linalg import IllegalArgumentException, _as_device


class DirectSolver:
    """schwarz/DirectSolver.java: dense inverse of each local operator, cached.

    Inside the device Schwarz decompositions the inverses are built and kept
    on the GPU (k_patch_inverse, one per distinct local operator).  As a
    SystemSolver of its own, solve(system, rhs, patch) follows
    DirectSolver.java:22-38: the first call for a patch inverts the given
    local system (device LU, jfg_dense_inverse) and caches the inverse under
    the patch number; every call returns inverse * rhs."""

    def __init__(self):
        self.inverses = {}

    def solve(self, system, rhs, patch: int):
        from .linalg import DenseMatrix
        patch = int(patch)
        if patch not in self.inverses:
            ctx = getattr(system, "ctx", None)
            if isinstance(system, DenseMatrix):
                a = system.a
            elif hasattr(system, "coo"):            # SparseMatrix / DeviceMatrix: duplicates summed
                r, c, v = system.coo()
                a = np.zeros((int(system.rows), int(system.cols)))
                np.add.at(a, (np.asarray(r), np.asarray(c)), np.asarray(v, dtype=np.float64))
            else:
                a = np.asarray(system, dtype=np.float64)
            if a.ndim != 2 or a.shape[0] != a.shape[1]:
                raise IllegalArgumentException("the local system must be a square matrix")
            self.inverses[patch] = DenseMatrix(a, ctx).inverse()
        b = N.f64(rhs)
        inv = self.inverses[patch]
        if b.shape != (inv.shape[1],):
            raise IllegalArgumentException("Vectors are of different size")
        return inv @ b


class MultiplicativeSubspaceCorrection:
    """schwarz/MultiplicativeSubspaceCorrection.java (patches one after another)."""
    kind = N.SCHWARZ_MULTIPLICATIVE
    omega = 1.0


class AdditiveSubspaceCorrection:
    """schwarz/AdditiveSubspaceCorrection.java (all patches from one residual)."""
    kind = N.SCHWARZ_ADDITIVE

    def __init__(self, omega: float):
        self.omega = float(omega)


class ColoredMultiplicativeSubspaceCorrection:
    """schwarz/ColoredMultiplicativeSubspaceCorrection.java (one residual per colour)."""
    kind = N.SCHWARZ_COLORED

    def __init__(self, omega: float):
        self.omega = float(omega)


def _space_cells(space):
    """(cx, cy, cell_dofs) of a space: cell (ix, iy) is row ix * cy + iy."""
    return space.cx, space.cy, space.cell_dofs


class UpFrontSchwarz:
    """Common part (schwarz/UpFrontSchwarz.java, AbstractSchwarz.java): patch
    DOF lists -> device decomposition with cached patch inverses."""

    def __init__(self, globalMatrix, patches, correction, solver=None, colours=None):
        if solver is not None and not isinstance(solver, DirectSolver):
            raise IllegalArgumentException("only the DirectSolver is implemented")
        self.A = _as_device(globalMatrix)
        self.ctx = self.A.ctx
        self.correction = correction
        self.patches = [np.unique(np.asarray(p, dtype=np.int32)) for p in patches]
        self.colours = colours
        ptr = np.zeros(len(self.patches) + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([p.size for p in self.patches])
        dofs = np.ascontiguousarray(np.concatenate(self.patches), dtype=np.int32)
        if correction.kind == N.SCHWARZ_COLORED:
            if colours is None:
                raise IllegalArgumentException("the coloured correction needs colours")
            cptr = np.zeros(len(colours) + 1, dtype=np.int32)
            cptr[1:] = np.cumsum([len(c) for c in colours])
            cpat = np.ascontiguousarray(np.concatenate([np.asarray(c, dtype=np.int32) for c in colours]),
                                        dtype=np.int32)
            nc = len(colours)
        else:
            cptr = np.zeros(1, dtype=np.int32)
            cpat = np.zeros(1, dtype=np.int32)
            nc = 0
        h = C.c_void_p()
        st = N.load().jfg_schwarz_create(self.ctx.handle, self.A.handle, correction.kind, correction.omega,
                                         len(self.patches), ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                                         N.iptr(dofs), nc, N.iptr(cptr), N.iptr(cpat), C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        self._h = h

    @property
    def handle(self):
        return self._h

    def getPatchCount(self) -> int:
        return len(self.patches)

    def getPatchDoFs(self, patch: int) -> np.ndarray:
        """Rows of the restriction matrix R_patch (ascending global DOFs)."""
        return self.patches[patch]

    def getLocalVector(self, patch: int, v):
        return np.asarray(v)[self.patches[patch]]

    def getGlobalVector(self, patch: int, local):
        out = np.zeros(self.A.rows)
        out[self.patches[patch]] = local
        return out

    def localInverse(self, patch: int) -> np.ndarray:
        m = C.c_int()
        N.load().jfg_schwarz_local_inverse(self._h, patch, C.byref(m), None, None)
        inv = np.empty(m.value * m.value)
        self.ctx.check(N.load().jfg_schwarz_local_inverse(self._h, patch, None, None, N.dptr(inv)))
        return inv.reshape(m.value, m.value)

    def info(self):
        mp, ent, ind = C.c_int(), C.c_int64(), C.c_int()
        N.load().jfg_schwarz_info(self._h, C.byref(mp), C.byref(ent), C.byref(ind))
        return {"max_patch": mp.value, "inverse_entries": ent.value, "independent_colours": ind.value}

    def getVectorSize(self):
        return self.A.rows

    def getTVectorSize(self):
        return self.A.cols

    def mvMul(self, vector):
        """AbstractSchwarz.mvMul = SubspaceCorrection.solve."""
        b = N.f64(vector)
        out = np.empty(self.A.rows)
        self.ctx.check(N.load().jfg_schwarz_solve(self._h, N.dptr(b), N.dptr(out)))
        return out

    def tvMul(self, vector):
        raise IllegalArgumentException("Not implemented")

    def apply(self, iterate, rhs):
        """SubspaceCorrection.apply(schwarz, iterate, rhs)."""
        x = N.f64(iterate).copy()
        self.ctx.check(N.load().jfg_schwarz_apply(self._h, N.dptr(N.f64(rhs)), N.dptr(x)))
        return x

    def time_apply(self, iters=10) -> float:
        ms = C.c_double()
        self.ctx.check(N.load().jfg_schwarz_time(self._h, iters, C.byref(ms)))
        return ms.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_schwarz_free(self._h)
        except Exception:
            pass


def cartesian_cell_patches(cx: int, cy: int, partitions, overlap: int):
    """Cell blocks of CartesianUpFrontSchwarz (CartesianUpFrontSchwarz.java:37-96).
    partitions = (px, py): px * py blocks of cells extended by `overlap` cells
    (clipped), in IntCoordinates.range order (last index fastest).
    partitions = (-1, ...): one patch per interior vertex, the 2*overlap x
    2*overlap cells around it.  Returns lists of (ix, iy) cell coordinates."""
    px, py = partitions
    out = []
    if px != -1:
        if cx % px or cy % py:
            raise IllegalArgumentException("partitions do not divide the cells")
        wx, wy = cx // px, cy // py
        for a in range(px):
            for b in range(py):
                xs = range(max(a * wx - overlap, 0), min(a * wx + wx + overlap, cx))
                ys = range(max(b * wy - overlap, 0), min(b * wy + wy + overlap, cy))
                out.append([(i, j) for i in xs for j in ys])
    else:
        for a in range(cx - 1):
            for b in range(cy - 1):
                ux, uy = a + 1, b + 1
                xs = range(max(ux - overlap, 0), min(ux + overlap, cx))
                ys = range(max(uy - overlap, 0), min(uy + overlap, cy))
                out.append([(i, j) for i in xs for j in ys])
    return out


def nine_colours(partitions):
    """ColoredCartesianSchwarz.getColors (ColoredCartesianSchwarz.java:82-127):
    colour 3 * (a % 3) + (b % 3) for partition (a, b)."""
    px, py = partitions
    cols = [[] for _ in range(9)]
    k = 0
    for a in range(px):
        for b in range(py):
            cols[3 * (a % 3) + (b % 3)].append(k)
            k += 1
    return cols


def _patch_dofs(cell_dofs_of, cy, cells):
    return np.unique(np.concatenate([cell_dofs_of(i * cy + j) for (i, j) in cells]))


def cartesian_patch_dofs(space, partitions, overlap):
    """(cell patches, DOF patches) of CartesianUpFrontSchwarz / ColoredCartesianSchwarz:
    the DOFs of a patch are the shape functions with support on its cells
    (buildRestrictionMatrix), ascending."""
    cx, cy, cd = _space_cells(space)
    cells = cartesian_cell_patches(cx, cy, partitions, overlap)
    return cells, [_patch_dofs(lambda c: cd[c], cy, cl) for cl in cells]


class CartesianUpFrontSchwarz(UpFrontSchwarz):
    """schwarz/CartesianUpFrontSchwarz.java.  ``space`` is any space with
    cx, cy and a ``cell_dofs`` table (Space, or a mixed space restricted to
    the fields a patch should cover)."""

    def __init__(self, globalMatrix, space, partitions, overlap, subspaceCorrection, solver=None):
        self.cellPatches, patches = cartesian_patch_dofs(space, partitions, overlap)
        super().__init__(globalMatrix, patches, subspaceCorrection, solver)

    def getCellPatch(self, patch):
        return self.cellPatches[patch]


class ColoredCartesianSchwarz(UpFrontSchwarz):
    """schwarz/ColoredCartesianSchwarz.java: partition blocks with overlap,
    nine colours, coloured multiplicative correction with damping omega."""

    def __init__(self, globalMatrix, space, partitions, overlap, solver=None, omega=1.0):
        cx, cy, _ = _space_cells(space)
        px, py = partitions
        if cx % px or cy % py:
            raise IllegalArgumentException("partitions do not divide the cells")
        if overlap >= cx // px or overlap >= cy // py:
            raise IllegalArgumentException("Too Much Overlap, can't color.")
        self.cellPatches, patches = cartesian_patch_dofs(space, partitions, overlap)
        super().__init__(globalMatrix, patches, ColoredMultiplicativeSubspaceCorrection(omega), solver,
                         colours=nine_colours(partitions))

    def getCellPatch(self, patch):
        return self.cellPatches[patch]


class VankaSchwarz(UpFrontSchwarz):
    """schwarz/VankaSchwarz.java: one patch per pressure DOF p -- the velocity
    DOFs with an entry in column p of the global matrix, plus p itself."""

    def __init__(self, globalMatrix, velocity_size: int, subspaceCorrection, solver=None, coo=None):
        if coo is None:
            raise IllegalArgumentException("VankaSchwarz needs the matrix pattern (rows, cols)")
        rows, cols = np.asarray(coo[0]), np.asarray(coo[1])
        n = _as_device(globalMatrix).rows
        sel = (cols >= velocity_size) & (rows < velocity_size)
        order = np.lexsort((rows[sel], cols[sel]))
        pc, pr = cols[sel][order], rows[sel][order]
        patches = []
        starts = np.searchsorted(pc, np.arange(velocity_size, n + 1))
        for k, p in enumerate(range(velocity_size, n)):
            vel = np.unique(pr[starts[k]:starts[k + 1]])
            patches.append(np.concatenate([vel, [p]]))
        super().__init__(globalMatrix, patches, subspaceCorrection, solver)


class SchwarzSmoother:
    """schwarz/SchwarzSmoother.java: runs x SubspaceCorrection.apply."""

    def __init__(self, runs: int, schwarz: UpFrontSchwarz):
        self.runs = int(runs)
        self.schwarz = schwarz

    def desc(self):
        return N.SmootherDesc(N.SMOOTH_SCHWARZ, self.runs, 1.0, self.schwarz.handle)

    def smooth(self, operator, rhs, iterate, verbose=False, prefix=""):
        x = N.f64(iterate).copy()
        s = self.schwarz
        s.ctx.check(N.load().jfg_schwarz_smooth(s.handle, self.runs, N.dptr(N.f64(rhs)), N.dptr(x)))
        if verbose:
            print(prefix, np.linalg.norm(s.A.spmv(x) - rhs))
        return x
