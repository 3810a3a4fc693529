"""Structured-grid finite-element assembly (the producer of the systems).

FE assembly is not part of the accelerated path: in JFEM it is done by the
Java spaces, which hand the solver a COO ``SparseMatrix`` and a ``DenseVector``
right-hand side.  This module restates that producer for uniform Cartesian
grids so that the solver sees the same kind of system the reference builds:

* ``ContinuousTPFESpace`` Q_p Lagrange spaces with equidistant nodes
  (tensorproduct/ContinuousTPFESpace.java:30-50,
  tensorproduct/LagrangeBasisFunction1D.java:14-20);
* global numbering by first appearance while looping cells (the cell loop
  runs the last coordinate fastest, linalg/IntCoordinates.java:186-263) and
  local functions x-fastest (ContinuousTPShapeFunction.decomposeIndex);
* cell integrals by a full 5x5 Gauss tensor rule
  (tensorproduct/TPCellIntegral.java:78-159, QuadratureRule1D.Gauss5), one
  COO triple per nonzero local pair (basic/MatrixFESpace.java:113-120: a zero
  integral is not added), duplicates kept;
* Dirichlet rows/columns zeroed in place and a unit diagonal appended
  (basic/AcceptsMatrixBoundaryValues.java:25-44);
* nodal prolongation between nested grids, P[f, c] = phi_c(x_f) with zero
  values omitted (multigrid/MGPreconditionerSpace.java:59-75).

``assemble`` is vectorised numpy on the host; ``assemble_device`` builds the
same system on the GPU (``jfg_assemble_tp``: numbering, cell integrals,
Dirichlet rows and the right-hand side in CUDA kernels) and leaves the matrix
on the device.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# Gauss-Legendre 5-point rule on [-1, 1] (QuadratureRule1D.Gauss5)
_S70 = np.sqrt(70.0)
_GW = np.array([(322.0 - 13 * _S70) / 900, (322.0 + 13 * _S70) / 900, 128.0 / 225,
                (322.0 + 13 * _S70) / 900, (322.0 - 13 * _S70) / 900])
_GP = np.array([-np.sqrt(5.0 + 2 * np.sqrt(10.0 / 7)) / 3, -np.sqrt(5.0 - 2 * np.sqrt(10.0 / 7)) / 3, 0.0,
                np.sqrt(5.0 - 2 * np.sqrt(10.0 / 7)) / 3, np.sqrt(5.0 + 2 * np.sqrt(10.0 / 7)) / 3])
# mapped to the reference interval [0, 1]
QUAD_T = 0.5 * (_GP + 1.0)
QUAD_W = 0.5 * _GW


def lagrange_1d(p: int, t: np.ndarray):
    """Values and derivatives of the p+1 equidistant Lagrange functions on
    [0, 1] at points t; shapes (p+1, len(t))."""
    t = np.asarray(t, dtype=np.float64)
    nodes = np.arange(p + 1) / p
    val = np.ones((p + 1, t.size))
    der = np.zeros((p + 1, t.size))
    for i in range(p + 1):
        others = [j for j in range(p + 1) if j != i]
        denom = np.prod([nodes[i] - nodes[j] for j in others])
        for j in others:
            val[i] *= (t - nodes[j])
        val[i] /= denom
        for k in others:
            term = np.ones(t.size)
            for j in others:
                if j != k:
                    term *= (t - nodes[j])
            der[i] += term
        der[i] /= denom
    return val, der


@dataclass
class Space:
    """A ContinuousTPFESpace Q_p on [x0,x1] x [y0,y1] with (cx, cy) cells."""
    p: int
    cx: int
    cy: int
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    # derived
    nx: int = field(init=False)
    ny: int = field(init=False)
    n: int = field(init=False)
    node_of_grid: np.ndarray = field(init=False, repr=False)   # (nx*ny,) grid id -> dof
    cell_dofs: np.ndarray = field(init=False, repr=False)      # (cells, (p+1)^2)

    def __post_init__(self):
        p = self.p
        self.nx, self.ny = p * self.cx + 1, p * self.cy + 1
        ix, iy = np.meshgrid(np.arange(self.cx), np.arange(self.cy), indexing="ij")
        ix, iy = ix.ravel(), iy.ravel()                     # cell order: y fastest
        loc = np.arange((p + 1) ** 2)
        lx, ly = loc % (p + 1), loc // (p + 1)              # local functions: x fastest
        gx = ix[:, None] * p + lx[None, :]
        gy = iy[:, None] * p + ly[None, :]
        gid = (gx * self.ny + gy).ravel()                   # grid id of each visit
        uniq, first = np.unique(gid, return_index=True)
        order = np.argsort(first, kind="stable")            # first-appearance order
        dof_of_uniq = np.empty(uniq.size, dtype=np.int64)
        dof_of_uniq[order] = np.arange(uniq.size)
        node_of_grid = np.empty(self.nx * self.ny, dtype=np.int64)
        node_of_grid[uniq] = dof_of_uniq
        self.node_of_grid = node_of_grid
        self.cell_dofs = node_of_grid[gid].reshape(ix.size, (p + 1) ** 2)
        self.n = int(uniq.size)

    @property
    def hx(self):
        return (self.x1 - self.x0) / self.cx

    @property
    def hy(self):
        return (self.y1 - self.y0) / self.cy

    def grid_coords(self):
        """(gx, gy) grid coordinates of every dof, indexed by dof."""
        g = np.empty(self.n, dtype=np.int64)
        g[self.node_of_grid] = np.arange(self.nx * self.ny)
        return g // self.ny, g % self.ny

    def node_points(self):
        gx, gy = self.grid_coords()
        return (self.x0 + gx * self.hx / self.p, self.y0 + gy * self.hy / self.p)

    def boundary_nodes(self):
        """Dofs whose node lies on the boundary, ascending."""
        gx, gy = self.grid_coords()
        mask = (gx == 0) | (gx == self.nx - 1) | (gy == 0) | (gy == self.ny - 1)
        return np.nonzero(mask)[0].astype(np.int32)

    def refined(self):
        return Space(self.p, 2 * self.cx, 2 * self.cy, self.x0, self.x1, self.y0, self.y1)

    def quadrature_points(self):
        """Physical quadrature points of every cell: arrays (cells, 25), x
        index slowest (the order of TPCellIntegral.integrateNonTensorProduct)."""
        ix, iy = np.meshgrid(np.arange(self.cx), np.arange(self.cy), indexing="ij")
        ix, iy = ix.ravel(), iy.ravel()
        qx = np.repeat(QUAD_T, 5)
        qy = np.tile(QUAD_T, 5)
        X = self.x0 + (ix[:, None] + qx[None, :]) * self.hx
        Y = self.y0 + (iy[:, None] + qy[None, :]) * self.hy
        return X, Y


def _ref_tables(p: int, hx: float, hy: float):
    """Per-quadrature-point products on one cell: (25, nloc, nloc) arrays for
    GRAD_GRAD and VALUE_VALUE, plus (25, nloc) basis values x quad weight."""
    v, d = lagrange_1d(p, QUAD_T)                            # (p+1, 5)
    nl = (p + 1) ** 2
    loc = np.arange(nl)
    lx, ly = loc % (p + 1), loc // (p + 1)
    qi, qj = np.repeat(np.arange(5), 5), np.tile(np.arange(5), 5)
    w = QUAD_W[qi] * QUAD_W[qj] * hx * hy                   # (25,)
    val = v[lx][:, qi] * v[ly][:, qj]                        # (nl, 25)
    gx = d[lx][:, qi] / hx * v[ly][:, qj]
    gy = v[lx][:, qi] * d[ly][:, qj] / hy
    gg = (gx[:, None, :] * gx[None, :, :] + gy[:, None, :] * gy[None, :, :]) * w  # (nl, nl, 25)
    vv = (val[:, None, :] * val[None, :, :]) * w
    return np.moveaxis(gg, 2, 0), np.moveaxis(vv, 2, 0), (val * w).T   # (25,nl,nl),(25,nl,nl),(25,nl)


@dataclass
class System:
    """An assembled system: COO triples in storage order plus rhs."""
    n: int
    rows: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    rhs: np.ndarray
    boundary: np.ndarray

    @property
    def nnz(self):
        return self.vals.size


def assemble(space: Space, grad_coef=1.0, mass_coef=0.0, source=None, boundary_value=None,
             grad_coef_cells=None, dirichlet=True) -> System:
    """GRAD_GRAD * grad_coef + VALUE_VALUE * mass_coef with a VALUE right-hand
    side ``source(x, y)`` and Dirichlet data ``boundary_value(x, y)`` (zero
    when None) on the whole boundary.

    ``grad_coef_cells`` (length = number of cells) multiplies the GRAD_GRAD
    integral cell by cell (a piecewise-constant coefficient kappa).
    ``dirichlet=False`` leaves the natural (Neumann) boundary: no row or
    column is overwritten.
    """
    p = space.p
    gg, vv, bw = _ref_tables(p, space.hx, space.hy)
    Egg = gg.sum(0)                                          # (nl, nl), constant per cell
    Evv = vv.sum(0)
    ncell = space.cx * space.cy
    nl = (p + 1) ** 2
    if grad_coef_cells is None:
        E = grad_coef * Egg + mass_coef * Evv
        Eall = np.broadcast_to(E, (ncell, nl, nl))
    else:
        kc = np.asarray(grad_coef_cells, dtype=np.float64).reshape(ncell)
        Eall = kc[:, None, None] * Egg[None] + mass_coef * Evv[None]
    dofs = space.cell_dofs
    R = np.broadcast_to(dofs[:, :, None], (ncell, nl, nl)).reshape(-1)
    Cc = np.broadcast_to(dofs[:, None, :], (ncell, nl, nl)).reshape(-1)
    V = np.ascontiguousarray(Eall).reshape(-1)
    keep = V != 0.0
    R, Cc, V = R[keep].astype(np.int32), Cc[keep].astype(np.int32), V[keep].copy()
    rhs = np.zeros(space.n)
    if source is not None:
        X, Y = space.quadrature_points()
        f = source(X, Y)                                     # (cells, 25)
        cell_rhs = f @ bw                                    # (cells, nl)
        np.add.at(rhs, dofs.reshape(-1), cell_rhs.reshape(-1))
    bd = space.boundary_nodes()
    if not dirichlet:
        return System(space.n, R, Cc, V, rhs, np.zeros(0, dtype=np.int32))
    # Dirichlet (AcceptsMatrixBoundaryValues.overWriteValue)
    is_bd = np.zeros(space.n, dtype=bool)
    is_bd[bd] = True
    if boundary_value is not None:
        px, py = space.node_points()
        g = np.zeros(space.n)
        g[bd] = boundary_value(px[bd], py[bd])
        col_bd = is_bd[Cc] & ~is_bd[R]
        np.add.at(rhs, R[col_bd], -V[col_bd] * g[Cc[col_bd]])
        rhs[bd] = g[bd]
    else:
        rhs[bd] = 0.0
    V[is_bd[R] | is_bd[Cc]] = 0.0
    R = np.concatenate([R, bd])
    Cc = np.concatenate([Cc, bd])
    V = np.concatenate([V, np.ones(bd.size)])
    return System(space.n, R, Cc, V, rhs, bd)


def prolongation_1d(p: int, c: int) -> np.ndarray:
    """Dense (p*2c+1) x (p*c+1) nodal interpolation from c to 2c cells."""
    nf, nc = 2 * p * c + 1, p * c + 1
    P = np.zeros((nf, nc))
    tf = np.arange(nf) / (2 * p * c)
    k = np.minimum((tf * c).astype(np.int64), c - 1)
    loc_t = tf * c - k
    v, _ = lagrange_1d(p, loc_t)
    for l in range(p + 1):
        P[np.arange(nf), k * p + l] += v[l]
    P[np.abs(P) < 1e-15] = 0.0
    return P


def prolongation(coarse: Space, fine: Space):
    """COO triples (rows=fine dof, cols=coarse dof, vals) of P."""
    assert fine.cx == 2 * coarse.cx and fine.cy == 2 * coarse.cy and fine.p == coarse.p
    Px = prolongation_1d(coarse.p, coarse.cx)
    Py = prolongation_1d(coarse.p, coarse.cy)
    fx, cx = np.nonzero(Px)
    fy, cy = np.nonzero(Py)
    # all combinations of the 1-D pairs (fine x, coarse x) and (fine y, coarse y)
    fxa = np.repeat(fx, fy.size)
    cxa = np.repeat(cx, fy.size)
    fya = np.tile(fy, fx.size)
    cya = np.tile(cy, fx.size)
    vals = Px[fxa, cxa] * Py[fya, cya]
    rows = fine.node_of_grid[fxa * fine.ny + fya]
    cols = coarse.node_of_grid[cxa * coarse.ny + cya]
    order = np.lexsort((cols, rows))
    return rows[order].astype(np.int32), cols[order].astype(np.int32), vals[order]


def assemble_device(space: Space, grad_coef=1.0, mass_coef=0.0, source=None, grad_coef_cells=None, dirichlet=True,
                    ctx=None):
    """``assemble`` on the GPU for zero Dirichlet data: returns (DeviceMatrix,
    rhs, boundary dofs, node_of_grid).  The source is evaluated on the host at
    the cells' Gauss points; the matrix stays on the device.  The numbering,
    the merged matrix and the rhs are those of ``assemble`` (matrix and rhs to
    rounding: the element tables and the Gauss sums are added in a different
    order)."""
    import ctypes as C

    from . import _native as N
    from .linalg import DeviceMatrix
    ctx = ctx or N.default_context()
    d = N.TPDesc(space.p, space.cx, space.cy, space.x0, space.x1, space.y0, space.y1, float(grad_coef),
                 float(mass_coef), 1 if dirichlet else 0)
    kap = None
    if grad_coef_cells is not None:
        kap = np.ascontiguousarray(grad_coef_cells, dtype=np.float64).reshape(space.cx * space.cy)
    f = None
    if source is not None:
        X, Y = space.quadrature_points()
        f = np.ascontiguousarray(source(X, Y), dtype=np.float64)
    n = space.nx * space.ny
    rhs = np.empty(n)
    nog = np.empty(n, dtype=np.int32)
    bd = np.empty(2 * (space.nx + space.ny) - 4, dtype=np.int32)
    h = C.c_void_p()
    st = N.load().jfg_assemble_tp(ctx.handle, C.byref(d), N.dptr(kap) if kap is not None else None,
                                  N.dptr(f) if f is not None else None, C.byref(h), N.dptr(rhs), N.iptr(nog),
                                  N.iptr(bd))
    ctx.check(st)
    A = DeviceMatrix._adopt(h, ctx)
    return A, rhs, (bd if dirichlet else np.zeros(0, dtype=np.int32)), nog
