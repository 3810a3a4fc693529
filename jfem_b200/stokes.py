"""Stationary Stokes with Taylor-Hood Q2/Q1 elements: the system producer
(host assembly) and the block-diagonal preconditioner of the saddle-point
solve (GPU).

Discretisation (mixed/TaylorHoodSpace.java, mixed/MixedTPCellIntegral.java,
examples StokesMG): velocity Q2 in both components, pressure Q1, on a
uniform Cartesian grid of the unit square;

    [ nu K    0     -B0^T ] [u0]   [f0]
    [  0     nu K   -B1^T ] [u1] = [f1]
    [ -B0    -B1      0   ] [p ]   [0 ]

with K the scalar Q2 GRAD_GRAD matrix and (B_c)_{q, v} = int q d(v)/dx_c
(DIV_VALUE with weight -1, written to both off-diagonal blocks).  Unknowns
are numbered as the reference's TreeSet of QkQkFunction orders them:
velocity before pressure, component 0 before component 1, and nodes by
their coordinates (x first, then y) -- grid id gx * ny + gy.  Velocity
Dirichlet data on the whole boundary (rows and columns eliminated, unit
diagonal), the first pressure unknown fixed to 0 (StokesMG's
overWriteValue(firstPressure, 0)).

The benchmark case: lid-driven cavity u = (1, 0) on the top edge y = 1
(corners included), no-slip elsewhere, body force with seeded Fourier
coefficients, solved by GMRES(50) with the preconditioner
diag(velocity GMG V-cycle with a coloured Schwarz smoother, lumped
pressure-mass inverse).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .assembly import QUAD_T, QUAD_W, lagrange_1d, prolongation_1d
from .linalg import IllegalArgumentException, _as_device


class VelocitySpace:
    """The velocity block of a Taylor-Hood space as a cell -> DOF table for
    the Schwarz patch builders (18 DOFs per cell)."""

    def __init__(self, th: "TaylorHoodSpace"):
        self.cx, self.cy = th.cx, th.cy
        self.cell_dofs = th.cell_velocity_dofs


class TaylorHoodSpace:
    def __init__(self, cx: int, cy: int):
        self.cx, self.cy = cx, cy
        self.vnx, self.vny = 2 * cx + 1, 2 * cy + 1          # Q2 node grid
        self.pnx, self.pny = cx + 1, cy + 1                  # Q1 node grid
        self.nv1 = self.vnx * self.vny
        self.nv = 2 * self.nv1
        self.np_ = self.pnx * self.pny
        self.n = self.nv + self.np_
        self.hx, self.hy = 1.0 / cx, 1.0 / cy
        ix, iy = np.meshgrid(np.arange(cx), np.arange(cy), indexing="ij")
        ix, iy = ix.ravel(), iy.ravel()                      # cell order: y fastest
        l2 = np.arange(9)
        vg = (2 * ix[:, None] + l2[None, :] % 3) * self.vny + (2 * iy[:, None] + l2[None, :] // 3)
        self.cell_vnodes = vg                                # (cells, 9) Q2 node ids, local x fastest
        l1 = np.arange(4)
        self.cell_pnodes = (ix[:, None] + l1[None, :] % 2) * self.pny + (iy[:, None] + l1[None, :] // 2)
        self.cell_velocity_dofs = np.concatenate([vg, vg + self.nv1], axis=1)
        self.velocity = VelocitySpace(self)

    def velocity_boundary(self):
        g = np.arange(self.nv1)
        gx, gy = g // self.vny, g % self.vny
        bd = np.nonzero((gx == 0) | (gx == self.vnx - 1) | (gy == 0) | (gy == self.vny - 1))[0]
        return np.concatenate([bd, bd + self.nv1]).astype(np.int32)

    def velocity_points(self):
        g = np.arange(self.nv1)
        return (g // self.vny) * self.hx / 2, (g % self.vny) * self.hy / 2

    def getVelocitySize(self):
        return self.nv


def _tables(hx, hy):
    v2, d2 = lagrange_1d(2, QUAD_T)                      # (3, 5)
    v1, _ = lagrange_1d(1, QUAD_T)                        # (2, 5)
    qi, qj = np.repeat(np.arange(5), 5), np.tile(np.arange(5), 5)
    w = QUAD_W[qi] * QUAD_W[qj] * hx * hy
    l2 = np.arange(9)
    lx, ly = l2 % 3, l2 // 3
    val2 = v2[lx][:, qi] * v2[ly][:, qj]                  # (9, 25)
    gx = d2[lx][:, qi] / hx * v2[ly][:, qj]
    gy = v2[lx][:, qi] * d2[ly][:, qj] / hy
    l1 = np.arange(4)
    val1 = v1[l1 % 2][:, qi] * v1[l1 // 2][:, qj]         # (4, 25)
    K = np.einsum("iq,jq,q->ij", gx, gx, w) + np.einsum("iq,jq,q->ij", gy, gy, w)
    B0 = np.einsum("pq,jq,q->pj", val1, gx, w)            # int q d(phi_j)/dx
    B1 = np.einsum("pq,jq,q->pj", val1, gy, w)
    Mp = np.einsum("pq,rq,q->pr", val1, val1, w)
    return K, B0, B1, Mp, val2 * w                         # val2*w: (9, 25) rhs weights


@dataclass
class StokesSystem:
    n: int
    nv: int
    rows: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    rhs: np.ndarray
    velocity_boundary: np.ndarray
    pressure_fixed: int


def fourier_force(K: int = 4, std: float = 0.1, seed: int = 0):
    """f_c(x, y) = sum_{k,l=1..K} a^c_kl sin(k pi x) sin(l pi y), a ~ N(0, std^2)."""
    rng = np.random.Generator(np.random.Philox(seed))
    a = rng.standard_normal((2, K, K)) * std
    k = np.arange(1, K + 1)

    def f(X, Y, c):
        sx = np.sin(np.pi * X[..., None] * k)
        sy = np.sin(np.pi * Y[..., None] * k)
        return np.einsum("...k,kl,...l->...", sx, a[c], sy)

    return f


def _eliminate(R, Cc, V, rhs, bd, g):
    """AcceptsMatrixBoundaryValues.overWriteValue for all bd at once."""
    n = rhs.size
    is_bd = np.zeros(n, dtype=bool)
    is_bd[bd] = True
    col_bd = is_bd[Cc] & ~is_bd[R]
    np.add.at(rhs, R[col_bd], -V[col_bd] * g[Cc[col_bd]])
    rhs[bd] = g[bd]
    V = V.copy()
    V[is_bd[R] | is_bd[Cc]] = 0.0
    return (np.concatenate([R, bd]).astype(np.int32), np.concatenate([Cc, bd]).astype(np.int32),
            np.concatenate([V, np.ones(bd.size)]), rhs)


def assemble_stokes(th: TaylorHoodSpace, nu: float = 1.0, force=None, lid: bool = True,
                    pin_pressure: bool = True) -> StokesSystem:
    """pin_pressure=False leaves the pressure determined up to a constant
    (a consistent singular system; pressure_fixed = -1)."""
    K, B0, B1, _, rw = _tables(th.hx, th.hy)
    nc = th.cx * th.cy
    vn, pn = th.cell_vnodes, th.cell_pnodes
    blocks = []

    def add(rloc, cloc, E):
        rr = np.broadcast_to(rloc[:, :, None], (nc,) + E.shape).reshape(-1)
        cc = np.broadcast_to(cloc[:, None, :], (nc,) + E.shape).reshape(-1)
        vv = np.broadcast_to(E, (nc,) + E.shape).reshape(-1)
        keep = vv != 0.0
        blocks.append((rr[keep], cc[keep], vv[keep]))

    for c in range(2):
        vd = vn + c * th.nv1
        add(vd, vd, nu * K)
        pd = pn + th.nv
        Bc = B0 if c == 0 else B1
        add(pd, vd, -Bc)            # pressure rows
        add(vd, pd, -Bc.T)          # velocity rows
    R = np.concatenate([b[0] for b in blocks]).astype(np.int32)
    Cc = np.concatenate([b[1] for b in blocks]).astype(np.int32)
    V = np.concatenate([b[2] for b in blocks])
    rhs = np.zeros(th.n)
    if force is not None:
        qi, qj = np.repeat(np.arange(5), 5), np.tile(np.arange(5), 5)
        ix, iy = np.meshgrid(np.arange(th.cx), np.arange(th.cy), indexing="ij")
        X = (ix.ravel()[:, None] + QUAD_T[qi][None, :]) * th.hx
        Y = (iy.ravel()[:, None] + QUAD_T[qj][None, :]) * th.hy
        for c in range(2):
            cell = force(X, Y, c) @ rw.T                   # (cells, 9)
            np.add.at(rhs, (vn + c * th.nv1).reshape(-1), cell.reshape(-1))
    bd = th.velocity_boundary()
    g = np.zeros(th.n)
    if lid:
        _, py = th.velocity_points()
        top = np.nonzero(np.isclose(py, 1.0))[0]
        g[top] = 1.0                                       # u0 = 1 on y = 1, u1 = 0
    # velocity Dirichlet data and the first pressure unknown fixed to zero
    fixed = np.concatenate([bd, np.array([th.nv], dtype=np.int32)]) if pin_pressure else bd
    R, Cc, V, rhs = _eliminate(R, Cc, V, rhs, fixed, g)
    return StokesSystem(th.n, th.nv, R, Cc, V, rhs, bd, th.nv if pin_pressure else -1)


def assemble_stokes_device(th: TaylorHoodSpace, nu: float = 1.0, force=None, lid: bool = True,
                           pin_pressure: bool = True, ctx=None):
    """``assemble_stokes`` on the GPU (jfg_assemble_taylor_hood): returns
    (DeviceMatrix, rhs, velocity boundary).  The force is evaluated on the
    host at the cells' Gauss points; the matrix stays on the device and
    equals the host system's merged matrix to rounding."""
    from . import _native as N
    from .linalg import DeviceMatrix
    ctx = ctx or N.default_context()
    f = None
    if force is not None:
        qi, qj = np.repeat(np.arange(5), 5), np.tile(np.arange(5), 5)
        ix, iy = np.meshgrid(np.arange(th.cx), np.arange(th.cy), indexing="ij")
        X = (ix.ravel()[:, None] + QUAD_T[qi][None, :]) * th.hx
        Y = (iy.ravel()[:, None] + QUAD_T[qj][None, :]) * th.hy
        f = np.ascontiguousarray(np.stack([force(X, Y, 0), force(X, Y, 1)]), dtype=np.float64)
    rhs = np.empty(th.n)
    bd = np.empty(2 * (2 * (th.vnx + th.vny) - 4), dtype=np.int32)
    h = C.c_void_p()
    ctx.check(N.load().jfg_assemble_taylor_hood(ctx.handle, th.cx, th.cy, float(nu),
                                                N.dptr(f) if f is not None else None, 1 if lid else 0,
                                                1 if pin_pressure else 0, C.byref(h), N.dptr(rhs), N.iptr(bd)))
    return DeviceMatrix._adopt(h, ctx), rhs, bd


def velocity_block(th: TaylorHoodSpace, nu: float = 1.0):
    """The velocity-velocity block with zero Dirichlet rows eliminated (COO)."""
    K, *_ = _tables(th.hx, th.hy)
    nc = th.cx * th.cy
    rr, cc, vv = [], [], []
    for c in range(2):
        vd = th.cell_vnodes + c * th.nv1
        rr.append(np.broadcast_to(vd[:, :, None], (nc, 9, 9)).reshape(-1))
        cc.append(np.broadcast_to(vd[:, None, :], (nc, 9, 9)).reshape(-1))
        vv.append(np.broadcast_to(nu * K, (nc, 9, 9)).reshape(-1))
    R, Cc, V = np.concatenate(rr), np.concatenate(cc), np.concatenate(vv)
    keep = V != 0
    R, Cc, V = R[keep], Cc[keep], V[keep]
    bd = th.velocity_boundary()
    R, Cc, V, _ = _eliminate(R, Cc, V, np.zeros(th.nv), bd, np.zeros(th.nv))
    return R, Cc, V, bd


def velocity_prolongation(coarse: TaylorHoodSpace, fine: TaylorHoodSpace):
    """Nodal Q2 interpolation in both components (COO rows, cols, vals)."""
    Px = prolongation_1d(2, coarse.cx)
    Py = prolongation_1d(2, coarse.cy)
    fx, cx_ = np.nonzero(Px)
    fy, cy_ = np.nonzero(Py)
    fxa, cxa = np.repeat(fx, fy.size), np.repeat(cx_, fy.size)
    fya, cya = np.tile(fy, fx.size), np.tile(cy_, fx.size)
    vals = Px[fxa, cxa] * Py[fya, cya]
    rows = fxa * fine.vny + fya
    cols = cxa * coarse.vny + cya
    R = np.concatenate([rows, rows + fine.nv1]).astype(np.int32)
    Cc = np.concatenate([cols, cols + coarse.nv1]).astype(np.int32)
    return R, Cc, np.concatenate([vals, vals])


def lumped_pressure_mass(th: TaylorHoodSpace):
    """Row sums of the Q1 pressure mass matrix."""
    *_, Mp, _ = _tables(th.hx, th.hy)
    d = np.zeros(th.np_)
    np.add.at(d, th.cell_pnodes.reshape(-1), np.broadcast_to(Mp.sum(1), th.cell_pnodes.shape).reshape(-1))
    return d


class BlockDiagonalPreconditioner:
    """z_v = V(r_v) (velocity multigrid), z_p = scale * r_p / m_p (lumped
    pressure mass), on the GPU (jfg_blockdiag).  The handle goes to the
    solvers as JFG_PREC_BLOCKDIAG."""

    def __init__(self, mg, nv: int, pressure_inverse, fp32_vcycle: bool = False):
        self.mg = mg
        self.ctx = mg.ctx
        pinv = np.ascontiguousarray(pressure_inverse, dtype=np.float64)
        h = C.c_void_p()
        st = N.load().jfg_blockdiag_create(self.ctx.handle, mg.handle, nv, pinv.size, N.dptr(pinv),
                                           1 if fp32_vcycle else 0, C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        self._h = h
        self.n = nv + pinv.size

    @property
    def handle(self):
        return self._h

    def mvMul(self, v):
        out = np.empty(self.n)
        self.ctx.check(N.load().jfg_blockdiag_apply(self._h, N.dptr(N.f64(v)), N.dptr(out)))
        return out

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_blockdiag_free(self._h)
        except Exception:
            pass


@dataclass
class StokesProblem:
    """The finest Stokes system plus what the velocity multigrid needs."""
    spaces: list                 # TaylorHoodSpace per level (0 = coarsest)
    system: StokesSystem
    velocity_blocks: list        # (rows, cols, vals) per level, zero Dirichlet rows eliminated
    velocity_boundary: list
    prolongations: list          # velocity P[l]: level l -> l + 1
    pressure_inverse: np.ndarray  # nu / lumped pressure mass, 1 on the fixed pressure unknown
    nu: float


def stokes_problem(cells: int = 256, coarse_cells: int = 4, nu: float = 1.0, seed: int = 0,
                   pin_pressure: bool = True) -> StokesProblem:
    """pin_pressure=True is the reference's system (first pressure unknown
    overwritten by 0).  Pinning one unknown turns the constant pressure into a
    near-null mode of the preconditioned operator (eigenvalue ~ h^2), which
    restarted GMRES resolves only slowly; pin_pressure=False keeps the
    consistent singular system, whose constant-pressure null space never
    enters the Krylov space, and StokesSolver.solve shifts the pressure so that
    the first unknown is 0 -- a solution of the pinned system."""
    levels = int(round(np.log2(cells // coarse_cells))) + 1
    if coarse_cells << (levels - 1) != cells:
        raise IllegalArgumentException("cells must be coarse_cells * 2^k")
    ths = [TaylorHoodSpace(coarse_cells << l, coarse_cells << l) for l in range(levels)]
    system = assemble_stokes(ths[-1], nu, fourier_force(seed=seed), pin_pressure=pin_pressure)
    vb, vbd = [], []
    for t in ths:
        R, Cc, V, bd = velocity_block(t, nu)
        vb.append((R, Cc, V))
        vbd.append(bd)
    prol = [velocity_prolongation(ths[l], ths[l + 1]) for l in range(levels - 1)]
    pinv = nu / lumped_pressure_mass(ths[-1])
    if pin_pressure:
        pinv[0] = 1.0
    return StokesProblem(ths, system, vb, vbd, prol, pinv, nu)


class StokesSolver:
    """GMRES(restart) on the Stokes system with the block-diagonal
    preconditioner: velocity V-cycle (coloured Schwarz smoother on 2 x 2-cell
    partitions with one cell of overlap, or damped Jacobi) and the lumped
    pressure-mass inverse."""

    def __init__(self, ctx, prob: StokesProblem, smoother: str = "schwarz", runs: int = 1, omega: float = 1.0,
                 fp32_vcycle: bool = False):
        from .linalg import DeviceMatrix
        from .multigrid import JacobiSmoother, MGPreconditioner
        from .schwarz import ColoredCartesianSchwarz, DirectSolver, SchwarzSmoother
        self.ctx, self.prob = ctx, prob
        s = prob.system
        self.A = DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx)
        L = len(prob.spaces)
        self.vmats = [DeviceMatrix(t.nv, t.nv, *prob.velocity_blocks[l], ctx) for l, t in enumerate(prob.spaces)]
        self.prol = [DeviceMatrix(prob.spaces[l + 1].nv, prob.spaces[l].nv, *prob.prolongations[l], ctx)
                     for l in range(L - 1)]
        sms = [None]
        self.schwarz = []
        for l in range(1, L):
            if smoother == "schwarz":
                c = prob.spaces[l].cx
                sw = ColoredCartesianSchwarz(self.vmats[l], prob.spaces[l].velocity, (c // 2, c // 2), 1,
                                             DirectSolver(), omega)
                self.schwarz.append(sw)
                sms.append(SchwarzSmoother(runs, sw))
            else:
                sms.append(JacobiSmoother(runs, omega))
        self.mg = MGPreconditioner(self.vmats, self.prol, prob.velocity_boundary, sms, cycles=1, use_fmg=False,
                                   precision="mixed" if fp32_vcycle else "fp64", ctx=ctx)
        self.P = BlockDiagonalPreconditioner(self.mg, prob.spaces[-1].nv, prob.pressure_inverse, fp32_vcycle)

    def solve(self, tol: float, restart: int = 50, max_restarts: int = 200):
        from .linalg import IterativeSolver
        it = IterativeSolver(ctx=self.ctx)
        it.gm.ITERATIONS_BEFORE_RESTART = restart
        it.gm.MAX_RESTARTS = max_restarts
        x = it.solvePGMRES(self.A, self.P, self.prob.system.rhs, tol)
        s = self.prob.system
        if s.pressure_fixed < 0:
            x[s.nv:] -= x[s.nv]          # the pinned system's pressure gauge
        return x, it


# ---------------------------------------------------------------------------
# Monolithic multigrid on the whole Taylor-Hood system (Examples/src/StokesMGSchwarz.java)
# ---------------------------------------------------------------------------
def pressure_prolongation(coarse: TaylorHoodSpace, fine: TaylorHoodSpace):
    """Nodal Q1 interpolation of the pressure (COO rows, cols, vals; pressure
    node numbering)."""
    Px = prolongation_1d(1, coarse.cx)
    Py = prolongation_1d(1, coarse.cy)
    fx, cx_ = np.nonzero(Px)
    fy, cy_ = np.nonzero(Py)
    fxa, cxa = np.repeat(fx, fy.size), np.repeat(cx_, fy.size)
    fya, cya = np.tile(fy, fx.size), np.tile(cy_, fx.size)
    return (fxa * fine.pny + fya).astype(np.int32), (cxa * coarse.pny + cya).astype(np.int32), Px[fxa, cxa] * Py[fya, cya]


def taylor_hood_prolongation(coarse: TaylorHoodSpace, fine: TaylorHoodSpace):
    """Prolongation of the whole mixed space (MGPreconditionerSpace.createProlongationMatrix
    on a TaylorHoodSpace): velocity by Q2 and pressure by Q1 nodal interpolation,
    block diagonal (pressure unknowns after the velocity ones)."""
    Rv, Cv, Vv = velocity_prolongation(coarse, fine)
    Rp, Cp, Vp = pressure_prolongation(coarse, fine)
    return (np.concatenate([Rv, Rp + fine.nv]).astype(np.int32), np.concatenate([Cv, Cp + coarse.nv]).astype(np.int32),
            np.concatenate([Vv, Vp]))


class MixedCells:
    """The cell table of a Taylor-Hood space for the Cartesian patch builders:
    cell_dofs[c] = the velocity unknowns (both components) and the pressure
    unknowns with support on cell c (getShapeFunctionsWithSupportOnCell)."""

    def __init__(self, th: TaylorHoodSpace):
        self.cx, self.cy = th.cx, th.cy
        self.cell_dofs = np.concatenate([th.cell_velocity_dofs, th.cell_pnodes + th.nv], axis=1)


def mixed_zero_boundary(th: TaylorHoodSpace) -> np.ndarray:
    """applyZeroBoundaryConditions of StokesMGSchwarz: the Dirichlet velocity
    unknowns and the first pressure unknown."""
    return np.concatenate([th.velocity_boundary(), [th.nv]]).astype(np.int32)


def schwarz_partitions(level: int) -> tuple:
    """createSmoothers of StokesMGSchwarz: 2 * 2^(level - 1) partitions per
    direction on level >= 1 (2 * max(1, 2^(level-1)))."""
    k = 2 * max(1, 2 ** (level - 1))
    return (k, k)


class MonolithicStokesMG:
    """StokesMGSchwarz: multigrid on the whole Taylor-Hood system of every
    level (velocity Dirichlet rows and the pinned first pressure unknown, as
    createSystem writes them), Taylor-Hood prolongations, and on every level
    above the coarsest a SchwarzSmoother(2, ColoredCartesianSchwarz(partitions
    2 * 2^(l-1), overlap 2, DirectSolver, omega 1)) whose patches take every
    velocity and pressure unknown with support on their cells; the
    preconditioner is the reference's MG mvMul (FMG + `cycles` V-cycles).
    solve() is PGMRES to the tolerance, as the driver solves."""

    def __init__(self, ctx, cells: int = 64, coarse_cells: int = 4, nu: float = 1.0, seed: int = 0, runs: int = 2,
                 overlap: int = 2, cycles: int = 3, use_fmg: bool = True, precision: str = "fp64"):
        from .linalg import DeviceMatrix
        from .multigrid import MGPreconditioner
        from .schwarz import ColoredCartesianSchwarz, DirectSolver, SchwarzSmoother
        levels = int(round(np.log2(cells // coarse_cells))) + 1
        if coarse_cells << (levels - 1) != cells:
            raise IllegalArgumentException("cells must be coarse_cells * 2^k")
        self.ctx = ctx
        self.spaces = [TaylorHoodSpace(coarse_cells << l, coarse_cells << l) for l in range(levels)]
        force = fourier_force(seed=seed)
        self.systems = [assemble_stokes(t, nu, force, pin_pressure=True) for t in self.spaces]
        self.prolong = [taylor_hood_prolongation(self.spaces[l], self.spaces[l + 1]) for l in range(levels - 1)]
        self.boundary = [mixed_zero_boundary(t) for t in self.spaces]
        self.mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in self.systems]
        self.prol = [DeviceMatrix(self.spaces[l + 1].n, self.spaces[l].n, *self.prolong[l], ctx)
                     for l in range(levels - 1)]
        self.schwarz, sms = [], [None]
        for l in range(1, levels):
            sw = ColoredCartesianSchwarz(self.mats[l], MixedCells(self.spaces[l]), schwarz_partitions(l), overlap,
                                         DirectSolver(), 1.0)
            self.schwarz.append(sw)
            sms.append(SchwarzSmoother(runs, sw))
        self.mg = MGPreconditioner(self.mats, self.prol, self.boundary, sms, cycles=cycles, use_fmg=use_fmg,
                                   precision=precision, ctx=ctx)
        self.A = self.mats[-1]
        self.rhs = self.systems[-1].rhs

    def solve(self, tol: float, restart: int = 50, max_restarts: int = 200):
        from .linalg import IterativeSolver
        it = IterativeSolver(ctx=self.ctx)
        it.gm.ITERATIONS_BEFORE_RESTART = restart
        it.gm.MAX_RESTARTS = max_restarts
        x = it.solvePGMRES(self.A, self.mg, self.rhs, tol)
        return x, it
