"""Raviart-Thomas mixed Darcy systems (a producer of saddle-point systems).

The reference assembles its mixed Darcy problem with ``MixedRTSpace``
(mixed/MixedRTSpace.java:24-70: pressure functions per cell, RT velocity
functions per cell, one global index each), the cell integrals
VALUE_VALUE on the velocity (TPVectorCellIntegral) and DIV_VALUE between
velocity and pressure (mixed/MixedTPCellIntegral.java:45-54:
integral of div(v) q), a constant pressure source f = -1
(MixedRightHandSideIntegral.fromPressureIntegral) and a zero normal
boundary value (NORMAL_VALUE boundary face integral, i.e. the natural
pressure condition p = 0), and solves it with unpreconditioned GMRES
(Examples/src/RTDarcy.java:20-78).

This module restates that system for the lowest-order space (RT0 velocity:
one normal-component unknown per cell edge; piecewise-constant pressure) on a
uniform cx x cy grid of [x0, x1] x [y0, y1], with the integrals evaluated
exactly:

    [ M   B^T ] [u]   [0]
    [ B   0   ] [p] = [f]

M_ij = int phi_i . phi_j, B_qi = int_cell q div(phi_i), f_q = int_cell -1 q.
Unknowns: the x-normal edges (cx + 1) * cy (index i * cy + j for the edge at
x_i in row j), then the y-normal edges cx * (cy + 1) (index i * (cy + 1) + j),
then the cell pressures cx * cy (index i * cy + j).  The basis function of an
edge has normal component 1 on that edge and 0 on the other edges, linear in
the normal direction: on a cell of size hx x hy the x-edge functions are
((x - x_{i-1}) / hx, 0) and ((x_{i+1} - x) / hx, 0), so
int phi phi = hx hy / 3 on the diagonal and hx hy / 6 between the two x-edges
of a cell, and div phi = +-1 / hx.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class DarcySystem:
    n: int
    nv: int               # velocity unknowns (edges)
    np_: int              # pressure unknowns (cells)
    rows: np.ndarray      # COO, duplicates kept (one triple per cell contribution)
    cols: np.ndarray
    vals: np.ndarray
    rhs: np.ndarray
    cx: int
    cy: int


def rt0_darcy(cx: int, cy: int, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, source=-1.0) -> DarcySystem:
    hx, hy = (x1 - x0) / cx, (y1 - y0) / cy
    nxe = (cx + 1) * cy
    nye = cx * (cy + 1)
    nv = nxe + nye
    npr = cx * cy
    ci, cj = np.meshgrid(np.arange(cx), np.arange(cy), indexing="ij")
    ci, cj = ci.ravel(), cj.ravel()
    # the four edges of every cell: x-edges left/right, y-edges bottom/top
    xl = ci * cy + cj
    xr = (ci + 1) * cy + cj
    yb = nxe + ci * (cy + 1) + cj
    yt = nxe + ci * (cy + 1) + cj + 1
    p = nv + ci * cy + cj
    area = hx * hy
    R, C, V = [], [], []

    def add(r, c, v):
        R.append(r)
        C.append(c)
        V.append(np.broadcast_to(np.asarray(v, dtype=np.float64), r.shape).copy())

    # VALUE_VALUE on the velocity: per cell 2 x 2 blocks for the x- and the y-edges
    for a, b in ((xl, xr), (yb, yt)):
        add(a, a, area / 3)
        add(b, b, area / 3)
        add(a, b, area / 6)
        add(b, a, area / 6)
    # DIV_VALUE: div of the left / bottom function is -1/h, of the right / top one +1/h (normal component 1
    # in the +x / +y direction on its edge); the integral over the cell times the constant pressure function
    for e, s in ((xl, -hy), (xr, hy), (yb, -hx), (yt, hx)):
        add(e, p, s)       # velocity row, pressure column
        add(p, e, s)       # pressure row, velocity column
    rows = np.concatenate(R).astype(np.int32)
    cols = np.concatenate(C).astype(np.int32)
    vals = np.concatenate(V)
    rhs = np.zeros(nv + npr)
    rhs[nv:] = source * area
    return DarcySystem(nv + npr, nv, npr, rows, cols, vals, rhs, cx, cy)
