"""Seeded synthetic systems of the benchmark configurations.

* ``poisson``: -Laplace u + c u = f on the unit square, zero Dirichlet data,
  Q_p elements (ContinuousTPFESpace), f = sum_{k,l=1..K} a_kl sin(k pi x)
  sin(l pi y) with a_kl ~ N(0, 1) from a seeded numpy Philox stream;
  GRAD_GRAD + c VALUE_VALUE.  Q1 64x64 with K=4 is the small CG case, Q2
  512x512 with K=16 the multigrid-PCG case.
* ``hierarchy``: the nested spaces, per-level systems, prolongations and
  Dirichlet lists of a geometric multigrid hierarchy (what
  MGPreconditionerSpace builds, multigrid/MGPreconditionerSpace.java:28-57).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .assembly import Space, System, assemble, prolongation


def modes_source(K: int, seed: int):
    rng = np.random.Generator(np.random.Philox(seed))
    a = rng.standard_normal((K, K))
    k = np.arange(1, K + 1)

    def f(X, Y):
        sx = np.sin(np.pi * X[..., None] * k)           # (..., K)
        sy = np.sin(np.pi * Y[..., None] * k)
        return np.einsum("...k,kl,...l->...", sx, a, sy)

    return f, a


def poisson(p: int, cells: int, mass: float = 5.0, modes: int = 4, seed: int = 0) -> tuple[Space, System]:
    sp = Space(p, cells, cells)
    f, _ = modes_source(modes, seed)
    return sp, assemble(sp, 1.0, mass, source=f)


@dataclass
class Hierarchy:
    spaces: list
    systems: list            # System per level (0 = coarsest)
    prolong: list            # (rows, cols, vals) per level l -> l+1
    boundary: list

    @property
    def finest(self) -> System:
        return self.systems[-1]


def hierarchy(p: int, coarse_cells: int, levels: int, mass: float = 5.0, modes: int = 4, seed: int = 0,
              grad_coef_cells=None) -> Hierarchy:
    """Levels 0..levels-1 with coarse_cells * 2^l cells per direction; the
    rhs of the finest level carries the seeded source."""
    spaces = [Space(p, coarse_cells << l, coarse_cells << l) for l in range(levels)]
    f, _ = modes_source(modes, seed)
    systems = []
    for l, sp in enumerate(spaces):
        kc = None
        if grad_coef_cells is not None:
            kc = grad_coef_cells(sp)
        systems.append(assemble(sp, 1.0, mass, source=f if l == levels - 1 else None, grad_coef_cells=kc))
    prol = [prolongation(spaces[l], spaces[l + 1]) for l in range(levels - 1)]
    return Hierarchy(spaces, systems, prol, [s.boundary for s in systems])


@dataclass
class HeatSystem:
    space: Space
    K: System        # M + dt A (COO)
    M: System        # mass matrix (COO)
    u0: np.ndarray


def heat_batch(nsys: int = 256, sizes=tuple(range(32, 257, 16)), dt: float = 1e-3, bumps: int = 8,
               seed: int = 0) -> list:
    """The batched heat workload: `nsys` Q1 systems on the unit square with
    cell grids drawn uniformly from `sizes` (square), implicit Euler
    K = M + dt A with the natural boundary condition, and u0 = a seeded sum
    of `bumps` Gaussian bumps with sigma ~ U(0.02, 0.1) (numpy Philox stream).
    """
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for s in range(nsys):
        c = int(rng.choice(np.asarray(sizes)))
        sp = Space(1, c, c)
        Mm = assemble(sp, 0.0, 1.0, dirichlet=False)
        Ka = assemble(sp, dt, 1.0, dirichlet=False)
        cx = rng.uniform(0.15, 0.85, bumps)
        cy = rng.uniform(0.15, 0.85, bumps)
        sg = rng.uniform(0.02, 0.1, bumps)
        am = rng.standard_normal(bumps)
        px, py = sp.node_points()
        u0 = np.zeros(sp.n)
        for j in range(bumps):
            u0 += am[j] * np.exp(-((px - cx[j]) ** 2 + (py - cy[j]) ** 2) / (2 * sg[j] ** 2))
        out.append(HeatSystem(sp, Ka, Mm, u0))
    return out


def grf_cells(cells: int, length: float = 0.05, variance: float = 1.0, seed: int = 0) -> np.ndarray:
    """A stationary Gaussian random field with squared-exponential covariance
    sigma^2 exp(-d^2 / (2 l^2)) sampled at the cell centres of a cells x cells
    grid on the unit square, by circulant embedding on a periodic grid of
    twice the size (exact covariance, FFT sampling, seeded Philox stream)."""
    N = 2 * cells
    h = 1.0 / cells
    idx = np.arange(N)
    d = np.minimum(idx, N - idx) * h
    cov = variance * np.exp(-(d[:, None] ** 2 + d[None, :] ** 2) / (2 * length ** 2))
    lam = np.maximum(np.fft.fft2(cov).real, 0.0)
    rng = np.random.Generator(np.random.Philox(seed))
    w = rng.standard_normal((N, N))
    g = np.fft.ifft2(np.sqrt(lam) * np.fft.fft2(w)).real
    return g[:cells, :cells]


def coarsen_cells(k: np.ndarray) -> np.ndarray:
    """Arithmetic mean over 2x2 blocks of cells."""
    return 0.25 * (k[0::2, 0::2] + k[1::2, 0::2] + k[0::2, 1::2] + k[1::2, 1::2])


def kappa_hierarchy(p: int, coarse_cells: int, levels: int, length=0.05, variance=1.0, kseed=0, modes=4,
                    fseed=0) -> tuple:
    """-div(kappa grad u) = f with kappa = exp(g), g a GRF on the finest cells;
    coarse levels rediscretise with 2x2-averaged kappa.  Returns the hierarchy
    and the finest kappa (cells x cells, index [ix, iy])."""
    fine = coarse_cells << (levels - 1)
    kf = np.exp(grf_cells(fine, length, variance, kseed))
    ks = [kf]
    for _ in range(levels - 1):
        ks.append(coarsen_cells(ks[-1]))
    ks = ks[::-1]
    spaces = [Space(p, coarse_cells << l, coarse_cells << l) for l in range(levels)]
    f, _ = modes_source(modes, fseed)
    systems = []
    for l, sp in enumerate(spaces):
        # Space orders cells with the y index fastest (ix-major)
        systems.append(assemble(sp, 1.0, 0.0, source=f if l == levels - 1 else None,
                                grad_coef_cells=ks[l].reshape(-1)))
    prol = [prolongation(spaces[l], spaces[l + 1]) for l in range(levels - 1)]
    return Hierarchy(spaces, systems, prol, [s.boundary for s in systems]), kf
