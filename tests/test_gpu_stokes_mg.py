"""Monolithic multigrid on the whole Taylor-Hood system with coloured
Cartesian Schwarz smoothing, the reference's Examples/src/StokesMGSchwarz.java
driver (levels 4·2^l cells, pinned first pressure unknown, Schwarz partitions
2·2^(l-1) per direction with overlap 2, SchwarzSmoother(2, ...), omega 1,
FMG + 3 V-cycles per application, PGMRES to 1e-8), on the GPU against the
oracle's MG with the oracle's Schwarz smoothers on the same patches."""
import numpy as np
import pytest

import oracle as O
from jfem_b200 import _native as N
from jfem_b200.stokes import MonolithicStokesMG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mono(ctx):
    return MonolithicStokesMG(ctx, cells=16, coarse_cells=4, seed=3)


@pytest.fixture(scope="module")
def oracle_mg(mono):
    L = len(mono.spaces)
    mats = [O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals) for s in mono.systems]
    prol = [O.CooMatrix(mono.spaces[l + 1].n, mono.spaces[l].n, *mono.prolong[l]) for l in range(L - 1)]
    mg = O.MGPreconditioner(mats, prol, mono.boundary, [None] + [(O.SMOOTH_JACOBI, 1, 1.0)] * (L - 1), cycles=3,
                            use_fmg=True)
    keep = []
    for l in range(1, L):
        sw = mono.schwarz[l - 1]
        So = O.Schwarz(mats[l], O.SCHWARZ_COLORED, sw.patches, 1.0, colours=sw.colours)
        keep.append(So)
        mg.set_schwarz(l, So, 2)
    return mats, mg, keep


def test_patches_cover_velocity_and_pressure(mono):
    th = mono.spaces[-1]
    sw = mono.schwarz[-1]
    # 4 partitions per direction, 4 cells each, overlap 2: interior patches of 8 x 8 cells
    sizes = [len(p) for p in sw.patches]
    assert len(sizes) == 16
    assert max(sizes) == 2 * 17 * 17 + 9 * 9
    for p in sw.patches:
        assert np.any(p >= th.nv) and np.any(p < th.nv)
    assert sw.info()["max_patch"] == max(sizes)


def test_preconditioner_matches_oracle(mono, oracle_mg):
    _, mg_o, _ = oracle_mg
    v = np.random.default_rng(4).standard_normal(mono.A.rows)
    got = mono.mg.mvMul(v)
    ref = mg_o.mvmul(v)
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


def test_pgmres_matches_oracle(mono, oracle_mg):
    mats, mg_o, _ = oracle_mg
    b = mono.rhs
    tol = 1e-8 * np.linalg.norm(b)
    ref = O.solve_gmres(mats[-1], b, tol, M=mg_o, restart=50)
    x, it = mono.solve(tol, restart=50)
    assert ref.status == O.OK and it.last.status == N.OK
    assert abs(it.iterations - ref.iterations) <= 1
    np.testing.assert_allclose(it.last.history[:ref.iterations], ref.history[:ref.iterations], rtol=1e-5)
    np.testing.assert_allclose(x, ref.x, rtol=1e-6, atol=1e-7 * np.abs(ref.x).max())
    # left preconditioning: the tolerance applies to the preconditioned residual
    assert np.linalg.norm(b - mats[-1].mvmul(x)) <= 1e-6 * np.linalg.norm(b)
