"""GPU Schwarz decompositions against the Schwarz oracle (patch inverses,
the three subspace corrections, smoothing, multigrid with a Schwarz
smoother, Schwarz-preconditioned Krylov solves)."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, mg_levels, schwarz_test_matrix
from jfem_b200 import IterativeSolver, JacobiSmoother, MGPreconditioner
from jfem_b200 import _native as N
from jfem_b200.assembly import Space
from jfem_b200.linalg import DeviceMatrix
from jfem_b200.schwarz import (AdditiveSubspaceCorrection, CartesianUpFrontSchwarz, ColoredCartesianSchwarz,
                               ColoredMultiplicativeSubspaceCorrection, DirectSolver,
                               MultiplicativeSubspaceCorrection, SchwarzSmoother, UpFrontSchwarz, VankaSchwarz,
                               cartesian_patch_dofs, nine_colours)

pytestmark = pytest.mark.gpu


def dev(sy, ctx):
    return DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)


def close(a, b, rtol=1e-11):
    np.testing.assert_allclose(a, b, rtol=rtol, atol=rtol * max(np.abs(b).max(), 1e-300))


def test_projection_with_gpu_inverses(ctx):
    """CartesianSchwarzTest.testSchwarzProjection with the GPU patch inverses."""
    sp = Space(1, 2, 2)
    a = schwarz_test_matrix(sp.n)
    r, c = np.nonzero(a)
    A = DeviceMatrix(sp.n, sp.n, r, c, a[r, c], ctx)
    S = CartesianUpFrontSchwarz(A, sp, (2, 2), 0, AdditiveSubspaceCorrection(1), DirectSolver())
    assert S.getPatchCount() == 4
    for i in range(S.getPatchCount()):
        d = S.getPatchDoFs(i)
        R = np.zeros((d.size, sp.n))
        R[np.arange(d.size), d] = 1.0
        P = R.T @ S.localInverse(i) @ R @ a
        assert np.abs(P @ P - P).max() < 1e-13
        assert np.abs(P.T @ a - a @ P).max() < 1e-12


@pytest.mark.parametrize("p,cells,parts,overlap", [(1, 12, (6, 6), 1), (2, 8, (4, 4), 1), (2, 6, (2, 2), 0)])
def test_patch_inverses_match_oracle(ctx, p, cells, parts, overlap):
    sp, sy = fe_system(p, cells)
    _, patches = cartesian_patch_dofs(sp, parts, overlap)
    S = UpFrontSchwarz(dev(sy, ctx), patches, AdditiveSubspaceCorrection(0.2))
    So = O.Schwarz(coo_oracle(sy), O.SCHWARZ_ADDITIVE, patches, 0.2)
    for i in range(len(patches)):
        close(S.localInverse(i), So.inverse(i), 1e-11)


def test_large_patch_global_memory_inverse(ctx):
    """Patches above the shared-memory size take the global-memory path (Q2, 3 x 3 cells + overlap)."""
    sp, sy = fe_system(2, 12)
    _, patches = cartesian_patch_dofs(sp, (4, 4), 2)
    S = UpFrontSchwarz(dev(sy, ctx), patches, AdditiveSubspaceCorrection(0.1))
    assert S.info()["max_patch"] > 168
    So = O.Schwarz(coo_oracle(sy), O.SCHWARZ_ADDITIVE, patches, 0.1)
    b = sy.rhs
    x0 = np.random.default_rng(3).standard_normal(sy.n)
    close(S.apply(x0, b), So.apply(x0, b), 1e-10)


def _kinds(sp, sy, ctx, parts, overlap):
    _, patches = cartesian_patch_dofs(sp, parts, overlap)
    cols = nine_colours(parts)
    A, Ao = dev(sy, ctx), coo_oracle(sy)
    return [
        (UpFrontSchwarz(A, patches, MultiplicativeSubspaceCorrection()),
         O.Schwarz(Ao, O.SCHWARZ_MULTIPLICATIVE, patches, 1.0)),
        (UpFrontSchwarz(A, patches, ColoredMultiplicativeSubspaceCorrection(0.8), colours=cols),
         O.Schwarz(Ao, O.SCHWARZ_COLORED, patches, 0.8, colours=cols)),
        (UpFrontSchwarz(A, patches, AdditiveSubspaceCorrection(0.2)),
         O.Schwarz(Ao, O.SCHWARZ_ADDITIVE, patches, 0.2)),
    ]


@pytest.mark.parametrize("p,cells,parts,overlap", [(1, 12, (6, 6), 1), (2, 9, (3, 3), 1), (1, 9, (9, 9), 0)])
def test_corrections_match_oracle(ctx, p, cells, parts, overlap):
    sp, sy = fe_system(p, cells)
    rng = np.random.default_rng(7)
    x0 = rng.standard_normal(sy.n)
    b = sy.rhs
    for S, So in _kinds(sp, sy, ctx, parts, overlap):
        close(S.apply(x0, b), So.apply(x0, b))
        close(S.mvMul(b), So.solve(b))
        sm = SchwarzSmoother(3, S)
        close(sm.smooth(S.A, b, x0), So.smooth(3, b, x0), 1e-10)


def test_colour_independence_detected(ctx):
    """2 x 2-cell partitions with overlap 1: same-colour patches are two cells
    apart, so every colour runs as one fused launch; all patches in one colour
    (overlapping) take the two-kernel path and still match the oracle."""
    sp, sy = fe_system(1, 12)
    _, patches = cartesian_patch_dofs(sp, (6, 6), 1)
    S = UpFrontSchwarz(dev(sy, ctx), patches, ColoredMultiplicativeSubspaceCorrection(1.0),
                       colours=nine_colours((6, 6)))
    assert S.info()["independent_colours"] == 9
    one = [list(range(len(patches)))]
    S1 = UpFrontSchwarz(dev(sy, ctx), patches, ColoredMultiplicativeSubspaceCorrection(0.25), colours=one)
    assert S1.info()["independent_colours"] == 0
    So = O.Schwarz(coo_oracle(sy), O.SCHWARZ_COLORED, patches, 0.25, colours=one)
    x0 = np.random.default_rng(2).standard_normal(sy.n)
    close(S1.apply(x0, sy.rhs), So.apply(x0, sy.rhs))


def test_colored_cartesian_builder(ctx):
    sp, sy = fe_system(2, 8)
    S = ColoredCartesianSchwarz(dev(sy, ctx), sp, (4, 4), 1, DirectSolver(), 1.0)
    So = O.Schwarz(coo_oracle(sy), O.SCHWARZ_COLORED, S.patches, 1.0, colours=nine_colours((4, 4)))
    x0 = np.zeros(sy.n)
    close(S.apply(x0, sy.rhs), So.apply(x0, sy.rhs))
    with pytest.raises(Exception):
        ColoredCartesianSchwarz(dev(sy, ctx), sp, (4, 4), 2, DirectSolver(), 1.0)     # overlap >= cells per partition


def test_vanka_patches(ctx):
    """VankaSchwarz on a saddle-point matrix [[K, B^T], [B, 0]]: one patch per
    'pressure' unknown with the velocity unknowns of its column."""
    sp, sy = fe_system(1, 6)
    nv = sy.n
    rng = np.random.default_rng(1)
    npres = 9
    B = (rng.random((npres, nv)) < 0.08) * rng.standard_normal((npres, nv))
    K = coo_oracle(sy).dense()
    M = np.block([[K, B.T], [B, -1e-2 * np.eye(npres)]])
    r, c = np.nonzero(M)
    A = DeviceMatrix(M.shape[0], M.shape[0], r, c, M[r, c], ctx)
    S = VankaSchwarz(A, nv, MultiplicativeSubspaceCorrection(), DirectSolver(), coo=(r, c))
    assert S.getPatchCount() == npres
    for k in range(npres):
        d = S.getPatchDoFs(k)
        assert d[-1] == nv + k
        assert set(d[:-1]) == set(np.nonzero(B[k])[0])
    Ao = O.CooMatrix(M.shape[0], M.shape[0], r.astype(np.int32), c.astype(np.int32), M[r, c])
    So = O.Schwarz(Ao, O.SCHWARZ_MULTIPLICATIVE, S.patches, 1.0)
    b = rng.standard_normal(M.shape[0])
    close(S.apply(np.zeros_like(b), b), So.apply(np.zeros_like(b), b), 1e-10)


def test_mg_with_schwarz_smoother(ctx):
    """A V-cycle with coloured Schwarz smoothing on every level above the
    coarsest against the oracle's V-cycle with the same smoothers."""
    L = 4
    h = mg_levels(2, 2, L, mass=5.0)
    mats = [dev(s, ctx) for s in h.systems]
    mats_o = [coo_oracle(s) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
    sms, keep = [None], []
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [(O.SMOOTH_JACOBI, 1, 0.5)] * (L - 1), cycles=1,
                              use_fmg=False)
    for l in range(1, L):
        cells = h.spaces[l].cx
        parts = (cells // 2, cells // 2)
        S = ColoredCartesianSchwarz(mats[l], h.spaces[l], parts, 1, DirectSolver(), 1.0)
        So = O.Schwarz(mats_o[l], O.SCHWARZ_COLORED, S.patches, 1.0, colours=nine_colours(parts))
        keep.append(So)
        mg_o.set_schwarz(l, So, 1)
        sms.append(SchwarzSmoother(1, S))
    mg = MGPreconditioner(mats, prol, h.boundary, sms, cycles=1, use_fmg=False, ctx=ctx)
    b = h.finest.rhs
    x0 = np.zeros(b.size)
    close(mg.vCycle(x0, b), mg_o.vcycle(x0, b), 1e-10)
    s = IterativeSolver(ctx=ctx)
    tol = 1e-10 * np.linalg.norm(b)
    x = s.solvePCG(mats[-1], mg, b, tol)
    assert s.last.status == N.OK and s.iterations < 15
    assert np.linalg.norm(b - mats_o[-1].mvmul(x)) <= tol * 1.0001


def test_schwarz_preconditioned_krylov(ctx):
    sp, sy = fe_system(1, 32, mass=0.0)
    _, patches = cartesian_patch_dofs(sp, (16, 16), 1)
    S = UpFrontSchwarz(dev(sy, ctx), patches, AdditiveSubspaceCorrection(0.25))
    A = dev(sy, ctx)
    b = np.random.default_rng(4).standard_normal(sy.n)     # all modes, so that CG is slow
    b[sy.boundary] = 0.0
    tol = 1e-9 * np.linalg.norm(b)
    s = IterativeSolver(ctx=ctx)
    x = s.solvePCG(A, S, b, tol)
    it_pcg = s.iterations
    s2 = IterativeSolver(ctx=ctx)
    s2.solveCG(A, b, tol)
    assert s.last.status == N.OK and it_pcg < s2.iterations
    assert np.linalg.norm(b - coo_oracle(sy).mvmul(x)) <= tol * 1.0001
    Sc = UpFrontSchwarz(A, patches, ColoredMultiplicativeSubspaceCorrection(1.0), colours=nine_colours((16, 16)))
    s3 = IterativeSolver(ctx=ctx)
    x3 = s3.solvePGMRES(A, Sc, b, tol)
    assert s3.last.status == N.OK
    # left preconditioning: the tolerance applies to the preconditioned residual
    assert np.linalg.norm(b - coo_oracle(sy).mvmul(x3)) <= 1e-6 * np.linalg.norm(b)


def test_shared_inverses_for_identical_patches(ctx, monkeypatch):
    """Interior patches of a uniform grid have identical local operators and
    share one inverse; the result is bit-identical to one inverse per patch."""
    sp, sy = fe_system(2, 16)
    _, patches = cartesian_patch_dofs(sp, (8, 8), 1)
    cols = nine_colours((8, 8))
    S1 = UpFrontSchwarz(dev(sy, ctx), patches, ColoredMultiplicativeSubspaceCorrection(1.0), colours=cols)
    monkeypatch.setenv("JFEM_SCHWARZ_DEDUP", "0")
    S2 = UpFrontSchwarz(dev(sy, ctx), patches, ColoredMultiplicativeSubspaceCorrection(1.0), colours=cols)
    e1, e2 = S1.info()["inverse_entries"], S2.info()["inverse_entries"]
    assert e1 < e2 / 4
    x0 = np.random.default_rng(9).standard_normal(sy.n)
    assert np.array_equal(S1.apply(x0, sy.rhs), S2.apply(x0, sy.rhs))
    for i in (0, 9, 27, 63):
        assert np.array_equal(S1.localInverse(i), S2.localInverse(i))


