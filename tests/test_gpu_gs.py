"""Gauss-Seidel family smoothers on the GPU (ForwardBackwardGaussSeidelSmoother,
GaussSeidelSmoother) in the natural and multicolour orderings, standalone and
as multigrid smoothers, against the oracle."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, mg_levels
from jfem_b200 import (ForwardBackwardGaussSeidelSmoother, GaussSeidelSmoother, JacobiSmoother, MGPreconditioner,
                       SingularMatrixException)
from jfem_b200 import _native as N
from jfem_b200.linalg import DeviceMatrix, IterativeSolver

pytestmark = pytest.mark.gpu

KINDS = [(ForwardBackwardGaussSeidelSmoother, O.SMOOTH_FBGS), (GaussSeidelSmoother, O.SMOOTH_GS)]


def dev(sy, ctx):
    return DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)


def close(got, ref, tol=1e-12):
    np.testing.assert_allclose(got, ref, rtol=tol, atol=tol * np.abs(ref).max())


@pytest.mark.parametrize("cls,kind", KINDS)
@pytest.mark.parametrize("ordering", ["natural", "multicolour"])
@pytest.mark.parametrize("p,cells", [(1, 16), (2, 8), (1, 128)])
def test_smoother_matches_oracle(ctx, cls, kind, ordering, p, cells):
    sp, sy = fe_system(p, cells)
    A = dev(sy, ctx)
    sm = cls(3, A, ordering)
    x0 = np.random.default_rng(1).standard_normal(sy.n)
    got = sm.smooth(A, sy.rhs, x0)
    rank = None if ordering == "natural" else sm.ranks()
    ref = O.gs_smooth(coo_oracle(sy), kind, 3, sy.rhs, x0, rank)
    close(got, ref)


def test_schedules(ctx):
    """Natural order: levels follow the dependency chains; multicolour: at
    most one level per colour, ranks a permutation."""
    sp, sy = fe_system(1, 32)
    A = dev(sy, ctx)
    nat = ForwardBackwardGaussSeidelSmoother(1, A)
    f, b, c = nat.info()
    assert c == 0 and f > 32 and b > 32
    assert np.array_equal(nat.ranks(), np.arange(sy.n))
    mc = ForwardBackwardGaussSeidelSmoother(1, A, "multicolour")
    f, b, c = mc.info()
    assert 2 <= c <= 9 and f <= c and b <= c
    rank = mc.ranks()
    assert np.array_equal(np.sort(rank), np.arange(sy.n))


def test_singular_diagonal(ctx):
    A = DeviceMatrix(3, 3, [0, 1, 2, 1], [0, 1, 2, 0], [1.0, 0.0, 2.0, 1.0], ctx)
    with pytest.raises(SingularMatrixException):
        ForwardBackwardGaussSeidelSmoother(1, A)


def build_mg(h, ctx, make):
    mats = [dev(s, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(len(mats) - 1)]
    sms = [None] + [make(mats[l]) for l in range(1, len(mats))]
    return mats, prol, sms


@pytest.mark.parametrize("cls,kind", KINDS)
def test_vcycle_matches_oracle(ctx, cls, kind):
    h = mg_levels(1, 4, 5, modes=6, seed=4)
    mats, prol, sms = build_mg(h, ctx, lambda A: cls(1, A))
    mg = MGPreconditioner(mats, prol, h.boundary, sms, cycles=1, use_fmg=False, ctx=ctx)
    mats_o = [coo_oracle(s) for s in h.systems]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(len(mats_o) - 1)]
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [(kind, 1, 1.0)] * (len(mats_o) - 1), cycles=1,
                              use_fmg=False)
    b = h.finest.rhs
    x0 = np.random.default_rng(2).standard_normal(b.size) * 0.1
    close(mg.vCycle(x0, b), mg_o.vcycle(x0, b), 1e-10)
    close(mg.mvMul(b), mg_o.mvmul(b), 1e-10)


@pytest.mark.parametrize("ordering", ["natural", "multicolour"])
@pytest.mark.parametrize("precision", ["fp64", "mixed-precond"])
def test_pcg_with_gs_multigrid(ctx, ordering, precision):
    """GMG-PCG with FBGS(1) smoothing converges to the FP64 true residual in
    no more iterations than with Jacobi 2 + 2, FP64 and FP32 V-cycles."""
    h = mg_levels(2, 4, 6, modes=8, seed=1)
    mats, prol, sms = build_mg(h, ctx, lambda A: ForwardBackwardGaussSeidelSmoother(1, A, ordering))
    hp = "mixed" if precision != "fp64" else "fp64"
    mg = MGPreconditioner(mats, prol, h.boundary, sms, cycles=1, use_fmg=False, precision=hp, ctx=ctx)
    mgj = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (len(mats) - 1), cycles=1,
                           use_fmg=False, precision=hp, ctx=ctx)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    its = []
    for m in (mg, mgj):
        s = IterativeSolver(ctx=ctx)
        s.precision = precision
        x = s.solvePCG(mats[-1], m, b, tol)
        assert s.last.status == N.OK
        assert np.linalg.norm(b - mats[-1].spmv(x)) <= tol
        its.append(s.iterations)
    assert its[0] <= its[1]
