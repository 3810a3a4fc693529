"""Batched implicit-Euler heat stepping in one persistent launch, against the
oracle's per-step FP64 CG (HeatEquation.java:81-94 for every system)."""
import numpy as np
import pytest

import oracle as O
from jfem_b200 import problems
from jfem_b200.batch import BatchedParabolicIntegrator
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu


def build(ctx, batch):
    K = [DeviceMatrix(s.K.n, s.K.n, s.K.rows, s.K.cols, s.K.vals, ctx) for s in batch]
    M = [DeviceMatrix(s.M.n, s.M.n, s.M.rows, s.M.cols, s.M.vals, ctx) for s in batch]
    return BatchedParabolicIntegrator(K, M, ctx)


def oracle_steps(s, steps):
    K = O.CooMatrix(s.K.n, s.K.n, s.K.rows, s.K.cols, s.K.vals)
    M = O.CooMatrix(s.M.n, s.M.n, s.M.rows, s.M.cols, s.M.vals)
    u = s.u0.copy()
    for _ in range(steps):
        rhs = M.mvmul(u)
        r = O.solve_cg(K, rhs, 1e-13 * np.linalg.norm(rhs), x0=u)
        u = r.x
    return u


@pytest.mark.parametrize("cluster,threads,rows", [(1, 256, 2), (2, 512, 3), (4, 256, 4), (8, 512, 3)])
def test_batch_matches_oracle(ctx, cluster, threads, rows):
    batch = problems.heat_batch(nsys=7, sizes=(4, 8, 12, 16, 24), dt=1e-3, seed=5)
    B = build(ctx, batch)
    steps = 4
    u = B.timeSteps([s.u0 for s in batch], steps, cluster=cluster, threads=threads, rows_per_thread=rows)
    assert B.last.status == 0 and B.last.failed == 0
    assert B.last.max_rel_residual <= 1e-10
    assert (B.last.cluster, B.last.threads, B.last.rows_per_thread) == (cluster, threads, rows)
    for s, us in zip(batch, B.unpack(u)):
        ref = oracle_steps(s, steps)
        assert np.linalg.norm(us - ref) / np.linalg.norm(ref) < 1e-8


def test_batch_autotune_and_uneven_sizes(ctx):
    batch = problems.heat_batch(nsys=20, sizes=(8, 16, 32, 48), dt=1e-3, seed=11)
    B = build(ctx, batch)
    u = B.timeSteps([s.u0 for s in batch], 3)
    assert B.last.failed == 0 and B.last.cluster in (1, 2, 4, 8) and B.last.threads in (256, 512)
    assert B.last.rows_per_thread in (2, 3, 4)
    with pytest.raises(Exception, match="rows_per_thread"):
        B.timeSteps([s.u0 for s in batch], 1, rows_per_thread=5)
    for s, us in zip(batch[:4], B.unpack(u)[:4]):
        ref = oracle_steps(s, 3)
        assert np.linalg.norm(us - ref) / np.linalg.norm(ref) < 1e-8


def test_batch_full_size_conservation(ctx):
    """256 Q1 systems, cells from {32, 48, ..., 256}^2, dt = 1e-3,
    50 steps.  With the natural boundary the mass 1^T M u is conserved by
    implicit Euler and the M-energy decays; both hold per system.  The
    systems of 32^2 and 48^2 cells of this full-size batch (solved in the
    same persistent launch as the large ones) match the oracle's per-step
    FP64 CG after all 50 steps."""
    batch = problems.heat_batch(nsys=256, dt=1e-3, seed=0)
    B = build(ctx, batch)
    u = B.timeSteps([s.u0 for s in batch], 50)
    assert B.last.failed == 0 and B.last.max_rel_residual <= 1e-10
    for s, us in zip(batch, B.unpack(u)):
        M = O.CooMatrix(s.M.n, s.M.n, s.M.rows, s.M.cols, s.M.vals)
        m0 = M.mvmul(s.u0).sum()
        m1 = M.mvmul(us).sum()
        assert abs(m1 - m0) <= 1e-9 * max(1.0, abs(m0)) + 1e-9 * np.abs(M.mvmul(s.u0)).sum()
        assert us @ M.mvmul(us) <= s.u0 @ M.mvmul(s.u0) * (1 + 1e-12)
    checked = 0
    for s, us in zip(batch, B.unpack(u)):
        if s.K.n > 49 * 49:
            continue
        ref = oracle_steps(s, 50)
        assert np.linalg.norm(us - ref) / np.linalg.norm(ref) < 5e-8
        checked += 1
    assert checked >= 10
