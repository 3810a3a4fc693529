"""FGMRES and the multigrid + learned-smoother preconditioner on the GPU,
against the numpy FGMRES oracle, the multigrid oracle and the float64 network
oracle."""
import numpy as np
import pytest
import torch

import oracle as O
import oracle.cnn_oracle as CO
from fixtures import coo_oracle, mg_levels
from jfem_b200 import IterativeSolver, JacobiSmoother, MGPreconditioner
from jfem_b200 import _native as N
from jfem_b200.cnn import LearnedSmoother, MGCNNPreconditioner, he_init, pixel_map, unpack
from jfem_b200.linalg import DeviceMatrix
from oracle.fgmres import solve_fgmres

pytestmark = pytest.mark.gpu


def setup(ctx, p=1, coarse=4, L=4, precision="fp64", cycles=1, use_fmg=False):
    h = mg_levels(p, coarse, L, mass=5.0)
    mats_o = [coo_oracle(s) for s in h.systems]
    prol_o = [O.CooMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l]) for l in range(L - 1)]
    mg_o = O.MGPreconditioner(mats_o, prol_o, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2 / 3)] * (L - 1),
                              cycles=cycles, use_fmg=use_fmg)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (L - 1), cycles=cycles,
                          use_fmg=use_fmg, precision=precision, ctx=ctx)
    return h, mg_o, mg, mats


@pytest.mark.parametrize("use_graph", [True, False])
def test_fgmres_mg_matches_oracle(ctx, use_graph):
    h, mg_o, mg, mats = setup(ctx)
    A_o = coo_oracle(h.finest)
    b = h.finest.rhs
    tol = 1e-10 * np.linalg.norm(b)
    x_o, it_o, rs_o, st_o, hist_o = solve_fgmres(A_o.mvmul, mg_o.mvmul, b, tol, restart=30)
    s = IterativeSolver(ctx=ctx)
    s.use_graph = use_graph
    x = s.solveFGMRES(mats[-1], mg, b, tol, restart=30)
    assert st_o == O.OK and s.last.status == N.OK
    assert s.iterations == it_o
    k = min(5, it_o)
    np.testing.assert_allclose(s.last.history[:k], hist_o[:k], rtol=1e-8)
    assert np.linalg.norm(b - A_o.mvmul(x)) <= tol
    np.testing.assert_allclose(x, x_o, rtol=1e-8, atol=1e-8 * np.abs(x_o).max())


def test_fgmres_short_restart(ctx):
    """restart = 3 exercises the restart rule of GMRES.java:92."""
    h, mg_o, mg, mats = setup(ctx)
    A_o = coo_oracle(h.finest)
    b = h.finest.rhs
    tol = 1e-10 * np.linalg.norm(b)
    x_o, it_o, rs_o, st_o, _ = solve_fgmres(A_o.mvmul, mg_o.mvmul, b, tol, restart=3)
    s = IterativeSolver(ctx=ctx)
    x = s.solveFGMRES(mats[-1], mg, b, tol, restart=3)
    assert s.last.status == N.OK and st_o == O.OK
    assert s.iterations == it_o and s.last.restarts == rs_o
    assert np.linalg.norm(b - A_o.mvmul(x)) <= tol


def _mgcnn(ctx, h, mg, mats, weights, use_net=True, out_scale=1.0):
    H, W, dof = pixel_map(h.spaces[-1])
    net = LearnedSmoother(ctx, weights=weights)
    pc = MGCNNPreconditioner(mg, net, mats[-1], H, W, dof, h.boundary[-1], out_scale=out_scale, use_net=use_net)
    return net, pc, H, W, dof


def test_mgcnn_apply_matches_oracles(ctx):
    """z = V32(v) + s * net(D^-1 r' / s): the V-cycle part against the FP64
    multigrid oracle (FP32 tolerance), the network part against the float64
    network oracle run on the GPU's own r' (BF16 tolerance)."""
    h, mg_o, mg, mats = setup(ctx, L=4)
    w = he_init(3, gain_last=0.5)
    net, pc, H, W, dof = _mgcnn(ctx, h, mg, mats, w, use_net=False)
    n = h.finest.n
    v = np.random.default_rng(5).standard_normal(n)
    vt = torch.tensor(v, device="cuda")
    z0 = pc.apply_dev(vt).cpu().numpy()
    ref = mg_o.mvmul(v)
    assert np.linalg.norm(z0 - ref) <= 1e-4 * np.linalg.norm(ref)
    pc.set(0.75, use_net=True)
    z1 = pc.apply_dev(vt).cpu().numpy()
    A_o = coo_oracle(h.finest)
    q = (v - A_o.mvmul(z0)) / A_o.diag()
    sc = np.sqrt(np.mean(q ** 2))
    img = (q[dof] / sc).reshape(1, H, W)
    y = CO.forward(unpack(w), img)[0].reshape(-1)
    corr = np.zeros(n)
    corr[dof] = y * sc * 0.75
    corr[h.boundary[-1]] = 0.0
    got = z1 - z0
    assert np.linalg.norm(got - corr) <= 3e-2 * np.linalg.norm(corr)
    assert np.all(got[h.boundary[-1]] == 0.0)


@pytest.mark.parametrize("use_net", [False, True])
def test_fgmres_mgcnn_converges(ctx, use_net):
    """FGMRES(30) with the nonlinear preconditioner reaches the FP64 true
    residual tolerance (random network weights: the flexible method absorbs a
    poor correction)."""
    h, mg_o, mg, mats = setup(ctx, L=5)
    net, pc, *_ = _mgcnn(ctx, h, mg, mats, he_init(7, gain_last=0.1), use_net=use_net)
    b = h.finest.rhs
    tol = 1e-8 * np.linalg.norm(b)
    s = IterativeSolver(ctx=ctx)
    x = s.solveFGMRES(mats[-1], pc, b, tol, restart=30)
    assert s.last.status == N.OK
    assert s.last.final_residual <= tol
    A_o = coo_oracle(h.finest)
    assert np.linalg.norm(b - A_o.mvmul(x)) <= tol * 1.0001
    assert s.iterations < 40


def test_mgcnn_rejects_other_solvers(ctx):
    h, mg_o, mg, mats = setup(ctx)
    net, pc, *_ = _mgcnn(ctx, h, mg, mats, he_init(1))
    s = IterativeSolver(ctx=ctx)
    with pytest.raises(Exception):
        s.solvePGMRES(mats[-1], pc, h.finest.rhs, 1e-8)
