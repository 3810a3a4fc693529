"""Finite-element assembly on the GPU (jfg_assemble_tp) against the host
assembler: numbering, Dirichlet list, merged matrix and right-hand side."""
import numpy as np
import pytest

from jfem_b200 import _native as N
from jfem_b200.assembly import Space, assemble, assemble_device
from jfem_b200.linalg import DeviceMatrix, IterativeSolver
from jfem_b200.problems import modes_source

pytestmark = pytest.mark.gpu


def host(space, **kw):
    sy = assemble(space, **kw)
    return sy, DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals)


def check(space, tol=1e-14, **kw):
    sy, Ah = host(space, **kw)
    dirichlet = kw.get("dirichlet", True)
    A, rhs, bd, nog = assemble_device(space, **kw)
    assert np.array_equal(nog, space.node_of_grid)
    if dirichlet:
        assert np.array_equal(bd, space.boundary_nodes())
    ph, ch, vh = Ah.csr()
    pg, cg, vg = A.csr()
    assert np.array_equal(pg, ph) and np.array_equal(cg, ch)
    np.testing.assert_allclose(vg, vh, rtol=tol, atol=tol * np.abs(vh).max())
    if kw.get("source") is not None:
        np.testing.assert_allclose(rhs, sy.rhs, rtol=1e-13, atol=1e-13 * np.abs(sy.rhs).max())
    else:
        assert not rhs.any()
    return sy, A, rhs


@pytest.mark.parametrize("p,cx,cy", [(1, 8, 8), (2, 6, 4), (3, 3, 5), (1, 1, 1), (2, 1, 3)])
def test_poisson_matches_host(ctx, p, cx, cy):
    f, _ = modes_source(4, 0)
    check(Space(p, cx, cy), grad_coef=1.0, mass_coef=5.0, source=f)


def test_domain_and_kappa(ctx):
    sp = Space(2, 10, 7, 0.5, 2.0, -1.0, 0.25)
    kap = np.exp(np.random.default_rng(3).standard_normal(sp.cx * sp.cy))
    f, _ = modes_source(3, 1)
    check(sp, grad_coef_cells=kap, mass_coef=0.0, source=f)


def test_natural_boundary_mass(ctx):
    """The heat-batch matrices: no Dirichlet rows (dirichlet=False)."""
    sp = Space(1, 12, 12)
    check(sp, grad_coef=1e-3, mass_coef=1.0, dirichlet=False)
    check(sp, grad_coef=0.0, mass_coef=1.0, dirichlet=False)


def test_full_size_q2_512(ctx):
    """The benchmark system (Q2 512^2, 16 x 16 modes) and a few CG steps on it."""
    f, _ = modes_source(16, 0)
    sy, A, rhs = check(Space(2, 512, 512), grad_coef=1.0, mass_coef=5.0, source=f)
    assert A.nnz == 16707665
    s = IterativeSolver(ctx=ctx)
    x = s._run(N.CG, A, None, rhs, 1e-30, s._start(len(rhs)), maxit=20)
    assert s.last.status == N.NOT_CONVERGED and np.isfinite(x).all()


@pytest.mark.parametrize("cx,cy,lid,pin", [(8, 8, True, True), (6, 10, True, False), (4, 4, False, True)])
def test_taylor_hood_matches_host(ctx, cx, cy, lid, pin):
    from jfem_b200.stokes import TaylorHoodSpace, assemble_stokes, assemble_stokes_device, fourier_force
    th = TaylorHoodSpace(cx, cy)
    f = fourier_force(seed=1)
    sy = assemble_stokes(th, 0.7, f, lid=lid, pin_pressure=pin)
    Ah = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals)
    A, rhs, bd = assemble_stokes_device(th, 0.7, f, lid=lid, pin_pressure=pin)
    ph, ch, vh = Ah.csr()
    pg, cg, vg = A.csr()
    assert np.array_equal(pg, ph) and np.array_equal(cg, ch)
    np.testing.assert_allclose(vg, vh, rtol=1e-14, atol=1e-14 * np.abs(vh).max())
    np.testing.assert_allclose(rhs, sy.rhs, rtol=1e-13, atol=1e-13 * np.abs(sy.rhs).max())
    assert np.array_equal(bd, sy.velocity_boundary)
