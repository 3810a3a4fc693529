"""Taylor-Hood Stokes assembly (host logic, no GPU)."""
import numpy as np
import scipy.sparse as sps
import scipy.sparse.linalg as spl

from jfem_b200.stokes import (TaylorHoodSpace, assemble_stokes, fourier_force, lumped_pressure_mass,
                              stokes_problem, velocity_block, velocity_prolongation)


def csr(R, C, V, n, m=None):
    return sps.coo_matrix((V, (R, C)), shape=(n, m or n)).tocsr()


def test_numbering_and_sizes():
    th = TaylorHoodSpace(4, 6)
    assert th.nv == 2 * 9 * 13 and th.np_ == 5 * 7 and th.n == th.nv + th.np_
    # velocity DOFs of a cell: 9 nodes per component, component 1 offset by nv1
    assert np.all(th.cell_velocity_dofs[:, 9:] - th.cell_velocity_dofs[:, :9] == th.nv1)
    bd = th.velocity_boundary()
    assert bd.size == 2 * (2 * 9 + 2 * 13 - 4)


def test_system_symmetric_and_solvable():
    th = TaylorHoodSpace(6, 6)
    s = assemble_stokes(th, force=fourier_force(seed=3))
    A = csr(s.rows, s.cols, s.vals, s.n)
    assert abs(A - A.T).max() < 1e-15
    x = spl.spsolve(A.tocsc(), s.rhs)
    assert np.linalg.norm(A @ x - s.rhs) < 1e-10
    u0 = x[:th.nv1]
    _, py = th.velocity_points()
    assert np.allclose(u0[np.isclose(py, 1.0)], 1.0)                # the lid
    assert x[th.nv] == 0.0                                          # the fixed pressure unknown


def test_divergence_of_linear_fields():
    """B u = 0 for the divergence-free u = (y, -x) on every pressure row
    (before boundary elimination); and B u = int q for u = (x, 0)."""
    th = TaylorHoodSpace(5, 4)
    s = assemble_stokes(th, lid=False)
    # rebuild the unconstrained B from the pressure rows of an unconstrained assembly
    from jfem_b200 import stokes as S
    K, B0, B1, Mp, _ = S._tables(th.hx, th.hy)
    gx, gy = th.velocity_points()
    nc = th.cx * th.cy
    B = np.zeros((th.np_, th.nv))
    for c in range(nc):
        for i, p in enumerate(th.cell_pnodes[c]):
            B[p, th.cell_vnodes[c]] += B0[i]
            B[p, th.cell_vnodes[c] + th.nv1] += B1[i]
    u = np.concatenate([gy, -gx])
    assert np.abs(B @ u).max() < 1e-14
    u = np.concatenate([gx, np.zeros(th.nv1)])
    np.testing.assert_allclose(B @ u, lumped_pressure_mass(th), rtol=1e-12)


def test_prolongation_interpolates_quadratics():
    c, f = TaylorHoodSpace(3, 3), TaylorHoodSpace(6, 6)
    R, C, V = velocity_prolongation(c, f)
    P = csr(R, C, V, f.nv, c.nv)
    xc, yc = c.velocity_points()
    xf, yf = f.velocity_points()
    q = lambda x, y: 1 + x - 2 * y + 3 * x * y + x * x - y * y
    u = np.concatenate([q(xc, yc), 2 * q(xc, yc)])
    np.testing.assert_allclose(P @ u, np.concatenate([q(xf, yf), 2 * q(xf, yf)]), atol=1e-13)


def test_velocity_block_is_the_system_block():
    th = TaylorHoodSpace(4, 4)
    s = assemble_stokes(th, nu=2.0, force=None, lid=False)
    A = csr(s.rows, s.cols, s.vals, s.n)
    R, C, V, _ = velocity_block(th, nu=2.0)
    Av = csr(R, C, V, th.nv)
    assert abs(A[:th.nv, :th.nv] - Av).max() < 1e-15


def test_problem_levels():
    p = stokes_problem(16, 4)
    assert [t.cx for t in p.spaces] == [4, 8, 16]
    assert p.pressure_inverse.size == p.spaces[-1].np_ and p.pressure_inverse[0] == 1.0


def test_taylor_hood_prolongation_and_patches():
    """The whole-space prolongation interpolates a quadratic velocity and a
    bilinear pressure exactly; the monolithic Schwarz patches take the
    velocity and pressure unknowns of their cells (8 x 8 cells inside the
    domain at partitions 2 * 2^(l-1), overlap 2) and the zero-boundary list is
    the Dirichlet velocity plus the first pressure unknown."""
    from jfem_b200.schwarz import cartesian_patch_dofs
    from jfem_b200.stokes import (MixedCells, TaylorHoodSpace, mixed_zero_boundary, schwarz_partitions,
                                  taylor_hood_prolongation)
    c, f = TaylorHoodSpace(4, 4), TaylorHoodSpace(8, 8)
    R, Cc, V = taylor_hood_prolongation(c, f)
    P = sps.csr_matrix((V, (R, Cc)), shape=(f.n, c.n))

    def field(th):
        xv, yv = th.velocity_points()
        g = np.arange(th.np_)
        xp, yp = (g // th.pny) * th.hx, (g % th.pny) * th.hy
        return np.concatenate([xv ** 2 - yv, 2 * xv * yv, 1 + xp - 3 * yp + xp * yp])

    np.testing.assert_allclose(P @ field(c), field(f), atol=1e-13)
    assert schwarz_partitions(1) == (2, 2) and schwarz_partitions(3) == (8, 8)
    th = TaylorHoodSpace(16, 16)
    _, patches = cartesian_patch_dofs(MixedCells(th), schwarz_partitions(2), 2)
    assert len(patches) == 16
    assert max(len(p) for p in patches) == 2 * 17 * 17 + 81
    inner = patches[5]                                  # partition (1, 1): cells 2..9 x 2..9
    assert len(inner) == 2 * 17 * 17 + 81 and np.all(np.diff(inner) > 0)
    assert np.sum(inner >= th.nv) == 81
    bd = mixed_zero_boundary(th)
    assert bd[-1] == th.nv and np.array_equal(np.sort(bd[:-1]), np.sort(th.velocity_boundary()))
