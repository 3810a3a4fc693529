"""The structured-grid assembler that produces the systems (no GPU)."""
import numpy as np

import oracle as O
from jfem_b200.assembly import Space, assemble, lagrange_1d, prolongation


def test_first_seen_numbering_q1():
    s = Space(1, 2, 2)
    # cell (0,0): local x-fastest -> 0,1,2,3 ; cell (0,1) shares its top edge
    assert s.cell_dofs[0].tolist() == [0, 1, 2, 3]
    assert s.cell_dofs[1].tolist() == [2, 3, 4, 5]
    assert s.n == 9


def test_lagrange_partition_of_unity():
    t = np.linspace(0, 1, 17)
    for p in (1, 2, 3):
        v, d = lagrange_1d(p, t)
        np.testing.assert_allclose(v.sum(0), 1.0, atol=1e-14)
        np.testing.assert_allclose(d.sum(0), 0.0, atol=1e-12)


def test_stiffness_kernel_and_symmetry():
    for p in (1, 2):
        s = Space(p, 3, 3)
        sy = assemble(s, 1.0, 0.0)            # no Dirichlet on constants check below uses raw element sums
        D = O.CooMatrix(s.n, s.n, sy.rows, sy.cols, sy.vals).dense()
        np.testing.assert_allclose(D, D.T, atol=1e-14)
        # Dirichlet rows/columns are identity
        bd = s.boundary_nodes()
        np.testing.assert_allclose(D[np.ix_(bd, bd)], np.eye(bd.size))
        inner = np.setdiff1d(np.arange(s.n), bd)
        assert np.all(D[np.ix_(inner, bd)] == 0)


def test_galerkin_identity():
    """multigrid/MultiGridSpaceTest.java:93-127: P^T A_f P = A_c (interior)."""
    for p in (1, 2):
        c = Space(p, 4, 4)
        f = c.refined()
        Af, Ac = assemble(f, 1.0, 0.0), assemble(c, 1.0, 0.0)
        r, cc, v = prolongation(c, f)
        P = np.zeros((f.n, c.n))
        P[r, cc] = v
        Dfx = O.CooMatrix(f.n, f.n, Af.rows, Af.cols, Af.vals).dense()
        Dcx = O.CooMatrix(c.n, c.n, Ac.rows, Ac.cols, Ac.vals).dense()
        ib = np.setdiff1d(np.arange(c.n), c.boundary_nodes())
        G = P.T @ Dfx @ P
        np.testing.assert_allclose(G[np.ix_(ib, ib)], Dcx[np.ix_(ib, ib)], atol=1e-12)


def test_prolongation_interpolates():
    """MultiGridSpaceTest.java:24-60: P reproduces the coarse FE function."""
    for p in (1, 2):
        c = Space(p, 3, 5)
        f = c.refined()
        r, cc, v = prolongation(c, f)
        P = np.zeros((f.n, c.n))
        P[r, cc] = v
        cx, cy = c.node_points()
        fx, fy = f.node_points()
        u = lambda x, y: x ** p + 2 * x * y - y ** p
        np.testing.assert_allclose(P @ u(cx, cy), u(fx, fy), atol=1e-13)


def test_rhs_converges():
    """Q1 solution of -Lap u + 5u = f with a single mode approaches the exact one."""
    errs = []
    for cells in (8, 16, 32):
        s = Space(1, cells, cells)
        k = 1
        f = lambda x, y: (2 * (k * np.pi) ** 2 + 5) * np.sin(k * np.pi * x) * np.sin(k * np.pi * y)
        sy = assemble(s, 1.0, 5.0, source=f)
        D = O.CooMatrix(s.n, s.n, sy.rows, sy.cols, sy.vals).dense()
        u = np.linalg.solve(D, sy.rhs)
        px, py = s.node_points()
        errs.append(np.abs(u - np.sin(np.pi * px) * np.sin(np.pi * py)).max())
    assert errs[1] < errs[0] / 3 and errs[2] < errs[1] / 3
