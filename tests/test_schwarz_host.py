"""Schwarz patch builders (host logic) and the Schwarz oracle (no GPU);
the cases follow the reference's CartesianSchwarzTest."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, schwarz_test_matrix
from jfem_b200.assembly import Space
from jfem_b200.schwarz import cartesian_cell_patches, cartesian_patch_dofs, nine_colours


def dense_coo(a):
    r, c = np.nonzero(a)
    return O.CooMatrix(a.shape[0], a.shape[1], r.astype(np.int32), c.astype(np.int32), a[r, c])


@pytest.mark.parametrize("cells,parts", [((4, 6), (2, 3)), ((24, 27), (4, 9))])
def test_patches_partition_the_cells(cells, parts):
    """CartesianSchwarzTest.testPatches / testPatches2 (:35-104): without
    overlap the patches hold cells/partitions cells each and tile the grid."""
    cx, cy = cells
    pt = cartesian_cell_patches(cx, cy, parts, 0)
    assert len(pt) == parts[0] * parts[1]
    seen = set()
    for p in pt:
        assert len(p) == cx // parts[0] * cy // parts[1]
        for c in p:
            assert c not in seen
            seen.add(c)
    assert len(seen) == cx * cy


def test_restriction_covers_all_dofs():
    """CartesianSchwarzTest.testRestriction (:106-134): subtracting
    R_i^T R_i v patch after patch leaves nothing (Q2 DOFs, 6 x 6 cells)."""
    sp = Space(2, 6, 6)
    _, patches = cartesian_patch_dofs(sp, (2, 3), 0)
    v = np.arange(sp.n, dtype=np.float64)
    for d in patches:
        w = np.zeros(sp.n)
        w[d] = v[d]
        v = v - w
    assert np.linalg.norm(v) < 1e-14


def test_vertex_patches_and_overlap():
    """partitions -1: one patch per interior vertex with 2*overlap cells a side."""
    pt = cartesian_cell_patches(5, 4, (-1, -1), 1)
    assert len(pt) == 4 * 3
    assert all(len(p) == 4 for p in pt)
    pt = cartesian_cell_patches(6, 6, (3, 3), 1)
    sizes = sorted(len(p) for p in pt)
    assert sizes[0] == 9 and sizes[-1] == 16         # corner and interior blocks


def test_nine_colours():
    cols = nine_colours((6, 4))
    assert len(cols) == 9
    assert sorted(sum(cols, [])) == list(range(24))
    assert cols[0] == [0, 3, 12, 15] and cols[4] == [5, 17]


def test_oracle_projection():
    """CartesianSchwarzTest.testSchwarzProjection (:136-173): P = R^T A_i^-1 R A
    is a projection and A-self-adjoint (Q1, 2 x 2 cells, 2 x 2 partitions)."""
    sp = Space(1, 2, 2)
    a = schwarz_test_matrix(sp.n)
    _, patches = cartesian_patch_dofs(sp, (2, 2), 0)
    S = O.Schwarz(dense_coo(a), O.SCHWARZ_ADDITIVE, patches, 1.0)
    for i, d in enumerate(patches):
        R = np.zeros((d.size, sp.n))
        R[np.arange(d.size), d] = 1.0
        Ai = S.inverse(i)
        np.testing.assert_allclose(np.linalg.inv(Ai), R @ a @ R.T, atol=1e-12)   # selectFrom = R A R^T
        P = R.T @ Ai @ R @ a
        assert np.abs(P @ P - P).max() < 1e-14
        assert np.abs(P.T @ a - a @ P).max() < 1e-13


def test_oracle_corrections_are_consistent():
    """Every correction leaves the exact solution fixed, and three smoothing
    runs reduce the error of a zero start."""
    sp, sy = fe_system(1, 8)
    A = coo_oracle(sy)
    xs = np.linalg.solve(A.dense(), sy.rhs)
    _, patches = cartesian_patch_dofs(sp, (4, 4), 1)
    cols = nine_colours((4, 4))
    # additive: omega below 1 / (patches per DOF) keeps the sum of corrections stable
    for kind, om in ((O.SCHWARZ_MULTIPLICATIVE, 1.0), (O.SCHWARZ_COLORED, 0.7), (O.SCHWARZ_ADDITIVE, 0.2)):
        S = O.Schwarz(A, kind, patches, om, colours=cols if kind == O.SCHWARZ_COLORED else None)
        np.testing.assert_allclose(S.apply(xs, sy.rhs), xs, rtol=1e-12, atol=1e-12)
        x = np.zeros(sy.n)
        e0 = np.linalg.norm(xs)
        x = S.smooth(3, sy.rhs, x)
        assert np.linalg.norm(x - xs) < 0.9 * e0
