"""GPU sparse products through the C ABI against the oracle's COO scatter."""
import numpy as np
import pytest

import oracle as O
from fixtures import coo_oracle, fe_system, java_sparse, java_vector
from jfem_b200 import IllegalArgumentException, SparseMatrix
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu

SEEDED = [  # SparseMvMulTest.java:12-113 (tiny, small, large)
    (10, 10, 14239078, 0.1, True, 124350987, 124350987),
    (500, 700, 891765234, 0.01, False, 124876, 81726534),
    (5000, 7000, 1627894, 0.05, False, 18429760, 323781645),
]


@pytest.mark.parametrize("case", SEEDED, ids=["tiny", "small", "large"])
def test_seeded_mvmul_tvmul(ctx, case):
    rows, cols, seed, dens, integer, vseed, tseed = case
    ri, ci, v = java_sparse(rows, cols, seed, dens, integer)
    ref = O.CooMatrix(rows, cols, ri, ci, v)
    A = SparseMatrix.from_coo(rows, cols, ri, ci, v, ctx)
    x = java_vector(cols, vseed, integer)
    t = java_vector(rows, tseed, integer)
    y, yr = A.mvMul(x), ref.mvmul(x)
    np.testing.assert_allclose(y, yr, rtol=1e-12, atol=1e-12 * np.abs(yr).max())
    z, zr = A.tvMul(t), ref.tvmul(t)
    np.testing.assert_allclose(z, zr, rtol=1e-12, atol=1e-12 * np.abs(zr).max())
    if integer:   # integer data: exact
        assert np.array_equal(y, yr) and np.array_equal(z, zr)


@pytest.mark.parametrize("p,cells", [(1, 64), (2, 32), (2, 128)])
def test_fe_matrix_spmv(ctx, p, cells):
    sp, sy = fe_system(p, cells)
    ref = coo_oracle(sy)
    A = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    x = np.random.default_rng(1).standard_normal(sy.n)
    yr = ref.mvmul(x)
    np.testing.assert_allclose(A.spmv(x), yr, rtol=1e-12, atol=1e-13 * np.abs(yr).max())
    np.testing.assert_allclose(A.diag(), ref.diag(), rtol=0, atol=0)


def test_duplicates_zeros_and_empty_rows(ctx):
    ri = np.array([0, 0, 0, 2, 2, 3, 3], np.int32)
    ci = np.array([1, 1, 0, 2, 0, 3, 3], np.int32)
    v = np.array([1.5, 2.5, 0.0, -1.0, 4.0, 2.0, -2.0])   # row 3 merges to an explicit zero
    ref = O.CooMatrix(5, 4, ri, ci, v)
    A = DeviceMatrix(5, 4, ri, ci, v, ctx)
    x = np.array([1.0, 2.0, 3.0, 4.0])
    assert np.array_equal(A.spmv(x), ref.mvmul(x))
    t = np.arange(5.0)
    assert np.array_equal(A.spmv_t(t), ref.tvmul(t))
    assert A.nnz == 3     # (0,1), (2,2), (2,0)


def test_empty_matrix(ctx):
    A = DeviceMatrix(3, 3, [], [], [], ctx)
    assert np.array_equal(A.spmv(np.ones(3)), np.zeros(3))


def test_long_rows(ctx):
    """A row longer than one staging block takes the long-row path."""
    n = 6000
    ri = np.concatenate([np.zeros(n, np.int32), np.arange(1, 50, dtype=np.int32)])
    ci = np.concatenate([np.arange(n, dtype=np.int32), np.arange(1, 50, dtype=np.int32)])
    v = np.concatenate([np.linspace(-1, 1, n), np.ones(49)])
    ref = O.CooMatrix(50, n, ri, ci, v)
    A = DeviceMatrix(50, n, ri, ci, v, ctx)
    x = np.cos(np.arange(n))
    np.testing.assert_allclose(A.spmv(x), ref.mvmul(x), rtol=1e-12, atol=1e-12)


def test_index_out_of_bounds(ctx):
    with pytest.raises(IllegalArgumentException):
        DeviceMatrix(2, 2, [0, 5], [0, 0], [1.0, 1.0], ctx)


def test_linearity_full_size(ctx):
    """Q2 512x512 (1,050,625 rows): A(a x + b y) = a A x + b A y."""
    sp, sy = fe_system(2, 512)
    A = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(sy.n), rng.standard_normal(sy.n)
    lhs = A.spmv(2.0 * x - 0.5 * y)
    rhs = 2.0 * A.spmv(x) - 0.5 * A.spmv(y)
    np.testing.assert_allclose(lhs, rhs, rtol=1e-10, atol=1e-10 * np.abs(rhs).max())


def test_wide_offsets_use_32bit_columns(ctx):
    """Column offsets beyond 16 bits keep the 32-bit index stream (a column
    150,000 away from its row); the product is unchanged."""
    n = 200_000
    rng = np.random.default_rng(8)
    ri = np.array([0, 0, 1, 2, 2, 2], np.int32)
    ci = np.array([0, 150_000, 1, 2, 199_999, 3], np.int32)
    v = rng.standard_normal(ri.size)
    A = DeviceMatrix(3, n, ri, ci, v, ctx)
    x = rng.standard_normal(n)
    ref = O.CooMatrix(3, n, ri, ci, v).mvmul(x)
    np.testing.assert_allclose(A.spmv(x), ref, rtol=1e-14, atol=1e-14)


def test_16bit_offsets_match_32bit(ctx, monkeypatch):
    """The 16-bit column-offset stream gives bit-identical products."""
    sp, sy = fe_system(2, 24)
    x = np.sin(np.arange(sy.n))
    A16 = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    monkeypatch.setenv("JFEM_IDX16", "0")
    A32 = DeviceMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals, ctx)
    assert np.array_equal(A16.spmv(x), A32.spmv(x))
    assert np.array_equal(A16.spmv_t(x), A32.spmv_t(x))


def test_transfer_matrices_slice_base_columns(ctx, monkeypatch):
    """Rectangular transfer matrices (the nodal prolongation between Q1
    grids of 256^2 and 512^2 cells: 263,169 x 66,049, and its transpose)
    have columns far from their rows; their 16-bit column offsets are taken
    from a base column per 32-row slice.  Products equal the oracle's COO
    scatter and, bit for bit, the 32-bit-column layout."""
    from fixtures import mg_levels
    h = mg_levels(1, 256, 2)
    ri, ci, v = h.prolong[0]
    nf, nc = h.systems[1].n, h.systems[0].n
    P = DeviceMatrix(nf, nc, ri, ci, v, ctx)
    ref = O.CooMatrix(nf, nc, ri, ci, v)
    rng = np.random.default_rng(21)
    xc, xf = rng.standard_normal(nc), rng.standard_normal(nf)
    y, z = P.spmv(xc), P.spmv_t(xf)
    np.testing.assert_allclose(y, ref.mvmul(xc), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(z, ref.tvmul(xf), rtol=1e-12, atol=1e-13)
    monkeypatch.setenv("JFEM_IDX16", "0")
    P32 = DeviceMatrix(nf, nc, ri, ci, v, ctx)
    assert np.array_equal(P32.spmv(xc), y) and np.array_equal(P32.spmv_t(xf), z)
