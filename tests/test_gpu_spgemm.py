"""Sparse products on the GPU (SparseMatrix.mmMul / Matrix.tmMul, Galerkin
coarse operators) and the AMG-from-matrix hierarchy, against the oracle.

The GPU sums each entry from 0 in ascending inner index without fused
multiply-adds, as the oracle does, so products are compared bit for bit."""
import numpy as np
import pytest

import oracle as O
from fixtures import mg_levels
from jfem_b200 import JacobiSmoother, MGPreconditioner
from jfem_b200 import _native as N
from jfem_b200.linalg import DeviceMatrix, IllegalArgumentException, IterativeSolver, SparseMatrix

pytestmark = pytest.mark.gpu


def random_sparse(rows, cols, density, seed, integer=False):
    rng = np.random.default_rng(seed)
    m = int(rows * cols * density)
    key = np.unique(rng.integers(0, rows * cols, m))       # no duplicates: the merge order is not under test
    ri, ci = (key // cols).astype(np.int32), (key % cols).astype(np.int32)
    v = rng.integers(-4, 5, key.size).astype(np.float64) if integer else rng.standard_normal(key.size)
    return ri, ci, v


def both(rows, cols, trip, ctx):
    return DeviceMatrix(rows, cols, *trip, ctx), O.CooMatrix(rows, cols, *trip)


def merged(dev):
    """The oracle matrix of the device matrix's merged entries (assembled FE
    matrices carry duplicates; their merge is checked elsewhere, so products
    are compared on identical inputs)."""
    return O.CooMatrix(dev.rows, dev.cols, *dev.coo())


def assert_same(dev, ref: O.CooMatrix):
    ptr, col, val = dev.csr()
    assert dev.rows == ref.rows and dev.cols == ref.cols
    assert np.array_equal(np.repeat(np.arange(dev.rows), np.diff(ptr)), ref.ri)
    assert np.array_equal(col, ref.ci)
    assert np.array_equal(val, ref.v)          # bitwise


@pytest.mark.parametrize("m,k,n,dens", [(50, 70, 40, 0.08), (300, 200, 250, 0.02), (1, 5, 1, 1.0)])
def test_mmmul_matches_oracle(ctx, m, k, n, dens):
    A, Ao = both(m, k, random_sparse(m, k, dens, 1), ctx)
    B, Bo = both(k, n, random_sparse(k, n, dens, 2), ctx)
    assert_same(A.mmMul(B), Ao.mmmul(Bo))


def test_tmmul_matches_oracle(ctx):
    A, Ao = both(120, 90, random_sparse(120, 90, 0.05, 3), ctx)
    B, Bo = both(120, 60, random_sparse(120, 60, 0.05, 4), ctx)
    assert_same(A.tmMul(B), Ao.tmmul(Bo))


def test_exact_zero_sums_are_not_stored(ctx):
    """[[1, -1]] [[1], [1]] = [[0]]: SparseMatrix.add skips zeros."""
    A = DeviceMatrix(1, 2, [0, 0], [0, 1], [1.0, -1.0], ctx)
    B = DeviceMatrix(2, 1, [0, 1], [0, 0], [1.0, 1.0], ctx)
    C = A.mmMul(B)
    assert C.nnz == 0 and C.rows == 1 and C.cols == 1
    # integer-valued product with many cancellations against a dense product
    ti, tb = random_sparse(80, 60, 0.1, 5, integer=True), random_sparse(60, 70, 0.1, 6, integer=True)
    A, B = DeviceMatrix(80, 60, *ti, ctx), DeviceMatrix(60, 70, *tb, ctx)
    Ad = np.zeros((80, 60)); Ad[ti[0], ti[1]] = ti[2]
    Bd = np.zeros((60, 70)); Bd[tb[0], tb[1]] = tb[2]
    ref = Ad @ Bd
    C = A.mmMul(B)
    ptr, col, val = C.csr()
    Cd = np.zeros((80, 70)); Cd[np.repeat(np.arange(80), np.diff(ptr)), col] = val
    assert np.array_equal(Cd, ref)
    assert C.nnz == np.count_nonzero(ref)


def test_empty_and_incompatible(ctx):
    A = DeviceMatrix(4, 3, [], [], [], ctx)
    B = DeviceMatrix(3, 5, [0], [1], [2.0], ctx)
    C = A.mmMul(B)
    assert (C.rows, C.cols, C.nnz) == (4, 5, 0)
    with pytest.raises(IllegalArgumentException):
        B.mmMul(B)
    with pytest.raises(IllegalArgumentException):
        A.tmMul(B)


def test_sparse_matrix_dropin(ctx):
    """SparseMatrix.mmMul / tmMul return SparseMatrix objects with the product's triples."""
    ri, ci, v = random_sparse(40, 30, 0.1, 7)
    S = SparseMatrix.from_coo(40, 30, ri, ci, v, ctx)
    T = S.tmMul(S)
    ref = O.CooMatrix(40, 30, ri, ci, v).tmmul(O.CooMatrix(40, 30, ri, ci, v))
    tri, tci, tv = T.coo()
    assert T.getRows() == 30 and T.getCols() == 30
    assert np.array_equal(tri, ref.ri) and np.array_equal(tci, ref.ci) and np.array_equal(tv, ref.v)
    U = S.mmMul(S.transpose())
    assert (U.getRows(), U.getCols()) == (40, 40)


@pytest.mark.parametrize("p,coarse,L", [(1, 4, 5), (2, 2, 5)])
def test_galerkin_matches_oracle(ctx, p, coarse, L):
    """(P^T A) P level by level (AMGFromMatrix's association), bit for bit."""
    h = mg_levels(p, coarse, L, modes=4, seed=3)
    fine = h.systems[-1]
    A = DeviceMatrix(fine.n, fine.n, fine.rows, fine.cols, fine.vals, ctx)
    Ao = merged(A)
    for l in range(L - 2, -1, -1):
        nf, nc = h.systems[l + 1].n, h.systems[l].n
        P = DeviceMatrix(nf, nc, *h.prolong[l], ctx)
        Po = merged(P)
        A, Ao = A.galerkin(P), Po.tmmul(Ao).mmmul(Po)
        assert_same(A, Ao)


def test_galerkin_with_restriction(ctx):
    """(R A) P with an explicit restriction (AMGSpace.createSystems)."""
    h = mg_levels(1, 4, 3, modes=4, seed=1)
    fine = h.systems[-1]
    nf, nc = h.systems[-1].n, h.systems[-2].n
    A = DeviceMatrix(nf, nf, fine.rows, fine.cols, fine.vals, ctx)
    P = DeviceMatrix(nf, nc, *h.prolong[-1], ctx)
    pr, pc, pv = h.prolong[-1]
    R = DeviceMatrix(nc, nf, pc, pr, pv * 0.25, ctx)
    Ao, Po, Ro = merged(A), merged(P), merged(R)
    assert_same(A.galerkin(P, R), Ro.mmmul(Ao).mmmul(Po))


def test_chunked_expansion_is_identical(ctx, monkeypatch):
    """Rows split into many chunks of at most 4,096 products give the same matrix."""
    h = mg_levels(2, 8, 2, modes=2, seed=5)
    fine = h.systems[-1]
    nf, nc = h.systems[1].n, h.systems[0].n
    A = DeviceMatrix(nf, nf, fine.rows, fine.cols, fine.vals, ctx)
    P = DeviceMatrix(nf, nc, *h.prolong[0], ctx)
    ref = A.galerkin(P)
    monkeypatch.setenv("JFEM_SPGEMM_CHUNK", "4096")
    got = A.galerkin(P)
    for a, b in zip(got.csr(), ref.csr()):
        assert np.array_equal(a, b)


def test_galerkin_full_size_property(ctx):
    """Q2 512^2 finest level (chunked expansion): (P^T A P) x = P^T (A (P x))."""
    h = mg_levels(2, 256, 2, modes=2, seed=0)
    fine = h.systems[-1]
    nf, nc = h.systems[1].n, h.systems[0].n
    A = DeviceMatrix(nf, nf, fine.rows, fine.cols, fine.vals, ctx)
    P = DeviceMatrix(nf, nc, *h.prolong[0], ctx)
    C = A.galerkin(P)
    x = np.random.default_rng(0).standard_normal(nc)
    ref = P.spmv_t(A.spmv(P.spmv(x)))
    got = C.spmv(x)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
    assert C.rows == nc and C.cols == nc
    # nested conforming spaces: on interior nodes the Galerkin operator is the assembled coarse operator
    sc = h.systems[0]
    Ac = DeviceMatrix(nc, nc, sc.rows, sc.cols, sc.vals, ctx)
    inner = np.ones(nc, bool)
    inner[np.asarray(h.boundary[0], dtype=np.int64)] = False
    xi = np.where(inner, x, 0.0)
    d = np.where(inner, C.spmv(xi) - Ac.spmv(xi), 0.0)
    assert np.linalg.norm(d) <= 1e-13 * np.linalg.norm(np.where(inner, Ac.spmv(xi), 0.0))


def test_amg_from_matrix(ctx):
    """AMGFromMatrix: Galerkin coarse systems, the V-cycle against the oracle's
    V-cycle on the oracle's Galerkin systems, and a PCG solve with it."""
    L = 5
    h = mg_levels(1, 4, L, modes=6, seed=2)
    mats = [DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx) for s in h.systems]
    prol = [DeviceMatrix(h.systems[l + 1].n, h.systems[l].n, *h.prolong[l], ctx) for l in range(L - 1)]
    mg = MGPreconditioner(mats, prol, h.boundary, [None] + [JacobiSmoother(2, 2 / 3)] * (L - 1), cycles=1,
                          use_fmg=False, ctx=ctx)
    amg = mg.AMGFromMatrix(mats[-1], lambda l, A: JacobiSmoother(2, 2 / 3))
    assert amg.maxLevel() == L - 1
    # oracle hierarchy with the oracle's Galerkin systems
    gal = [merged(mats[-1])]
    prol_o = [merged(P) for P in prol]
    for l in range(L - 2, -1, -1):
        gal.append(prol_o[l].tmmul(gal[-1]).mmmul(prol_o[l]))
    gal.reverse()
    for l in range(L):
        assert_same(amg.getSystem(l), gal[l])
    mg_o = O.MGPreconditioner(gal, prol_o, h.boundary, [None] + [(O.SMOOTH_JACOBI, 2, 2 / 3)] * (L - 1), cycles=1,
                              use_fmg=False)
    b = h.finest.rhs
    x0 = np.random.default_rng(1).standard_normal(b.size) * 0.1
    got, ref = amg.vCycle(x0, b), mg_o.vcycle(x0, b)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    tol = 1e-8 * np.linalg.norm(b)
    s = IterativeSolver(ctx=ctx)
    x = s.solvePCG(mats[-1], amg, b, tol)
    ref = O.solve_pcg(gal[-1], mg_o, b, tol)
    assert s.last.status == N.OK and abs(s.iterations - ref.iterations) <= 1
    assert np.linalg.norm(b - mats[-1].spmv(x)) <= tol
