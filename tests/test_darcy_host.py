"""The Raviart-Thomas (RT0) mixed Darcy fixture on the CPU: structure and a
dense solve against the continuous problem it discretises."""
import numpy as np
import scipy.sparse as sps

from jfem_b200.darcy import rt0_darcy


def test_rt0_structure_and_dense_solve():
    s = rt0_darcy(16, 16)
    A = sps.csr_matrix((s.vals, (s.rows, s.cols)), shape=(s.n, s.n)).toarray()
    assert s.n == 2 * 16 * 17 + 256
    assert np.allclose(A, A.T)                              # VALUE_VALUE and DIV_VALUE both ways
    M = A[:s.nv, :s.nv]
    assert np.all(np.linalg.eigvalsh(M) > 0)                # the RT mass matrix is SPD
    assert np.allclose(A[s.nv:, s.nv:], 0)                  # saddle point
    B = A[s.nv:, :s.nv]
    # sum over a cell's edges of +-h: a constant-divergence field has zero net flux
    assert np.allclose(B.sum(axis=1), 0)
    x = np.linalg.solve(A, s.rhs)
    p = x[s.nv:].reshape(16, 16)
    # div grad p = -1 on [-1, 1]^2 with p = 0 on the boundary: max p = 0.2947 at the centre (cell means slightly lower)
    assert 0.27 < p.max() < 0.2947 and p.min() > 0
    assert np.allclose(p, p.T, atol=1e-12) and np.allclose(p, p[::-1, :], atol=1e-12)
