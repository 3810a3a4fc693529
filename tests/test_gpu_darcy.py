"""Raviart-Thomas mixed Darcy systems (the saddle-point systems MixedRTSpace
produces; Examples/src/RTDarcy.java:76-77 solves them with unpreconditioned
GMRES to 1e-10) through jfg_solve on the GPU, against the oracle's GMRES
(linalg/GMRES.java:40-251) on the same system."""
import numpy as np
import pytest

import oracle as O
from jfem_b200 import IterativeSolver
from jfem_b200 import _native as N
from jfem_b200.darcy import rt0_darcy
from jfem_b200.linalg import DeviceMatrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cells", [(8, 8), (24, 16)])
def test_rt_darcy_gmres_vs_oracle(ctx, cells):
    s = rt0_darcy(*cells)
    A_o = O.CooMatrix(s.n, s.n, s.rows, s.cols, s.vals)
    tol = 1e-10                                     # RTDarcy.java:77, absolute
    ref = O.solve_gmres(A_o, s.rhs, tol)
    A = DeviceMatrix(s.n, s.n, s.rows, s.cols, s.vals, ctx)
    it = IterativeSolver(ctx=ctx)
    x = it.solveGMRES(A, s.rhs, tol)
    assert ref.status == O.OK and it.last.status == N.OK
    # FMA and summation order differ from the oracle's loops; unpreconditioned
    # GMRES on the indefinite saddle-point system amplifies them over its
    # hundred-odd iterations: the count may move by a few (96 vs 98 measured
    # on 8 x 8 cells)
    assert abs(it.iterations - ref.iterations) <= max(4, ref.iterations // 100)
    assert abs(it.last.restarts - ref.restarts) <= 1
    assert np.linalg.norm(s.rhs - A_o.mvmul(x)) <= tol
    assert np.linalg.norm(x - ref.x) / np.linalg.norm(ref.x) < 1e-8
    # the pressure block of the solution solves div grad p = -1 (cell means below the continuous maximum 0.2947)
    p = x[s.nv:]
    assert p.min() > 0 and p.max() < 0.2947
