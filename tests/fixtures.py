"""Shared fixtures: the seeded matrices of the reference's tests and small
finite-element systems, built on the CPU."""
import json
import os

import numpy as np

import oracle as O
from jfem_b200 import problems
from jfem_b200.assembly import Space, assemble, prolongation

HERE = os.path.dirname(os.path.abspath(__file__))


def kat():
    with open(os.path.join(HERE, "golden", "kat.json")) as f:
        return json.load(f)


def java_sparse(rows, cols, seed, density, integer=False):
    """SparseMvMulTest.createTiny/Small/LargeSparseMatrix (SparseMvMulTest.java:12-49):
    loops over the shape range (last index fastest), draws nextDouble() < density,
    then a value ((int)(10*u - 5) or u - 0.4) from the same generator."""
    n = rows * cols
    # at most two draws per position; draw enough and consume sequentially
    u = O.java_random_doubles(seed, 2 * n)
    ri, ci, v = [], [], []
    k = 0
    for r in range(rows):
        for c in range(cols):
            d = u[k]
            k += 1
            if d < density:
                w = u[k]
                k += 1
                val = float(int(10 * w - 5)) if integer else w - 0.4
                if val != 0:
                    ri.append(r)
                    ci.append(c)
                    v.append(val)
    return np.array(ri, np.int32), np.array(ci, np.int32), np.array(v)


def java_vector(n, seed, integer=False):
    u = O.java_random_doubles(seed, n)
    return np.trunc(10 * u - 5) if integer else u - 0.4


def fe_system(p=1, cells=16, mass=5.0, modes=4, seed=0):
    sp, sy = problems.poisson(p, cells, mass, modes, seed)
    return sp, sy


def coo_oracle(sy):
    return O.CooMatrix(sy.n, sy.n, sy.rows, sy.cols, sy.vals)


def mg_levels(p, coarse, L, mass=5.0, modes=4, seed=0):
    return problems.hierarchy(p, coarse, L, mass, modes, seed)


def schwarz_test_matrix(n):
    """CartesianSchwarzTest.createSparseMatrix (CartesianSchwarzTest.java:20-33):
    over the n x n shape range a draw < 0.4 adds (int)(10 u - 5), every
    diagonal entry gets 15, and the result is A + A^T (dense float64)."""
    u = O.java_random_doubles(14239078, 2 * n * n)
    a = np.zeros((n, n))
    k = 0
    for r in range(n):
        for c in range(n):
            d = u[k]
            k += 1
            if d < 0.4:
                a[r, c] += float(int(10 * u[k] - 5))
                k += 1
            if r == c:
                a[r, c] += 15.0
    return a + a.T
