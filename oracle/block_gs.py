"""numpy restatement of multigrid/BlockGaussseidelSmoother.java (test
infrastructure: the oracle the GPU block Gauss-Seidel smoother is checked
against).

A block matrix is given as a dict {(i, j): dense block} over a partition of
the unknowns into consecutive ranges starts[i] .. ends[i].  The smoother
(BlockGaussseidelSmoother.java:33-66), omega = 1:

    for each run:
        subRhs_i = (rhs - U x)_i              U: the blocks (i, j) with i < j
        x = 0
        for i in block order:
            t = subRhs_i - sum_{j < i} L_ij subRet_j    (L: the blocks with i > j)
            subRet_i = D_i^-1 t                 D_i^-1: dense inverse of block (i, i)
            x_i += subRet_i

The diagonal inverses are those of BlockSparseMatrix.getInvertedDiagonalMatrix
(BlockSparseMatrix.java:194-220): a block that cannot be inverted is replaced
by the identity.
"""
import numpy as np


def inverted_diagonal(blocks, nblocks):
    inv = []
    for i in range(nblocks):
        d = blocks[(i, i)]
        try:
            inv.append(np.linalg.inv(d))
        except np.linalg.LinAlgError:
            inv.append(np.eye(d.shape[0]))
    return inv


def block_gauss_seidel(blocks, starts, ends, rhs, iterate, runs, omega=1.0):
    nb = len(starts)
    dinv = inverted_diagonal(blocks, nb)
    x = np.array(iterate, dtype=np.float64)
    rhs = np.asarray(rhs, dtype=np.float64)
    for _ in range(runs):
        ux = np.zeros_like(x)
        for (i, j), blk in blocks.items():
            if i < j:
                ux[starts[i]:ends[i]] += blk @ x[starts[j]:ends[j]]
        sub = rhs - ux * omega
        x = np.zeros_like(x)
        ret = []
        for i in range(nb):
            t = sub[starts[i]:ends[i]].copy()
            for j in range(i):
                if (i, j) in blocks:
                    t -= (blocks[(i, j)] @ ret[j]) * omega
            ret.append(dinv[i] @ t)
            x[starts[i]:ends[i]] += ret[i]
    return x
