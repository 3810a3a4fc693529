"""Schur-complement block solvers (the inner solves of JFEM's DLM solvers) on
the GPU.

Reference: linalg/BlockSparseMatrix.java, linalg/AbstractSchurSolver.java,
linalg/ExplicitSchurSolver.java, linalg/IterativeExplicitSchur.java,
linalg/DirectSchur.java, linalg/RichardsonExplicitSchur.java.

A block matrix with the Schur block A00 in the top left corner, diagonal blocks
D_i, top blocks T_i = block(0, i) and left blocks L_i = block(i, 0):

    [ A00  T_1 ... T_k ] [u0]   [f0]
    [ L_1  D_1         ] [u1] = [f1]
    [ ...       ...    ] [..]   [..]
    [ L_k          D_k ] [uk]   [fk]

is solved by block elimination (AbstractSchurSolver.mvMul, lines 104-134):
f0' = f0 - sum_i T_i D_i^-1 f_i, u0 = S^-1 f0' with S = A00 - sum_i T_i D_i^-1 L_i,
u_i = D_i^-1 f_i - D_i^-1 L_i u0.  The diagonal inverses are dense
(AbstractSchurSolver.java:28-46 inverts each D_i once) and computed by the
device LU (jfg_dense_inverse); the explicit Schur complement
(ExplicitSchurSolver.java:15-29) is formed by the device sparse products
(jfg_matrix_mmmul: T_i D_i^-1, then times L_i) and one device COO merge; every
product with a block or an inverse is a device SpMV.  The Schur system is
solved by the subclass: preconditioned GMRES with the dense inverse of A00 as
the preconditioner to 1e-9 (IterativeExplicitSchur), the dense inverse of S
(DirectSchur) or a preconditioned Richardson iteration to 1e-7
(RichardsonExplicitSchur).
"""
from __future__ import annotations

import numpy as np

from . import _native as N
import ctypes as C

from .linalg import (DenseMatrix, DeviceMatrix, IllegalArgumentException, IterativeSolver, SolveResult,
                     SparseMatrix, VectorMultiplyable)

__all__ = ["BlockSparseMatrix", "AbstractSchurSolver", "ExplicitSchurSolver", "IterativeExplicitSchur",
           "DirectSchur", "RichardsonExplicitSchur", "ImplicitSchurSolver", "IterativeImplicitSchur",
           "SchurOperator", "BlockGaussSeidelSmoother"]


def _coo_of(block):
    """(rows, cols, vals, shape) of a block given as a SparseMatrix, a
    DeviceMatrix, a dense array or a (rows, cols, vals, shape) tuple."""
    if isinstance(block, SparseMatrix):
        r, c, v = block.coo()
        return np.asarray(r), np.asarray(c), np.asarray(v, dtype=np.float64), (block.getRows(), block.getCols())
    if isinstance(block, DeviceMatrix):
        r, c, v = block.coo()
        return np.asarray(r), np.asarray(c), np.asarray(v, dtype=np.float64), (block.rows, block.cols)
    if isinstance(block, tuple) and len(block) == 4:
        r, c, v, shape = block
        return np.asarray(r), np.asarray(c), np.asarray(v, dtype=np.float64), tuple(shape)
    a = np.asarray(block, dtype=np.float64)
    if a.ndim != 2:
        raise IllegalArgumentException("a block must be a matrix")
    r, c = np.nonzero(a)
    return r, c, a[r, c], a.shape


class BlockSparseMatrix(VectorMultiplyable):
    """linalg/BlockSparseMatrix.java: sparse blocks keyed by the (row, column)
    of their top left entry; the block partition is given by the diagonal
    blocks (BlockSparseMatrix.java:75-117)."""

    def __init__(self, blocks: dict, rows: int, cols: int | None = None, ctx: N.Context | None = None):
        cols = rows if cols is None else cols
        if rows != cols:
            raise IllegalArgumentException("block matrices must be square")
        self._ctx = ctx
        self._coo = {}
        for key, blk in blocks.items():
            y, x = int(key[0]), int(key[1])
            self._coo[(y, x)] = _coo_of(blk)
        starts = sorted(y for (y, x) in self._coo if y == x)
        if not starts or starts[0] != 0:
            raise IllegalArgumentException("the diagonal blocks must start at 0")
        ends = starts[1:] + [rows]
        for s, e in zip(starts, ends):
            if self._coo[(s, s)][3] != (e - s, e - s):
                raise IllegalArgumentException("diagonal blocks do not tile the matrix")
        self.blockStarts = np.array(starts, dtype=np.int64)
        self.blockEnds = np.array(ends, dtype=np.int64)
        for (y, x), (_, _, _, shape) in self._coo.items():
            if y not in starts or x not in starts:
                raise IllegalArgumentException("a block does not start on the block partition")
            iy, ix = starts.index(y), starts.index(x)
            if shape != (ends[iy] - y, ends[ix] - x):
                raise IllegalArgumentException("block has the wrong shape")
        self.rows = rows
        self._dev = {}

    @property
    def ctx(self) -> N.Context:
        if self._ctx is None:
            self._ctx = N.default_context()
        return self._ctx

    def getBlockStarts(self):
        return self.blockStarts.copy()

    def getBlockEnds(self):
        return self.blockEnds.copy()

    def getBlockSizes(self):
        return self.blockEnds - self.blockStarts

    def getVectorSize(self):
        return self.rows

    def getTVectorSize(self):
        return self.rows

    def hasBlock(self, y: int, x: int) -> bool:
        return (int(y), int(x)) in self._coo

    def getBlockCoo(self, y: int, x: int):
        return self._coo[(int(y), int(x))]

    def getBlock(self, y: int, x: int) -> DeviceMatrix | None:
        """The block whose top left entry is (y, x) as a device matrix (None if absent)."""
        key = (int(y), int(x))
        if key not in self._coo:
            return None
        if key not in self._dev:
            r, c, v, (nr, nc) = self._coo[key]
            self._dev[key] = DeviceMatrix(nr, nc, r, c, v, self.ctx)
        return self._dev[key]

    def getBlockMatrix(self, i: int, j: int) -> DeviceMatrix | None:
        """Block number (i, j) of the partition (getBlockMatrix(int...), line 29)."""
        return self.getBlock(self.blockStarts[i], self.blockStarts[j])

    @staticmethod
    def partitionVector(vector, starts, ends):
        """BlockSparseMatrix.partitionVector (line 411): the sub-vectors of the blocks."""
        v = N.f64(vector)
        return [v[int(s):int(e)].copy() for s, e in zip(starts, ends)]

    def mvMul(self, vector):
        v = N.f64(vector)
        if v.shape != (self.rows,):
            raise IllegalArgumentException("Vectors are of different size")
        out = np.zeros(self.rows)
        for (y, x) in sorted(self._coo):
            blk = self.getBlock(y, x)
            out[y:y + blk.rows] += blk.spmv(v[x:x + blk.cols])
        return out


class AbstractSchurSolver(VectorMultiplyable):
    """linalg/AbstractSchurSolver.java: block elimination around a Schur
    solve; a VectorMultiplyable whose mvMul applies the inverse of the block
    matrix."""

    def __init__(self, blockMatrix: BlockSparseMatrix):
        self.blockMatrix = blockMatrix
        self.ctx = blockMatrix.ctx
        self.blockStarts = blockMatrix.getBlockStarts()
        self.blockEnds = blockMatrix.getBlockEnds()
        self.blockSizes = blockMatrix.getBlockSizes()
        self.diagonalInverses = []            # dense numpy inverses D_i^-1
        self._dinv_dev = []                   # the same as device matrices
        for i in range(1, len(self.blockStarts)):
            s = int(self.blockStarts[i])
            if not blockMatrix.hasBlock(s, s):
                raise IllegalArgumentException("matrix does not contain necessary diagonal block")
            r, c, v, (m, _) = blockMatrix.getBlockCoo(s, s)
            d = np.zeros((m, m))
            np.add.at(d, (r, c), v)
            inv = DenseMatrix(d, self.ctx).inverse()          # device LU (jfg_dense_inverse)
            if not blockMatrix.hasBlock(0, s):
                raise IllegalArgumentException("matrix does not contain necessary top block")
            if not blockMatrix.hasBlock(s, 0):
                raise IllegalArgumentException("matrix does not contain necessary left block")
            self.diagonalInverses.append(inv)
            ri, ci = np.nonzero(inv)
            self._dinv_dev.append(DeviceMatrix(m, m, ri, ci, inv[ri, ci], self.ctx))

    def getBlockSize(self):
        return len(self.diagonalInverses) + 1

    def getDiagonalBlock(self, i) -> DeviceMatrix:
        s = self.blockStarts[i + 1]
        return self.blockMatrix.getBlock(s, s)

    def getDiagonalInverse(self, i) -> np.ndarray:
        return self.diagonalInverses[i]

    def getTopBlock(self, i) -> DeviceMatrix:
        return self.blockMatrix.getBlock(0, self.blockStarts[i + 1])

    def getLeftBlock(self, i) -> DeviceMatrix:
        return self.blockMatrix.getBlock(self.blockStarts[i + 1], 0)

    def getSchurBlock(self) -> DeviceMatrix:
        return self.blockMatrix.getBlockMatrix(0, 0)

    def schurMvMul(self):
        raise NotImplementedError

    def solveSchur(self, A, b):
        raise NotImplementedError

    def getVectorSize(self):
        return self.blockMatrix.getVectorSize()

    def getTVectorSize(self):
        return self.blockMatrix.getTVectorSize()

    def mvMul(self, vector):
        """AbstractSchurSolver.mvMul (lines 104-134)."""
        v = N.f64(vector)
        if v.shape != (self.getVectorSize(),):
            raise IllegalArgumentException("Vectors are of different size")
        sub = BlockSparseMatrix.partitionVector(v, self.blockStarts, self.blockEnds)
        schur_vector = sub.pop(0)
        solved = [self._dinv_dev[i].spmv(sub[i]) for i in range(len(sub))]
        for i in range(len(sub)):
            schur_vector = schur_vector - self.getTopBlock(i).spmv(solved[i])
        u0 = N.f64(self.solveSchur(self.schurMvMul(), schur_vector))
        ret = np.zeros(self.getVectorSize())
        ret[:u0.size] = u0
        for i in range(len(sub)):
            ui = solved[i] - self._dinv_dev[i].spmv(self.getLeftBlock(i).spmv(u0))
            ret[int(self.blockStarts[i + 1]):int(self.blockEnds[i + 1])] = ui
        return ret

    def tvMul(self, vector):
        raise NotImplementedError("not implemented yet")


class ExplicitSchurSolver(AbstractSchurSolver):
    """linalg/ExplicitSchurSolver.java: the Schur complement
    S = A00 - sum_i T_i D_i^-1 L_i formed once, on the device."""

    def __init__(self, blockMatrix: BlockSparseMatrix):
        super().__init__(blockMatrix)
        self.schurComplement = self._form()

    def _form(self) -> DeviceMatrix:
        n0 = int(self.blockSizes[0])
        rows, cols, vals = [], [], []
        for i in range(len(self.diagonalInverses)):
            # getTopBlock(i).mmMul(new SparseMatrix(D_i^-1)).mmMul(getLeftBlock(i)) (lines 16-22)
            prod = self.getTopBlock(i).mmMul(self._dinv_dev[i]).mmMul(self.getLeftBlock(i))
            r, c, v = prod.coo()
            rows.append(np.asarray(r))
            cols.append(np.asarray(c))
            vals.append(-np.asarray(v, dtype=np.float64))     # mulInPlace(-1)
        r, c, v, _ = self.blockMatrix.getBlockCoo(0, 0)         # addInPlace(getSchurBlock())
        rows.append(np.asarray(r))
        cols.append(np.asarray(c))
        vals.append(np.asarray(v, dtype=np.float64))
        return DeviceMatrix(n0, n0, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), self.ctx)

    def resetOffDiagonals(self, systemMatrix: BlockSparseMatrix):
        """ExplicitSchurSolver.resetOffDiagonals: new off-diagonal blocks, the
        diagonal inverses are kept."""
        self.blockMatrix = systemMatrix
        self.schurComplement = self._form()

    def getSchurComplement(self) -> DeviceMatrix:
        return self.schurComplement

    def schurMvMul(self):
        return self.schurComplement


class IterativeExplicitSchur(ExplicitSchurSolver):
    """linalg/IterativeExplicitSchur.java: PGMRES on S with the dense inverse
    of A00 as the preconditioner, tolerance 1e-9."""

    def __init__(self, blockMatrix: BlockSparseMatrix):
        super().__init__(blockMatrix)
        r, c, v, (n0, _) = blockMatrix.getBlockCoo(0, 0)
        a = np.zeros((n0, n0))
        np.add.at(a, (r, c), v)
        inv = DenseMatrix(a, self.ctx).inverse()
        ri, ci = np.nonzero(inv)
        self.firstInverse = DeviceMatrix(n0, n0, ri, ci, inv[ri, ci], self.ctx)
        self.it = IterativeSolver(ctx=self.ctx)

    def solveSchur(self, A, b):
        return self.it.solvePGMRES(A, self.firstInverse, b, 1e-9)


class DirectSchur(ExplicitSchurSolver):
    """linalg/DirectSchur.java: the dense inverse of S, computed on first use."""

    def __init__(self, blockMatrix: BlockSparseMatrix):
        super().__init__(blockMatrix)
        self.inverse = None

    def solveSchur(self, A, b):
        if self.inverse is None:
            r, c, v = A.coo()
            n0 = A.rows
            a = np.zeros((n0, n0))
            np.add.at(a, (np.asarray(r), np.asarray(c)), np.asarray(v))
            inv = DenseMatrix(a, self.ctx).inverse()
            ri, ci = np.nonzero(inv)
            self.inverse = DeviceMatrix(n0, n0, ri, ci, inv[ri, ci], self.ctx)
        return self.inverse.spmv(b)


class RichardsonExplicitSchur(ExplicitSchurSolver):
    """linalg/RichardsonExplicitSchur.java: x += P (b - S x) until
    ||b - S x|| <= 1e-7.  The reference loops without bound; here the loop
    stops after maxit steps with ArithmeticError."""

    def __init__(self, blockMatrix: BlockSparseMatrix, maxit: int = 100000):
        super().__init__(blockMatrix)
        self.preconditioner = None
        self.maxit = maxit

    def solveSchur(self, A, b):
        if self.preconditioner is None:
            raise IllegalArgumentException("RichardsonExplicitSchur needs a preconditioner")
        b = N.f64(b)
        x = np.zeros_like(b)
        r = b - A.spmv(x)
        k = 0
        while np.linalg.norm(r) > 1e-7:
            if k >= self.maxit:
                raise ArithmeticError("Richardson iteration on the Schur complement did not converge")
            x = x + N.f64(self.preconditioner.mvMul(r))
            r = b - A.spmv(x)
            k += 1
        self.iterations = k
        return x


class SchurOperator(VectorMultiplyable):
    """The implicit Schur complement S v = A00 v - sum_i T_i D_i^-1 L_i v as a
    composed device operator (libjfem_gpu's jfg_schur): the VectorMultiplyable
    that ImplicitSchurSolver.schurMvMul returns
    (linalg/ImplicitSchurSolver.java:17-57); S is never formed."""

    def __init__(self, solver: "AbstractSchurSolver"):
        self.ctx = solver.ctx
        self._keep = (solver.getSchurBlock(), [solver.getTopBlock(i) for i in range(len(solver._dinv_dev))],
                      list(solver._dinv_dev), [solver.getLeftBlock(i) for i in range(len(solver._dinv_dev))])
        A00, T, D, L = self._keep
        k = len(D)
        arr = lambda ms: (C.c_void_p * max(k, 1))(*([m.handle for m in ms] + ([None] if k == 0 else [])))
        h = C.c_void_p()
        st = N.load().jfg_schur_create(self.ctx.handle, A00.handle, k, arr(T), arr(D), arr(L), C.byref(h))
        if st == N.ERR_BAD_ARG:
            raise IllegalArgumentException(N.load().jfg_last_error(self.ctx.handle).decode())
        self.ctx.check(st)
        self._h = h
        self.n = A00.rows

    @property
    def handle(self):
        return self._h

    def getVectorSize(self):
        return self.n

    def getTVectorSize(self):
        return self.n

    def mvMul(self, vector):
        v = N.f64(vector)
        if v.shape != (self.n,):
            raise IllegalArgumentException("Vectors are of different size")
        out = np.empty(self.n)
        self.ctx.check(N.load().jfg_schur_apply(self._h, N.dptr(v), N.dptr(out)))
        return out

    def tvMul(self, vector):
        raise NotImplementedError("not implemented yet")   # ImplicitSchurSolver.java:53-56

    def solvePGMRES(self, preconditioner: DeviceMatrix, rhs, tol, it: IterativeSolver | None = None):
        """IterativeSolver.solvePGMRES on S from zero (GMRES.java:59-60), on the GPU."""
        b = N.f64(rhs)
        if b.shape != (self.n,):
            raise IllegalArgumentException("Vectors are of different size")
        x = np.zeros(self.n)
        it = it or IterativeSolver(ctx=self.ctx)
        opts = N.SolverOpts()
        N.load().jfg_solver_opts_default(C.byref(opts))
        opts.tol = tol
        opts.restart = it.gm.ITERATIONS_BEFORE_RESTART
        opts.max_restarts = it.gm.MAX_RESTARTS
        hist = np.zeros(max(it.history_cap, 1))
        opts.h_history = N.dptr(hist)
        opts.history_cap = it.history_cap
        info = N.SolveInfo()
        st = N.load().jfg_schur_solve(self._h, N.PGMRES, N.PREC_MATRIX, preconditioner.handle, N.dptr(b), N.dptr(x),
                                      C.byref(opts), C.byref(info))
        self.ctx.check(st, allow=(N.OK, N.NOT_CONVERGED, N.NONFINITE))
        it.last = SolveResult(info, hist)
        it.iterations = info.iterations
        it.lastSolution = x
        return x

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_schur_free(self._h)
        except Exception:
            pass


class ImplicitSchurSolver(AbstractSchurSolver):
    """linalg/ImplicitSchurSolver.java: the Schur system is solved through
    the composed operator S v = A00 v - sum_i T_i D_i^-1 L_i v without forming
    S (schurMvMul, lines 17-57)."""

    def __init__(self, blockMatrix: BlockSparseMatrix):
        super().__init__(blockMatrix)
        self._op = None

    def schurMvMul(self) -> SchurOperator:
        if self._op is None:
            self._op = SchurOperator(self)
        return self._op


class IterativeImplicitSchur(ImplicitSchurSolver):
    """linalg/IterativeImplicitSchur.java: PGMRES on the implicit Schur
    operator, preconditioned by the dense inverse of A00, to 1e-9."""

    def __init__(self, blockMatrix: BlockSparseMatrix):
        super().__init__(blockMatrix)
        r, c, v, (n0, _) = blockMatrix.getBlockCoo(0, 0)
        a = np.zeros((n0, n0))
        np.add.at(a, (r, c), v)
        inv = DenseMatrix(a, self.ctx).inverse()              # firstInverse (lines 12-14), device LU
        ri, ci = np.nonzero(inv)
        self.firstInverse = DeviceMatrix(n0, n0, ri, ci, inv[ri, ci], self.ctx)
        self.it = IterativeSolver(ctx=self.ctx)

    def solveSchur(self, A, b):
        return A.solvePGMRES(self.firstInverse, b, 1e-9, self.it)


class BlockGaussSeidelSmoother:
    """multigrid/BlockGaussseidelSmoother.java: block Gauss-Seidel over the
    partition of a BlockSparseMatrix, omega = 1.  Each run (lines 33-66):
    the strictly upper blocks applied to the iterate, then the blocks in
    order, block i solved with the dense inverse of its diagonal block after
    subtracting the strictly lower blocks times the blocks already solved.
    The diagonal inverses come from the device LU (jfg_dense_inverse), an
    uninvertible block is replaced by the identity as in
    BlockSparseMatrix.getInvertedDiagonalMatrix (BlockSparseMatrix.java:194-220);
    every block product is a device SpMV."""

    omega = 1.0

    def __init__(self, blockMatrix: BlockSparseMatrix, runs: int):
        from .linalg import SingularMatrixException
        self.runs = int(runs)
        self.blockMatrix = blockMatrix
        self.ctx = blockMatrix.ctx
        self.starts = blockMatrix.getBlockStarts()
        self.ends = blockMatrix.getBlockEnds()
        nb = len(self.starts)
        self._dinv = []
        for i in range(nb):
            r, c, v, (m, _) = blockMatrix.getBlockCoo(self.starts[i], self.starts[i])
            d = np.zeros((m, m))
            np.add.at(d, (r, c), v)
            try:
                inv = DenseMatrix(d, self.ctx).inverse()
            except SingularMatrixException:
                inv = np.eye(m)
            ri, ci = np.nonzero(inv)
            self._dinv.append(DeviceMatrix(m, m, ri, ci, inv[ri, ci], self.ctx))
        # block (i, j) of the partition for every stored block off the diagonal
        self._upper, self._lower = [], {}
        for i in range(nb):
            for j in range(nb):
                if i != j and blockMatrix.hasBlock(self.starts[i], self.starts[j]):
                    if i < j:
                        self._upper.append((i, j))
                    else:
                        self._lower.setdefault(i, []).append(j)

    def smooth(self, operator, rhs, iterate, verbose: bool = False, prefix: str = ""):
        b = N.f64(rhs)
        x = N.f64(iterate).copy()
        n = self.blockMatrix.getVectorSize()
        if b.shape != (n,) or x.shape != (n,):
            raise IllegalArgumentException("Vectors are of different size")
        bm, st, en = self.blockMatrix, self.starts, self.ends
        if verbose:
            print(prefix + " " + str(np.linalg.norm(operator.mvMul(x) - b)))
        for _ in range(self.runs):
            ux = np.zeros(n)
            for (i, j) in self._upper:
                ux[st[i]:en[i]] += bm.getBlockMatrix(i, j).spmv(x[st[j]:en[j]])
            sub = b - ux * self.omega
            x = np.zeros(n)
            ret = []
            for i in range(len(st)):
                t = sub[st[i]:en[i]].copy()
                for j in sorted(self._lower.get(i, [])):
                    t -= bm.getBlockMatrix(i, j).spmv(ret[j]) * self.omega
                ret.append(self._dinv[i].spmv(t))
                x[st[i]:en[i]] += ret[i]
            if verbose:
                print(prefix + " " + str(np.linalg.norm(operator.mvMul(x) - b)))
        return x
