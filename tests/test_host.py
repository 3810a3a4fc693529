"""Host-side mirror of the reference API: argument checks that raise before any
device call (IllegalArgumentException as in the Java code), no GPU needed."""
import numpy as np
import pytest

from jfem_b200 import IllegalArgumentException, IterativeSolver, SparseMatrix
from jfem_b200.linalg import DenseMatrix


def test_add_bounds():
    m = SparseMatrix(3, 4)
    with pytest.raises(IllegalArgumentException):
        m.add(1.0, 3, 0)
    with pytest.raises(IllegalArgumentException):
        m.add(1.0, 0, 4)


def test_add_skips_zero_and_keeps_duplicates():
    m = SparseMatrix(2, 2)
    m.add(0.0, 0, 0)
    m.add(1.0, 0, 1)
    m.add(2.0, 0, 1)
    assert m.getSparseEntryCount() == 2
    assert m.at(0, 1) == 3.0
    m.set(5.0, 0, 1)           # appends 5 - 3
    assert m.at(0, 1) == 5.0


def test_mvmul_size_check():
    m = SparseMatrix.identity(4)
    with pytest.raises(IllegalArgumentException):
        m.mvMul(np.ones(3))
    with pytest.raises(IllegalArgumentException):
        m.tvMul(np.ones(5))


def test_coo_bounds():
    with pytest.raises(IllegalArgumentException):
        SparseMatrix.from_coo(2, 2, [0, 2], [0, 0], [1.0, 1.0])


def test_square_from_values():
    with pytest.raises(IllegalArgumentException):
        DenseMatrix.squareMatrixFromValues(1, 2, 3)


def test_start_vectors():
    s = IterativeSolver()
    x = s._start(5)
    assert x.tolist() == [1, 0, 0, 0, 0]          # iterate.set(1, 0)
    assert s._start(3, zero=True).tolist() == [0, 0, 0]
    s.lastSolution = np.arange(3.0)
    assert s._start(3).tolist() == [0, 1, 2]      # warm start


def test_block_sparse_matrix_partition_and_checks():
    """BlockSparseMatrix: the partition comes from the diagonal blocks; blocks
    off the partition or of the wrong shape are rejected (no device needed)."""
    import numpy as np
    import pytest
    from jfem_b200.linalg import IllegalArgumentException
    from jfem_b200.schur import BlockSparseMatrix
    blocks = {(0, 0): np.eye(4), (4, 4): 2 * np.eye(3), (0, 4): np.ones((4, 3)), (4, 0): np.ones((3, 4))}
    B = BlockSparseMatrix(blocks, 7)
    assert list(B.getBlockStarts()) == [0, 4] and list(B.getBlockEnds()) == [4, 7]
    parts = BlockSparseMatrix.partitionVector(np.arange(7.0), B.getBlockStarts(), B.getBlockEnds())
    assert [list(p) for p in parts] == [[0, 1, 2, 3], [4, 5, 6]]
    with pytest.raises(IllegalArgumentException):
        BlockSparseMatrix({(0, 0): np.eye(4), (4, 4): np.eye(2)}, 7)
    with pytest.raises(IllegalArgumentException):
        BlockSparseMatrix({(0, 0): np.eye(4), (4, 4): np.eye(3), (0, 4): np.ones((4, 2))}, 7)
    with pytest.raises(IllegalArgumentException):
        BlockSparseMatrix({(0, 0): np.eye(4), (4, 4): np.eye(3), (0, 2): np.ones((4, 3))}, 7)
