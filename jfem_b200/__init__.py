"""jfem_b200 -- B200 (sm_100a) implementation of JFEM's linear-solve path.

The compute lives in ``libjfem_gpu.so`` (hand-written CUDA behind the C ABI of
``include/jfem_gpu.h``); this package is the host-side mirror of the
reference's Java solver API (``linalg``, ``multigrid``) plus the structured
grid assembler that produces the systems (``assembly``, ``problems``).
"""
from . import _native
from .linalg import (DenseMatrix, DeviceMatrix, GMRES, IllegalArgumentException, IterativeSolver,
                     SingularMatrixException, SparseMatrix, VectorMultiplyable)
from .multigrid import (ForwardBackwardGaussSeidelSmoother, GaussSeidelSmoother, JacobiSmoother,
                        MGPreconditioner, RichardsonSmoother)
from .schur import (BlockSparseMatrix, DirectSchur, ExplicitSchurSolver, ImplicitSchurSolver,
                    IterativeExplicitSchur, IterativeImplicitSchur, RichardsonExplicitSchur)

__all__ = ["DenseMatrix", "DeviceMatrix", "GMRES", "IllegalArgumentException", "IterativeSolver",
           "SingularMatrixException", "SparseMatrix", "VectorMultiplyable", "JacobiSmoother",
           "MGPreconditioner", "RichardsonSmoother", "ForwardBackwardGaussSeidelSmoother", "GaussSeidelSmoother",
           "BlockSparseMatrix", "ExplicitSchurSolver", "IterativeExplicitSchur", "DirectSchur",
           "RichardsonExplicitSchur", "ImplicitSchurSolver", "IterativeImplicitSchur"]
