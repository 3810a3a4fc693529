/*
 * jfem_gpu.h -- C ABI of the B200 (sm_100a) linear-solve library for JFEM.
 *
 * The library replaces the Java/JNI layer under JFEM's solver API.  Every
 * entry point below names the reference interface it stands in for
 * (paths relative to the JFEM project root).  Conventions:
 *   - plain C types only; opaque handles; every call returns a jfg_status;
 *   - host pointers ("h_") are copied in/out inside the call; device pointers
 *     ("d_") must be device memory of the context's GPU;
 *   - the caller owns host buffers, the library owns device buffers;
 *   - a context owns one CUDA stream; one context per host thread.
 * Index arrays follow JFEM's COO naming: `rows` are the row indices
 * (SparseMatrix.sparseYs) and `cols` the column indices (sparseXs).
 */
#ifndef JFEM_GPU_H
#define JFEM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    JFG_OK = 0,
    JFG_NOT_CONVERGED = 1,   /* iteration cap hit; x holds the last iterate */
    JFG_BREAKDOWN = 2,       /* BiCGStab rho ~ 0 (after the GMRES fallback converged, see jfg_solve) */
    JFG_NONFINITE = 3,       /* NaN/Inf met in a reduction */
    JFG_ERR_BAD_ARG = 4,
    JFG_ERR_SINGULAR = 5,
    JFG_ERR_CUDA = 6,
    JFG_ERR_NO_DEVICE = 7,
    JFG_ERR_UNSUPPORTED = 8
} jfg_status;

typedef struct jfg_ctx jfg_ctx;
typedef struct jfg_mat jfg_mat;
typedef struct jfg_mg jfg_mg;

/* ---- context --------------------------------------------------------- */
/* Creates a context (one CUDA stream) on `device`. */
int jfg_create(int device, jfg_ctx** out);
int jfg_destroy(jfg_ctx* ctx);
/* Message of the last failing call on this context ("" if none). */
const char* jfg_last_error(jfg_ctx* ctx);
/* Waits for all work queued on the context's stream. */
int jfg_synchronize(jfg_ctx* ctx);
/* Frees the grow-only scratch the sparse products keep in the context (up to
 * ~70 bytes per product of the largest row chunk, i.e. a few GB after a
 * Galerkin product of a 1 M-row matrix).  Not part of the reference surface. */
int jfg_release_scratch(jfg_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for callers that time or order work. */
void* jfg_stream(jfg_ctx* ctx);
/* Library version string. */
const char* jfg_version(void);
/* Kernels this process has launched through the library, counting each
 * executed kernel node of a replayed CUDA graph.  Measurement helper with no
 * counterpart in the reference. */
int jfg_kernel_launches(uint64_t* count);

/* ---- sparse matrices ------------------------------------------------- */
/* Builds a device matrix from COO triples in any order with duplicates,
 * summing duplicates (the merge of SparseMatrix.getCoordinateEntryList,
 * Core/src/main/java/linalg/SparseMatrix.java:196-225) and dropping entries
 * that are exactly zero (e.g. Dirichlet rows zeroed in place,
 * Core/src/main/java/basic/AcceptsMatrixBoundaryValues.java:39-40).
 * Replaces: new SparseMatrix(rows, cols) + add(...) (SparseMatrix.java:274-294). */
int jfg_matrix_from_coo(jfg_ctx* ctx, int n_rows, int n_cols, int64_t nnz, const int* h_rows,
                        const int* h_cols, const double* h_vals, jfg_mat** out);
int jfg_matrix_free(jfg_mat* m);
/* Dimensions and merged nonzero count. */
int jfg_matrix_info(jfg_mat* m, int* n_rows, int* n_cols, int64_t* nnz);
/* y = A x.  Replaces SparseMatrix.mvMul (SparseMatrix.java:480-489) and
 * SparseMvMul.mvMul (Core/src/main/java/linalg/SparseMvMul.java:73-94). */
int jfg_spmv(jfg_mat* m, const double* h_x, double* h_y);
/* y = A^T x.  Replaces SparseMatrix.tvMul (SparseMatrix.java:492-501) and
 * SparseMvMul.tvMul (SparseMvMul.java:96-116). */
int jfg_spmv_t(jfg_mat* m, const double* h_x, double* h_y);
/* Device-pointer forms of the two products (no copies, queued on the stream). */
int jfg_spmv_dev(jfg_mat* m, const double* d_x, double* d_y);
int jfg_spmv_t_dev(jfg_mat* m, const double* d_x, double* d_y);
/* FP32 product on FP32 device vectors (values rounded to FP32 once). */
int jfg_spmv_f32_dev(jfg_mat* m, const float* d_x, float* d_y);
/* Product y = A x with FP32 vectors and sums and the matrix values read as
 * values = 0: FP32, 1: BF16, 2: FP16 scaled by a power of two (the storage
 * formats of the mixed-precision multigrid levels).  Checking and
 * measurement helper, not part of the reference surface. */
int jfg_spmv_lowp_dev(jfg_mat* m, int values, const float* d_x, float* d_y);
/* The product layout the library picked for the matrix: *stencil = 1 when
 * the rows [lo, lo + regular_rows) use the values-only 9-point layout with
 * grid stride *stride (no column indices; the other_rows rows, with
 * other_nnz entries, keep a CSR copy), 2 / 3 for the values-only layouts of
 * a Q1 prolongation / restriction that a multigrid set-up gave the matrix
 * (*stride: the stride of the grid of the rows), 0 for SELL-32 (then
 * other_rows = rows and other_nnz = nnz).  fp16_scale_inv: the factor of the
 * FP16 copy's row sums (0 before that copy exists).  Returns JFG_ERR_CUDA
 * when a staged product of this matrix found its bulk copies incomplete
 * after the bounded wait (the product's rows are then not written). */
int jfg_matrix_layout(jfg_mat* m, int* stencil, int* stride, int* regular_rows, int* other_rows,
                      int64_t* other_nnz, double* fp16_scale_inv);
/* Diagonal with duplicates summed.  Replaces Matrix.diag (Core/src/main/java/linalg/Matrix.java:157-175). */
int jfg_matrix_diag(jfg_mat* m, double* h_diag);
/* The merged CSR of the matrix (rows sorted, columns ascending within a row):
 * h_ptr[n_rows + 1], h_col[nnz], h_val[nnz] (sizes from jfg_matrix_info).
 * Replaces reading SparseMatrix.getCoordinateEntryList (SparseMatrix.java:403-417). */
int jfg_matrix_csr(jfg_mat* m, int* h_ptr, int* h_col, double* h_val);
/* Sparse products on the device; *out is a new matrix owned by the caller
 * (jfg_matrix_free).  Each entry is the sum over k of the rounded products
 * a_ik * b_kj, added from 0 in ascending k without fused multiply-adds;
 * entries whose sum is exactly zero are not stored (SparseMatrix.add skips
 * zeros, SparseMatrix.java:289).  JFG_ERR_BAD_ARG on incompatible sizes.
 *   jfg_matrix_mmmul:    C = A B    -- SparseMatrix.mmMul (SparseMatrix.java:549-593)
 *   jfg_matrix_tmmul:    C = A^T B  -- Matrix.tmMul (Core/src/main/java/linalg/Matrix.java:142-148)
 *   jfg_matrix_galerkin: C = (R A) P, or (P^T A) P when r is NULL -- the coarse
 *     systems of AMGSpace.createSystems (Core/src/main/java/multigrid/AMGSpace.java:60-78)
 *     and MGPreconditionerInterface.AMGFromMatrix
 *     (Core/src/main/java/multigrid/MGPreconditionerInterface.java:387-402), same association. */
int jfg_matrix_mmmul(jfg_mat* a, jfg_mat* b, jfg_mat** out);
int jfg_matrix_tmmul(jfg_mat* a, jfg_mat* b, jfg_mat** out);
int jfg_matrix_galerkin(jfg_mat* r, jfg_mat* a, jfg_mat* p, jfg_mat** out);
/* Times `iters` FP64 (precision 0) or FP32 (precision 1) products y = A x
 * on the context stream, each with CUDA events around the launch and the L2
 * flushed before it (a 256 MB buffer read between products, not timed); returns
 * the mean milliseconds per product.  x and y are library-owned device
 * vectors (x = 1).  Measurement helper, not part of the reference surface. */
int jfg_spmv_time(jfg_mat* m, int precision, int iters, double* ms_per_spmv);
/* Times products over `count` matrices of one context taken in turn, back to
 * back on the context stream (rounds of count products, one event pair
 * around all `iters` rounds after one untimed round); returns the mean
 * milliseconds per product.  With matrices whose bytes together exceed the
 * L2, every product reads its matrix from HBM with no flush between
 * launches.  Measurement helper, not part of the reference surface. */
int jfg_spmv_time_rotating(jfg_mat* const* ms, int count, int precision, int iters, double* ms_per_spmv);

/* ---- smoothers ------------------------------------------------------- */
typedef struct jfg_schwarz jfg_schwarz;
typedef struct jfg_gs jfg_gs;
typedef enum {
    JFG_SMOOTH_JACOBI = 0,
    JFG_SMOOTH_RICHARDSON = 1,
    JFG_SMOOTH_SCHWARZ = 2,
    JFG_SMOOTH_FBGS = 3,   /* ForwardBackwardGaussSeidelSmoother */
    JFG_SMOOTH_GS = 4      /* GaussSeidelSmoother */
} jfg_smoother_kind;
typedef struct {
    int kind;      /* jfg_smoother_kind */
    int runs;      /* sweeps (Schwarz: SubspaceCorrection.apply calls) */
    double omega;  /* damping (Jacobi / Richardson; a Schwarz handle keeps its own) */
    jfg_schwarz* schwarz;  /* JFG_SMOOTH_SCHWARZ: the decomposition of this level's matrix */
    jfg_gs* gs;            /* JFG_SMOOTH_FBGS / JFG_SMOOTH_GS: the triangular parts of this level's matrix */
} jfg_smoother_desc;
/* x <- smooth(A, rhs, x).  Replaces Smoother.smooth
 * (Core/src/main/java/multigrid/Smoother.java:15) as implemented by
 * JacobiSmoother.smooth (multigrid/JacobiSmoother.java:28-50),
 * RichardsonSmoother.smooth (multigrid/RichardsonSmoother.java:31-50),
 * SchwarzSmoother.smooth (schwarz/SchwarzSmoother.java:21-43),
 * ForwardBackwardGaussSeidelSmoother.smooth (multigrid/ForwardBackwardGaussSeidelSmoother.java:23-44:
 * runs x { x += L^-1 D U^-1 (b - A x) }, L / U the lower / upper triangles
 * with the diagonal) and GaussSeidelSmoother.smooth
 * (multigrid/GaussSeidelSmoother.java:24-32: runs x { x = (L + D)^-1 (b - R x) },
 * R the strict upper triangle). */
int jfg_smooth(jfg_mat* A, const jfg_smoother_desc* sm, const double* h_rhs, double* h_x);

/* ---- finite-element assembly on the device ---------------------------- */
/* Assembles grad_coef * GRAD_GRAD + mass_coef * VALUE_VALUE (+ a VALUE right-
 * hand side) of a Q_p Lagrange space (ContinuousTPFESpace with equidistant
 * nodes, tensorproduct/ContinuousTPFESpace.java:30-50) on a uniform cx x cy
 * grid of [x0,x1] x [y0,y1], replacing MatrixFESpace.writeCellIntegralsToMatrix
 * / writeCellIntegralsToRhs (basic/MatrixFESpace.java:29-131) with the cell
 * integrals of TPCellIntegral (tensorproduct/TPCellIntegral.java:78-159, a 5x5
 * Gauss rule) and, when dirichlet != 0, the zero-data Dirichlet treatment of
 * AcceptsMatrixBoundaryValues (basic/AcceptsMatrixBoundaryValues.java:25-44):
 * boundary rows and columns zeroed, a unit diagonal, rhs 0 on the boundary.
 *   numbering: the reference's first-appearance numbering (cells with the
 *     last coordinate fastest, local functions x-fastest);
 *   h_kappa_cells: optional per-cell factor of GRAD_GRAD (cx * cy, same cell order);
 *   h_source_qp: optional source values at the 25 Gauss points of every cell
 *     (cells x 25, x index slowest), NULL for a zero rhs;
 *   outputs: the merged matrix, h_rhs[n], h_node_of_grid[nx * ny] (dof of grid
 *     node gx * ny + gy) when not NULL, h_boundary (ascending boundary dofs,
 *     2 (nx + ny) - 4 of them) when not NULL;  n = (p cx + 1)(p cy + 1). */
typedef struct {
    int p, cx, cy;
    double x0, x1, y0, y1;
    double grad_coef, mass_coef;
    int dirichlet;
} jfg_tp_desc;
int jfg_assemble_tp(jfg_ctx* ctx, const jfg_tp_desc* d, const double* h_kappa_cells, const double* h_source_qp,
                    jfg_mat** A, double* h_rhs, int* h_node_of_grid, int* h_boundary);

/* The Taylor-Hood Q2/Q1 Stokes system on the unit square with cx x cy cells
 * (unknowns: u0 and u1 on the Q2 node grid, then p on the Q1 grid, each grid
 * numbered x-major): nu * GRAD_GRAD per velocity component and the
 * divergence blocks -B, -B^T (the lid-driven-cavity setup of the Stokes
 * configuration); velocity Dirichlet data on the whole boundary, u0 = 1 on the
 * top side when lid != 0, and the first pressure unknown fixed to 0 when
 * pin_pressure != 0, eliminated as AcceptsMatrixBoundaryValues does
 * (basic/AcceptsMatrixBoundaryValues.java:25-44: rows and columns zeroed, a
 * unit diagonal, the boundary values lifted into the rhs).
 * h_force_qp: optional body force at the 25 Gauss points of every cell
 * (2 x cells x 25: component, cell, point); outputs the matrix, h_rhs[n] and
 * the ascending velocity boundary dofs (2 (2 (vnx + vny) - 4) of them). */
int jfg_assemble_taylor_hood(jfg_ctx* ctx, int cx, int cy, double nu, const double* h_force_qp, int lid,
                             int pin_pressure, jfg_mat** A, double* h_rhs, int* h_velocity_boundary);

/* ---- Gauss-Seidel triangular parts ---------------------------------- */
/* The lower and upper triangles of a square matrix in an ordering of its
 * rows, with schedules of independent row sets for the two triangular
 * solves.  Row i of a triangular solve computes, as
 * LowerTriangularSparseMatrix / UpperTriangularSparseMatrix.solve do
 * (linalg/LowerTriangularSparseMatrix.java:173-212,
 * linalg/UpperTriangularSparseMatrix.java:185-221),
 *     sol_i = rhs_i / d_i;  sol_i += (-sol_j / d_i) * a_ij  for its entries j
 * (ascending column; the reference visits them in HashMap order).
 *   JFG_GS_NATURAL     the matrix's own row order (the reference's algorithm);
 *                      rows are grouped into dependency levels, so a solve
 *                      takes as many steps as the longest dependency chain.
 *   JFG_GS_MULTICOLOR  rows ordered colour by colour (greedy colouring of the
 *                      graph of A + A^T in row order): the same smoothers
 *                      applied to the symmetrically permuted system; one step
 *                      per colour.
 * JFG_ERR_SINGULAR when a diagonal entry is zero ("Singular Matrix"). */
typedef enum { JFG_GS_NATURAL = 0, JFG_GS_MULTICOLOR = 1 } jfg_gs_ordering;
int jfg_gs_create(jfg_ctx* ctx, jfg_mat* A, int ordering, jfg_gs** out);
int jfg_gs_free(jfg_gs* g);
/* Steps of the forward and backward solves, and colours (0 for natural). */
int jfg_gs_info(jfg_gs* g, int* forward_levels, int* backward_levels, int* colours);
/* Position of every row in the ordering (h_rank[n_rows]). */
int jfg_gs_ranks(jfg_gs* g, int* h_rank);

/* ---- overlapping Schwarz decompositions -------------------------------- */
/* Subspace corrections over patches of DOFs with cached dense patch inverses.
 * Replaces UpFrontSchwarz (schwarz/UpFrontSchwarz.java:11-81) with its
 * DirectSolver (schwarz/DirectSolver.java:12-38, inverse of R A R^T per
 * patch, RestrictionMatrix.selectFrom, schwarz/RestrictionMatrix.java:22-43)
 * and the subspace corrections
 *   JFG_SCHWARZ_MULTIPLICATIVE  MultiplicativeSubspaceCorrection (schwarz/MultiplicativeSubspaceCorrection.java:29-81)
 *   JFG_SCHWARZ_COLORED         ColoredMultiplicativeSubspaceCorrection (schwarz/ColoredMultiplicativeSubspaceCorrection.java:33-123)
 *   JFG_SCHWARZ_ADDITIVE        AdditiveSubspaceCorrection (schwarz/AdditiveSubspaceCorrection.java:22-46)
 * Patches: patch_dofs[patch_ptr[p] .. patch_ptr[p+1]) (any order; sorted
 * internally, at most 1024 DOFs).  Colours (JFG_SCHWARZ_COLORED only):
 * color_patches[color_ptr[c] .. color_ptr[c+1]).  The patch builders
 * (CartesianUpFrontSchwarz, ColoredCartesianSchwarz, VankaSchwarz) live in the
 * host package and produce these lists.  JFG_ERR_SINGULAR: a patch matrix is
 * singular. */
typedef enum { JFG_SCHWARZ_MULTIPLICATIVE = 0, JFG_SCHWARZ_COLORED = 1, JFG_SCHWARZ_ADDITIVE = 2 } jfg_schwarz_kind;
int jfg_schwarz_create(jfg_ctx* ctx, jfg_mat* A, int kind, double omega, int npatches, const int64_t* patch_ptr,
                       const int* patch_dofs, int ncolors, const int* color_ptr, const int* color_patches,
                       jfg_schwarz** out);
int jfg_schwarz_free(jfg_schwarz* s);
/* Largest patch, number of stored inverse entries, colours run as one fused launch. */
int jfg_schwarz_info(jfg_schwarz* s, int* max_patch, int64_t* inverse_entries, int* independent_colors);
/* x <- SubspaceCorrection.apply(schwarz, x, rhs) (SubspaceCorrection.java:11-18 and overrides). */
int jfg_schwarz_apply(jfg_schwarz* s, const double* h_rhs, double* h_x);
/* out = SubspaceCorrection.solve(schwarz, rhs) = AbstractSchwarz.mvMul (AbstractSchwarz.java:62-66). */
int jfg_schwarz_solve(jfg_schwarz* s, const double* h_rhs, double* h_out);
/* x <- SchwarzSmoother.smooth: runs x apply. */
int jfg_schwarz_smooth(jfg_schwarz* s, int runs, const double* h_rhs, double* h_x);
int jfg_schwarz_smooth_dev(jfg_schwarz* s, int runs, const double* d_rhs, double* d_x);
/* Patch p's size, sorted DOFs and row-major inverse (each output may be NULL). */
int jfg_schwarz_local_inverse(jfg_schwarz* s, int patch, int* m, int* h_dofs, double* h_inv);
/* Mean milliseconds of one apply (CUDA events). */
int jfg_schwarz_time(jfg_schwarz* s, int iters, double* ms_apply);

/* ---- geometric multigrid -------------------------------------------- */
typedef struct {
    int cycles;        /* V-cycles per application (MGPreconditionerSpace.cycles, default 3) */
    int use_fmg;       /* 1: FMG correction first (MGPreconditionerInterface.mvMul, :353-379);
                          0: start the V-cycles from the boundary copy only */
    int precision;     /* 0: FP64 hierarchy; 1: FP32 hierarchy (for mixed-precision solves);
                          2: FP32 hierarchy whose SpMVs read BF16 matrix values (FP32 vectors and sums);
                          3: FP32 hierarchy whose SpMVs read FP16 matrix values scaled by a power of two
                             per matrix (max |a| * 2^k in [2^14, 2^15)), FP32 vectors and sums */
    int cycle;         /* 0: the application runs V-cycles (mvMul);
                          1: W-cycles, MGPreconditionerSpace.mvMulW (multigrid/MGPreconditionerSpace.java:165-183) */
} jfg_mg_desc;
/* Builds a hierarchy from per-level systems A[0..levels) (0 = coarsest),
 * prolongations P[l] (n_{l+1} x n_l, l < levels-1), Dirichlet node lists and
 * smoothers (sm[l] for l >= 1; sm[0] ignored: level 0 is solved by dense LU).
 * Replaces the MGPreconditionerSpace constructor's products
 * (Core/src/main/java/multigrid/MGPreconditionerSpace.java:28-57). */
int jfg_mg_create(jfg_ctx* ctx, int levels, jfg_mat* const* A, jfg_mat* const* P,
                  const int* const* h_bdry, const int* n_bdry, const jfg_smoother_desc* sm,
                  const jfg_mg_desc* desc, jfg_mg** out);
int jfg_mg_free(jfg_mg* mg);
/* out = M v, the preconditioner application.  Replaces
 * MGPreconditionerInterface.mvMul (multigrid/MGPreconditionerInterface.java:352-379). */
int jfg_mg_apply(jfg_mg* mg, const double* h_v, double* h_out);
/* out = vCycle(x0, rhs).  Replaces MGPreconditionerInterface.vCycle (:293-298). */
int jfg_mg_vcycle(jfg_mg* mg, const double* h_x0, const double* h_rhs, double* h_out);
/* out = wCycle(x0, rhs).  Replaces MGPreconditionerInterface.wCycle (:300-305), i.e. mgStepW
 * (:200-291): smoothing, two coarse-grid corrections by mgStepV on the next coarser level, smoothing. */
int jfg_mg_wcycle(jfg_mg* mg, const double* h_x0, const double* h_rhs, double* h_out);
/* out = fullVCycleCorrection(defect).  Replaces MGPreconditionerInterface.fullVCycleCorrection (:307-326). */
int jfg_mg_fmg(jfg_mg* mg, const double* h_defect, double* h_out);

/* ---- iterative solvers ----------------------------------------------- */
typedef enum {
    JFG_CG = 0,          /* IterativeSolver.solveCG        (linalg/IterativeSolver.java:48-100) */
    JFG_PCG = 1,         /* IterativeSolver.solvePCG       (:102-162) */
    JFG_BICGSTAB = 2,    /* IterativeSolver.solveBiCGStab  (:256-323) */
    JFG_PBICGSTAB = 3,   /* IterativeSolver.solvePBiCGStab (:325-402) */
    JFG_GMRES = 4,       /* IterativeSolver.solveGMRES / GMRES.solve (linalg/GMRES.java:103-134) */
    JFG_PGMRES = 5,      /* IterativeSolver.solvePGMRES / GMRES.solve with preconditioner (GMRES.java:64-101) */
    JFG_GMRES2 = 6,      /* GMRES2.solve (linalg/GMRES2.java:34-104) */
    JFG_FGMRES = 7       /* flexible right-preconditioned GMRES(restart); no counterpart in the reference
                            (needed for a preconditioner that changes between iterations) */
} jfg_solver_kind;

typedef enum {
    JFG_PREC_NONE = 0,
    JFG_PREC_MG = 1,       /* handle = jfg_mg* */
    JFG_PREC_JACOBI = 2,   /* diagonal of A */
    JFG_PREC_MATRIX = 3,   /* handle = jfg_mat* applied as y = M x (e.g. an identity or an inverse) */
    JFG_PREC_MG_CNN = 4,   /* handle = jfg_mgcnn*: FP32 V-cycle followed by the learned smoother */
    JFG_PREC_SCHWARZ = 5,  /* handle = jfg_schwarz*: AbstractSchwarz.mvMul (FP64 solves) */
    JFG_PREC_BLOCKDIAG = 6 /* handle = jfg_blockdiag*: velocity multigrid + diagonal pressure block */
} jfg_precond_kind;

typedef enum {
    JFG_FP64 = 0,          /* every operation in FP64 */
    JFG_MIXED = 1,         /* FP64 defect-correction outer loop around an FP32 inner solve */
    JFG_MIXED_PRECOND = 2  /* FP64 Krylov iteration (true residual, dots) with an FP32 preconditioner */
} jfg_precision;

typedef struct {
    double tol;            /* absolute residual tolerance, as the reference's `tol` */
    int maxit;             /* 0: reference default (n for CG/BiCGStab, 10 n for PBiCGStab) */
    int restart;           /* GMRES: GMRES.ITERATIONS_BEFORE_RESTART (default 150) */
    int max_restarts;      /* GMRES: GMRES.MAX_RESTARTS (default 200) */
    int precision;         /* jfg_precision */
    double inner_rtol;     /* JFG_MIXED: relative tolerance of each inner solve (default 1e-4) */
    int use_graph;         /* 1: replay the Krylov iteration as a CUDA graph */
    int graph_chunk;       /* iterations per graph launch between convergence polls (default 8) */
    double* h_history;     /* optional: residual norm per iteration */
    int history_cap;
    int start;             /* jfg_solve: 0 = x holds the start iterate (copied in, e.g. lastSolution);
                              1 = start from e0 (IterativeSolver.java:69-70) and 2 = from zero, without
                              reading x (one host-to-device copy fewer) */
} jfg_solver_opts;

typedef struct {
    int iterations;        /* IterativeSolver.iterations */
    int restarts;
    int status;            /* jfg_status */
    int outer_iterations;  /* JFG_MIXED: defect-correction steps */
    double final_residual; /* FP64 true residual ||b - A x|| at exit */
    double final_norm;     /* last residual norm published by the iteration */
    int history_len;
    int not_pd;            /* CG met p.Ap <= 0 ("CG warning: Matrix not PD") */
} jfg_solve_info;

/* Fills opts with the reference defaults (tol 1e-10 absolute, restart 150,
 * 200 restarts, FP64, CUDA graph on). */
void jfg_solver_opts_default(jfg_solver_opts* opts);

/* Solves A x = b.  x holds the start iterate on entry (the reference starts
 * from e0, or from the previous solution when an IterativeSolver is reused,
 * IterativeSolver.java:69-72) and the solution on exit.  `precond` is a
 * jfg_mg* for JFG_PREC_MG, a jfg_mat* for JFG_PREC_MATRIX, NULL otherwise.
 * Replaces the IterativeSolver.solve* methods listed in jfg_solver_kind. */
int jfg_solve(jfg_ctx* ctx, int kind, jfg_mat* A, int precond_kind, void* precond, const double* h_b,
              double* h_x, const jfg_solver_opts* opts, jfg_solve_info* info);
/* Same on device vectors (no host copies; synchronises at exit). */
int jfg_solve_dev(jfg_ctx* ctx, int kind, jfg_mat* A, int precond_kind, void* precond, const double* d_b,
                  double* d_x, const jfg_solver_opts* opts, jfg_solve_info* info);

/* ---- batched implicit time stepping ----------------------------------- */
/* Many independent systems of uneven size advanced together by implicit
 * Euler: K_s u_s^{k+1} = M_s u_s^k + f_s with K_s = M_s + dt A_s, for every
 * system s and step k, each solve an FP32 Jacobi-PCG inside an FP64
 * refinement loop accepted on the FP64 relative true residual.  Replaces the
 * time loop of Examples/src/HeatEquation.java:81-94 (solveCG(M + dt A,
 * source + M u, 1e-10) per step) and FullyImplicitParabolicIntegrator.timeStep
 * (Core/src/main/java/basic/FullyImplicitParabolicIntegrator.java:41-53) for a
 * whole batch.  All systems' iterations run in one persistent launch:
 * thread-block clusters take systems from a work queue (largest first) and
 * reduce across the cluster through distributed shared memory. */
typedef struct jfg_batch jfg_batch;
typedef struct {
    int cluster;        /* CTAs per system (1, 2, 4, 8); 0 = autotuned */
    int threads;        /* threads per CTA (256, 512); 0 = autotuned */
    double rtol;        /* relative FP64 residual per step (default 1e-10) */
    double inner_rtol;  /* FP32 inner PCG relative tolerance (default 1e-5) */
    int inner_max;      /* inner iteration cap (default 500) */
    int max_refine;     /* refinement steps per time step (default 6) */
    int rows_per_thread; /* rows of a thread in flight per inner pass (2, 3, 4); 0 = autotuned */
} jfg_batch_opts;
typedef struct {
    int total_inner_iterations;
    int max_refine_used;
    double max_rel_residual;   /* worst FP64 relative residual over systems (last step) */
    int failed;                /* systems that missed rtol within max_refine */
    int cluster, threads;      /* configuration used */
    double ms;                 /* device time of the persistent launch */
    int rows_per_thread;       /* configuration used */
} jfg_batch_info;
void jfg_batch_opts_default(jfg_batch_opts* o);
/* K[s], M[s]: square matrices of the same size n_s; f (optional) packed
 * sum_s n_s right-hand-side increments added every step. */
int jfg_batch_create(jfg_ctx* ctx, int nsys, jfg_mat* const* K, jfg_mat* const* M, jfg_batch** out);
int jfg_batch_free(jfg_batch* b);
/* Total unknowns (sum of n_s) and the offset of system s in packed vectors. */
int jfg_batch_layout(jfg_batch* b, int64_t* total, int64_t* offsets);
/* Advances every system `steps` implicit-Euler steps.  h_u: packed FP64
 * states (in: u0, out: u after the last step); h_f: packed increments or NULL. */
int jfg_batch_heat(jfg_batch* b, int steps, const double* h_f, double* h_u, const jfg_batch_opts* opts,
                   jfg_batch_info* info);

/* ---- learned smoother network ------------------------------------------ */
/* No counterpart in the reference (JFEM has no neural-network code): a 6-layer
 * 3x3 convolutional residual network on the node grid (32 channels, no
 * biases), BF16 tensor-core forward and backward kernels with FP32
 * accumulation, FP32 Adam master weights.  Images are (B, H, W) FP32 device
 * arrays.  Weights: 37,440 FP32 values, layer by layer in (Cout, Cin, 3, 3)
 * order (conv1 32x1, conv2..5 32x32, conv6 1x32). */
typedef struct jfg_cnn jfg_cnn;
int jfg_cnn_num_params(int* count);
int jfg_cnn_create(jfg_ctx* ctx, jfg_cnn** out);
int jfg_cnn_free(jfg_cnn* n);
int jfg_cnn_set_weights(jfg_cnn* n, const float* h_w);
int jfg_cnn_get_weights(jfg_cnn* n, float* h_w);
/* y = net(x) on device images. */
int jfg_cnn_forward_dev(jfg_cnn* n, int B, int H, int W, const float* d_x, float* d_y);
/* loss = mean (net(x) - t)^2 and its weight gradient (kept for the next
 * Adam step; copied to h_grad when non-NULL). */
int jfg_cnn_loss_grad_dev(jfg_cnn* n, int B, int H, int W, const float* d_x, const float* d_t, double* loss,
                          float* h_grad);
/* One Adam step with the last computed gradient. */
int jfg_cnn_adam_step(jfg_cnn* n, double lr, double beta1, double beta2, double eps);
/* Times the forward pass (ms per pass) and one 32 -> 32 tensor-core layer. */
int jfg_cnn_time_forward(jfg_cnn* n, int B, int H, int W, int iters, double* ms_total, double* ms_mid);

/* The preconditioner "FP32 V-cycle, then the learned smoother" for FGMRES:
 *   z = V(v);  r' = v - A z;  q = D^-1 r' (D = diag A);  s = rms(q);
 *   z += out_scale * s * scatter(net(gather(q) / s))   (zero on Dirichlet nodes)
 * where the node grid is H x W and h_dof_of_pixel[i] is the unknown at pixel
 * i (row-major).  The V-cycle runs on mg's FP32 copy of the hierarchy
 * (built on first use); A is the system matrix.  use_net = 0 applies the
 * V-cycle only (the method without the network, for comparison).  The
 * network's current weights are used at every application.  Pass the handle
 * to jfg_solve with JFG_PREC_MG_CNN and JFG_FGMRES. */
typedef struct jfg_mgcnn jfg_mgcnn;
int jfg_mgcnn_create(jfg_ctx* ctx, jfg_mg* mg, jfg_cnn* net, jfg_mat* A, int H, int W, const int* h_dof_of_pixel,
                     const int* h_bdry, int n_bdry, double out_scale, int use_net, jfg_mgcnn** out);
/* Changes out_scale and use_net of an existing handle. */
int jfg_mgcnn_set(jfg_mgcnn* p, double out_scale, int use_net);
/* z = the preconditioner applied to v (FP64 device vectors of the system size). */
int jfg_mgcnn_apply_dev(jfg_mgcnn* p, const double* d_v, double* d_z);
int jfg_mgcnn_free(jfg_mgcnn* p);

/* ---- block-diagonal saddle-point preconditioner ------------------------ */
/* For systems ordered velocity first (TaylorHoodSpace numbering): z_v = mg
 * applied to r_v (mg built on the velocity block, nv unknowns; FP32 V-cycle
 * when fp32_vcycle), z_p = pinv * r_p (np unknowns, e.g. the inverse lumped
 * pressure mass).  The block-diagonal preconditioner of the Stokes
 * examples (examples StokesMG / StokesMGBS*: velocity multigrid, pressure
 * mass scaling).  Pass to jfg_solve with JFG_PREC_BLOCKDIAG. */
typedef struct jfg_blockdiag jfg_blockdiag;
int jfg_blockdiag_create(jfg_ctx* ctx, jfg_mg* mg, int nv, int np, const double* h_pinv, int fp32_vcycle,
                         jfg_blockdiag** out);
int jfg_blockdiag_apply(jfg_blockdiag* b, const double* h_v, double* h_out);
int jfg_blockdiag_free(jfg_blockdiag* b);

/* ---- implicit Schur complement (DLM block solvers) ------------------- */
/* S x = A00 x - sum_i T_i (Dinv_i (L_i x)) as a composed device operator,
 * never formed: the Schur operator of ImplicitSchurSolver.schurMvMul
 * (linalg/ImplicitSchurSolver.java:17-57).  A00 is n0 x n0, T_i n0 x n_i,
 * Dinv_i n_i x n_i (the inverse of the diagonal block D_i, as a matrix), L_i
 * n_i x n0; the matrices are borrowed (they must outlive the handle). */
typedef struct jfg_schur jfg_schur;
int jfg_schur_create(jfg_ctx* ctx, jfg_mat* A00, int k, jfg_mat* const* T, jfg_mat* const* Dinv,
                     jfg_mat* const* L, jfg_schur** out);
/* y = S x (host vectors of n0 entries). */
int jfg_schur_apply(jfg_schur* s, const double* h_x, double* h_y);
/* GMRES (kind JFG_GMRES) or preconditioned GMRES (JFG_PGMRES, e.g. with
 * the dense inverse of A00 as a JFG_PREC_MATRIX preconditioner) on S, with
 * jfg_solve's options and report; the final residual is ||b - S x||.
 * IterativeImplicitSchur.solveSchur (linalg/IterativeImplicitSchur.java:19-23)
 * is JFG_PGMRES to 1e-9 preconditioned by the inverse of A00. */
int jfg_schur_solve(jfg_schur* s, int kind, int precond_kind, void* precond, const double* h_b, double* h_x,
                    const jfg_solver_opts* opts, jfg_solve_info* info);
int jfg_schur_free(jfg_schur* s);

/* ---- dense direct solves --------------------------------------------- */
/* x = A^-1 b for a dense row-major n x n A (partial-pivot LU on the GPU).
 * Replaces DenseMatrix.solve (linalg/DenseMatrix.java:516-519) and the JNI
 * iSolve (JSparse/src/native/sparseSolver.cpp:10-60). */
int jfg_dense_solve(jfg_ctx* ctx, int n, const double* h_A, const double* h_b, double* h_x);
/* Ainv = A^-1.  Replaces DenseMatrix.inverse and the JNI iInverse (sparseSolver.cpp:63-113). */
int jfg_dense_inverse(jfg_ctx* ctx, int n, const double* h_A, double* h_Ainv);
/* CG on a system the caller already holds on the device as CSR (row
 * pointers, column indices, values; no duplicates), for callers that must not
 * allocate device memory while they solve -- e.g. a host framework that owns
 * the device heap (a pool or budget the library must not touch), or a loop
 * that cannot take cudaMalloc's latency and implicit synchronisation.  No
 * counterpart in the reference: it is the allocation-free twin of
 * jfg_solve_dev(JFG_CG, ...), with the same iteration and semantics (x holds
 * the start iterate on entry, the solution on exit; absolute tolerance;
 * maxit <= 0 means n).  All work memory (three vectors of n doubles, the
 * reduction partials, the control block) is one fixed __device__ array of
 * about 6.3 MB per GPU: n is limited to 262,144 unknowns (larger n is
 * rejected with JFG_ERR_BAD_ARG).  The array is shared by every call and
 * keeps the last call's contents; calls that overlap on the GPU race on it.
 * The call runs eagerly on the context's stream and synchronises the host
 * with it (it polls the convergence flag every 8 iterations).  The first call
 * on a device looks up the array's address and caches it for the process
 * lifetime (the device's primary context; no cudaDeviceReset in between).
 * A met p.Ap <= 0 (indefinite matrix) is reported through jfg_last_error.
 * Calls no cudaMalloc/cudaFree. */
int jfg_cg_noalloc(jfg_ctx* ctx, int n, const int* d_rowptr, const int* d_col, const double* d_val,
                   const double* d_b, double* d_x, double tol, int maxit, int* iterations, double* final_norm);

/* Drop-in for SparseMatrix.solve(rhs) (linalg/SparseMatrix.java:142-150): COO in, x out.
 * n <= 4096: dense LU of the merged matrix on the GPU (the reference's method);
 * larger: FP64 GMRES with a Jacobi preconditioner to ||b - A x|| <= 1e-12 ||b||. */
int jfg_sparse_solve(jfg_ctx* ctx, int n, int64_t nnz, const int* h_rows, const int* h_cols,
                     const double* h_vals, const double* h_b, double* h_x);

#ifdef __cplusplus
}
#endif
#endif /* JFEM_GPU_H */
