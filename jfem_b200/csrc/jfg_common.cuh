// Shared definitions of the JFEM linear-solve library for sm_100a.
//
// Layout decisions (all device memory is owned by the library):
//   * matrices live in SELL-32-sigma for the products (see Matrix) plus a
//     plain CSR copy for set-up work;
//   * values exist in FP64 and, on demand, FP32 / BF16 (mixed-precision
//     hierarchies) -- all copies share the index arrays;
//   * all scalars of an iterative solve (alpha, beta, <r,r>, flags, the
//     iteration counter and the residual history) live in a device control
//     block, so a whole Krylov iteration is a fixed kernel sequence that can be
//     captured into a CUDA graph and replayed without host round trips.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <atomic>
#include <stdio.h>
#include <string>
#include <vector>

#include "../../include/jfem_gpu.h"

namespace jfg {

constexpr int kThreads = 256;          // threads per CTA in streaming kernels
constexpr int kVecGrid = 148 * 8;      // fixed grid of the vector kernels (SM count x 8)

struct Error {
    int status;
    std::string msg;
};

#define JFG_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw ::jfg::Error{JFG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define JFG_CHECK(cond, code, text)                                                        \
    do {                                                                                   \
        if (!(cond)) throw ::jfg::Error{(code), (text)};                                   \
    } while (0)

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        if (count <= n && p) return;
        release();
        JFG_CUDA(cudaMalloc(&p, (count ? count : 1) * sizeof(T)));
        n = count;
    }
};

// The control block of one iterative solve (device resident).
struct Ctl {
    double alpha, beta, omega, rho, rho_last;
    double rr, rz, pAp;
    double tol;             // absolute residual tolerance (the reference's `tol`)
    double res_norm;        // latest published residual norm
    double s_norm;          // BiCGStab: ||s||
    double true_res;        // GMRES: ||A x - b|| after a cycle
    int iter;               // iterations done (IterativeSolver.iterations)
    int maxit;
    int done;               // 1 = stop iterating
    int status;             // jfg_status of the solve
    int not_pd;             // CG met p.Ap <= 0
    int sdone;              // BiCGStab: ||s|| < tol branch taken
    int skip;               // BiCGStab: skip the second half of the iteration
    int j;                  // GMRES: current Arnoldi index
    int jfin;               // GMRES: index of the last column used
    int cycle_done;         // GMRES: inner loop finished
    int restart_len;        // GMRES: ITERATIONS_BEFORE_RESTART
    int n;                  // problem size
    int hist_cap;
    double* hist;           // residual history (device)
};

struct Context;

// Row-block CSR matrix on the device.
// Two layouts on the device:
//   * CSR (csr_*): merged, sorted by row then column; used by set-up code
//     (transposes, diagonal, dense extraction);
//   * SELL-32-sigma (the SpMV layout): rows are sorted by length inside
//     windows of kSellSigma rows, cut into slices of 32 rows, and each slice
//     is stored column-major padded to its longest row: entry k of slice lane
//     l lives at off[s] + 32 k + l.  perm[32 s + l] is the original row (-1
//     for the padding rows of the last slice).  One thread owns one row.
constexpr int kSliceRows = 32;
constexpr int kSellSigma = 256;

struct Matrix {
    Context* ctx = nullptr;
    int rows = 0, cols = 0;
    int64_t nnz = 0;              // stored nonzeros after merging
    DevBuf<int> csr_ptr;          // rows + 1
    DevBuf<int> csr_col;          // nnz
    DevBuf<double> csr_val;       // nnz
    int nslices = 0;
    int64_t sell_len = 0;         // length of the SELL col/val arrays
    int nblocks = 0;              // CTAs of one SpMV launch
    int tpr_log2 = 0;             // log2 of the threads per row in the SpMV
    DevBuf<int> off;              // nslices + 1 slice offsets
    DevBuf<int> perm;             // nslices * 32 original row of each slot
    DevBuf<int> col;              // sell_len
    DevBuf<int16_t> col16;        // sell_len: 16-bit column offsets (idx16 = 1: col - max(row, 0);
                                  // idx16 = 2: col - cbase[slice])
    DevBuf<int> cbase;            // nslices: base column of each slice (idx16 = 2; rectangular matrices)
    int idx16 = 0;                // the SpMV reads col16 instead of col
    DevBuf<double> val;           // sell_len
    DevBuf<float> val32;          // optional FP32 copy
    DevBuf<__nv_bfloat16> val16;  // optional BF16 copy
    DevBuf<double> diag;          // merged diagonal
    DevBuf<__half> valh;          // optional FP16 copy of the values scaled by 2^k (fits the FP16 range)
    float hscale_inv = 1.0f;      // 2^-k: row sums of valh times this are the sums of the values
    int has32 = 0, has16 = 0, hash = 0;
    int csr_only = 0;             // no SELL layout (an intermediate of a sparse product)
    // Values-only 9-point stencil layout (square matrices of 2-D Q1 grids
    // numbered lexicographically with stride st_S over a contiguous range of
    // rows): row r in [st_lo, st_hi) couples only to the columns
    // r + {-S-1, -S, -S+1, -1, 0, 1, S-1, S, S+1}, and all nine of those
    // columns exist.  Its values are stored per offset, st_val[k * nreg +
    // (r - st_lo)] (zero where the matrix has no entry), with no column
    // indices at all.  The rows outside the range ("irregular", a prefix and
    // a suffix of the numbering) keep a CSR copy: st_irow / st_iptr / st_icol
    // and their values at st_val[9 * st_ld + k].  The per-offset stride st_ld
    // is nreg rounded up to a multiple of 8, so a thread's pair of rows loads
    // its values with one aligned vector load per offset.  The SELL layout is kept as
    // well (other kernels read it); products with a stencil copy of their
    // value type use this layout.
    // The same point layout also serves the grid transfers between Q1 levels
    // (st_kind 1: prolongation, fine rows; 2: restriction, coarse rows): the
    // columns of a regular row are center(r) + offsets, center(r) computed
    // from the row's grid position (strides st_S of the rows, st_S2 of the
    // columns); st_K values per row (4 or 9).
    int st = 0;
    int st_staged = 0;            // 1: the staged kernel (k_spmv_pt) for the 9-point kind; 0: k_spmv_st
    DevBuf<int> st_err;           // set by k_spmv_pt when a bulk copy does not complete
    int st_kind = 0, st_K = 9, st_S2 = 0;
    int st_S = 0, st_lo = 0, st_hi = 0, st_nirr = 0, st_ld = 0;
    int st_nb_reg = 0;                  // CTAs of the regular rows (a persistent grid over row pairs)
    int st_nb_irr = 0;                  // CTAs of the irregular rows
    int64_t st_len = 0;                 // 9 * st_ld + irregular entries
    DevBuf<int> st_irow, st_iptr, st_icol;
    DevBuf<double> st_val;
    DevBuf<float> st_val32;
    DevBuf<__nv_bfloat16> st_val16;
    DevBuf<__half> st_valh;
    int cg_small_nnz = -1;        // small-system CG: largest CSR slice of its 8 row blocks (-1: not computed)
    Matrix* transposed = nullptr; // lazily built for tvMul
    uint64_t uid = 0;             // unique id (keys of cached CUDA graphs)
    Matrix();
    ~Matrix();
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    // reduction scratch shared by the vector kernels of this context
    DevBuf<double> partials;      // kVecGrid * 4 or nblocks * 4 doubles
    DevBuf<unsigned> counters;    // last-block counters
    DevBuf<double> scal;          // small scalar results
    // grow-only scratch of the sparse products (per-row counts; products and sort space)
    DevBuf<char> gemm_rows, gemm_ws;
};

// host-side helpers implemented in jfg_matrix.cu
Matrix* matrix_from_coo(Context* c, int rows, int cols, int64_t nnz, const int* ri, const int* ci,
                        const double* v, bool keep_zeros);
Matrix* matrix_from_csr_host(Context* c, int rows, int cols, const std::vector<int64_t>& rp,
                             const std::vector<int>& ci, const std::vector<double>& v);
Matrix* matrix_transpose(Matrix* m);
// merged, sorted (key = row * cols + col ascending), zero-free entries on the device -> Matrix
// (sell = false: CSR only, no SpMV layout -- for intermediates of products)
Matrix* matrix_from_sorted_keys(Context* c, int rows, int cols, int64_t m, const uint64_t* d_key,
                                const double* d_val, bool sell = true);
// sparse products (jfg_spgemm.cu)
Matrix* matrix_mmmul(Matrix* a, Matrix* b, bool sell = true);
Matrix* matrix_tmmul(Matrix* a, Matrix* b, bool sell = true);
Matrix* matrix_galerkin(Matrix* r, Matrix* a, Matrix* p);
// finite-element assembly (jfg_assembly.cu)
Matrix* assemble_tp(Context* c, const jfg_tp_desc& d, const double* h_kappa, const double* h_f, double* h_rhs,
                    int* h_node_of_grid, int* h_boundary);
Matrix* assemble_th(Context* c, int cx, int cy, double nu, const double* h_force_qp, int lid, int pin,
                    double* h_rhs, int* h_boundary);
// The transfer point layout (Matrix::st, kinds 1 / 2) of a prolongation or
// restriction between Q1 grids with strides S (rows) and S2 (columns); a
// no-op when it does not fit or after precision copies exist.
void matrix_build_transfer_layout(Matrix* m, int kind, int S, int S2);
void matrix_ensure_fp32(Matrix* m);
void matrix_ensure_bf16(Matrix* m);
void matrix_ensure_fp16(Matrix* m);
uint64_t next_uid();

// Kernels launched by this process (graph replays are added per executed
// body); read through jfg_kernel_launches.
extern std::atomic<unsigned long long> g_launches;
inline void note_launch(unsigned long long k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

}  // namespace jfg
