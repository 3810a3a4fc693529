// Geometric multigrid hierarchy on the device (one instance per precision).
#pragma once
#include <memory>

#include "jfg_ops.cuh"

namespace jfg {

struct SchwarzImpl;
struct GSImpl;

struct SmootherDesc {
    int kind = JFG_SMOOTH_JACOBI;
    int runs = 2;
    double omega = 2.0 / 3.0;
    SchwarzImpl* schwarz = nullptr;   // JFG_SMOOTH_SCHWARZ
    GSImpl* gs = nullptr;             // JFG_SMOOTH_FBGS / JFG_SMOOTH_GS
};

// The hierarchy of MGPreconditionerSpace / MGPreconditionerInterface
// (multigrid/MGPreconditionerInterface.java:125-379) with every level's
// vectors resident.  T is the arithmetic type of the smoothing, transfers and
// residuals (double, or float for mixed-precision inner solves); the coarsest
// level is always solved in FP64 from a device-computed inverse.
template <typename T>
struct MGImpl {
    Context* c = nullptr;
    uint64_t uid = next_uid();
    int L = 0;
    int cycles = 3;
    int use_fmg = 1;
    int wcycle = 0;                         // apply: mgStepW (MGPreconditionerSpace.mvMulW) instead of mgStepV
    int vbf16 = 0;                          // float hierarchy: matrices read as BF16 (FP32 vectors, FP32 sums)
    int vfp16 = 0;                          // float hierarchy: matrices read as scaled FP16 (FP32 vectors, sums)
    int tail = -1;                          // levels 0..tail run as one cluster kernel (-1: none)
    int tail_ctas = 0;                      // CTAs of that cluster
    int tail_pkg_bytes = 0;                 // constant shared-memory package per CTA
    int tail_smem_bytes = 0;                // package + the level vectors per CTA
    DevBuf<uint4> tail_pkg;                 // the matrices of levels 1..tail as per-CTA ELL slices
    std::vector<int> tail_meta;             // per level: shared-memory layout (see build_tail)
    std::vector<Matrix*> A, P, R;          // A[l], P[l] : n_{l+1} x n_l, R[l] = P[l]^T
    std::vector<int> n;
    std::vector<DevBuf<T>> x, t, b, r, fr;
    std::vector<DevBuf<T>> dinv;
    std::vector<DevBuf<unsigned char>> mask;
    std::vector<SmootherDesc> sm;
    DevBuf<double> ainv0;                   // n0 x n0 row-major inverse of A[0]
    int coarse_status = JFG_OK;
    // finest-level boundary copy (MGPreconditionerInterface.java:355-357):
    // defect = v - A * (v restricted to boundary nodes) only differs from v on
    // rows that have entries in boundary columns; those rows are kept as CSR.
    DevBuf<int> bd_fine;
    int nbd_fine = 0;
    bool bd_unique = true;              // the finest boundary list names no unknown twice
    // apply(): the last post-smoothing sweep adds bc_src at the finest boundary
    // (instead of a separate k_bc_add launch); bc_done reports that it did
    const T* bc_src = nullptr;
    bool bc_done = false;
    DevBuf<int> aff_row, aff_ptr, aff_col;
    DevBuf<T> aff_val;
    int naff = 0;
    DevBuf<int> flags;                      // per-level smoother flags
    DevBuf<int> zero_flag;                  // a flag that stays 0

    // Builds all level data; A/P are borrowed (must outlive the hierarchy).
    // bf16: (float hierarchy only) SpMVs read BF16 copies of the matrices.
    void init(Context* ctx, int levels, Matrix* const* As, Matrix* const* Ps, const int* const* bdry,
              const int* nbdry, const SmootherDesc* sms, int cycles_, int use_fmg_, int vfmt = 0);

    // out = M v (the preconditioner application).  v and out are device
    // vectors of the finest size; `done` is an optional skip flag.
    void apply(const T* v, T* out, const Scratch& sc, const int* done, cudaStream_t st);
    // out = vCycle(x0, rhs) on the finest level.
    void vcycle(const T* x0, const T* rhs, T* out, const Scratch& sc, const int* done, cudaStream_t st);
    // out = wCycle(x0, rhs) on the finest level.
    void wcycle_apply(const T* x0, const T* rhs, T* out, const Scratch& sc, const int* done, cudaStream_t st);
    // out = fullVCycleCorrection(defect).
    void fmg(const T* defect, T* out, const Scratch& sc, const int* done, cudaStream_t st);

    // internals
    // dest (optional): where the level's final smoothing result goes instead of x[l]
    void vstep(int l, const T* rhs, bool xzero, const Scratch& sc, const int* done, cudaStream_t st,
               bool first_sweep_done = false, T* dest = nullptr);
    // mgStepW: guess in x[l] (or zero); two coarse-grid corrections by mgStepV
    void wstep(int l, const T* rhs, bool xzero, const Scratch& sc, const int* done, cudaStream_t st,
               T* dest = nullptr);
    // restricted defect of x[l] into level l-1 (with the fused first Jacobi
    // sweep there when possible), mgStepV on l-1 from zero, prolongation + add
    void coarse_correction(int l, const T* rhs, const Scratch& sc, const int* done, cudaStream_t st);
    void smooth(int l, const T* rhs, bool xzero, const Scratch& sc, const int* done, cudaStream_t st,
                bool first_sweep_done = false, T* dest = nullptr);
    void coarse(const T* rhs, T* out, const int* done, cudaStream_t st);
    // the V-cycle below and including level `tail`, entered from the restriction above
    void run_tail(bool first_sweep_done, const int* done, cudaStream_t st);
    void build_tail();
    void fmg_into_top(const T* defect, const Scratch& sc, const int* done, cudaStream_t st);
    int max_blocks() const;
};

// Smoother.smooth on one level (JacobiSmoother / RichardsonSmoother).
void smooth_standalone(Context* c, Matrix* A, const SmootherDesc& d, const double* d_rhs, double* d_x,
                       const Scratch& sc);

// Dense LU helpers (jfg_dense.cu).
// Factorises the row-major n x n matrix in place (partial pivoting) and
// writes its inverse; returns JFG_OK or JFG_ERR_SINGULAR.
int dense_inverse_device(Context* c, int n, double* d_A, double* d_inv);
int dense_solve_device(Context* c, int n, double* d_A, const double* d_b, double* d_x);

}  // namespace jfg

// The public handle keeps both precisions; the FP32 copy is built on first use.
struct jfg_mg {
    jfg::Context* ctx = nullptr;
    int levels = 0;
    std::vector<jfg::Matrix*> A, P;
    std::vector<std::vector<int>> bdry;
    std::vector<jfg::SmootherDesc> sm;
    int cycles = 3, use_fmg = 1, precision = 0, wcycle = 0;
    std::unique_ptr<jfg::MGImpl<double>> d64;
    std::unique_ptr<jfg::MGImpl<float>> d32;
    jfg::MGImpl<float>* fp32();
};
