// Gauss-Seidel family on the device: shared declarations.
#pragma once
#include <vector>

#include "jfg_ops.cuh"

namespace jfg {

// The two triangles of a square matrix A in an ordering of its rows (rank),
// each with a schedule of dependency levels: rows of one level only read
// solution entries of earlier levels.  Level l of a triangle holds its rows
// (rows[start_l .. start_l + count_l)) and their off-diagonal entries in ELL
// form, column-major with width_l columns: entry k of slot q at
// base_l + k * count_l + q (column -1 pads a short row).  Entries keep the
// ascending column order of the row.
struct GSImpl {
    struct Tri {
        int nlevels = 0;
        std::vector<int> start, width;      // host copies, start has nlevels + 1 entries
        std::vector<int64_t> base;
        DevBuf<int> d_start, d_width;
        DevBuf<int64_t> d_base;
        DevBuf<int> rows;
        DevBuf<int> col;
        DevBuf<double> val;
        DevBuf<float> val32;                // FP32 copy for FP32 hierarchies (built on first use)
        // consecutive levels run by one launch: a run of small levels in one
        // cluster (a cluster barrier between levels), or one large level on a grid
        struct Seg {
            int l0 = 0, l1 = 0;
            bool cta = false;
            bool cluster = false;           // run of levels larger than one CTA's threads
        };
        std::vector<Seg> segs;
    };
    Context* c = nullptr;
    Matrix* A = nullptr;
    int n = 0;
    int ordering = 0;
    int colours = 0;
    std::vector<int> rank;                  // host: position of each row in the ordering
    Tri lower, upper;
    DevBuf<float> diag32;
    // strict upper triangle in row order (CSR, ascending columns) for b - R x
    DevBuf<int> sup_ptr, sup_col;
    DevBuf<double> sup_val;
    DevBuf<float> sup_val32;
    int64_t sup_nnz = 0;

    void init(Context* ctx, Matrix* A, int ordering);
    // The steps of the smoothers (T = double, or float for FP32 hierarchies;
    // sol never aliases rhs):
    //   backward:      sol = U^-1 rhs
    //   forward_fbgs:  sol = L^-1 (D y), x += sol      (the second half of a FBGS run)
    //   forward:       sol = L^-1 rhs                  (GaussSeidelSmoother, sol = the new iterate)
    //   strict_upper:  t = b - R x                      (R: strict upper triangle)
    template <typename T>
    void backward(const T* rhs, T* sol, const int* done, cudaStream_t st);
    template <typename T>
    void forward_fbgs(const T* y, T* sol, T* x, const int* done, cudaStream_t st);
    template <typename T>
    void forward(const T* rhs, T* sol, const int* done, cudaStream_t st);
    template <typename T>
    void strict_upper(const T* b, const T* x, T* t, const int* done, cudaStream_t st);

private:
    template <typename T>
    const T* tvals(Tri& tri);
    template <typename T>
    const T* dvals();
    template <typename T>
    const T* svals();
    template <typename T, bool SCALE, bool ADDX>
    void solve(Tri& tri, const T* rhs, T* sol, T* x, const int* done, cudaStream_t st);
};

}  // namespace jfg

struct jfg_gs {
    jfg_ctx* ctx = nullptr;
    jfg::GSImpl g;
};

namespace jfg {
GSImpl* gs_of(jfg_gs* g);
}  // namespace jfg
