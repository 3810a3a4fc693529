// Overlapping Schwarz subspace corrections on the device: shared declarations.
#pragma once
#include <vector>

#include "jfg_ops.cuh"

namespace jfg {

// One Schwarz decomposition of a square matrix A (schwarz/UpFrontSchwarz.java):
// patches are sorted global-DOF lists (the rows of the restriction matrices
// R_p), every patch keeps the dense inverse of R_p A R_p^T (DirectSolver), and
// the subspace correction is multiplicative (sequential over patches),
// coloured multiplicative (patches of one colour from one residual) or additive.
struct SchwarzImpl {
    Context* c = nullptr;
    Matrix* A = nullptr;
    int n = 0;
    int kind = 0;
    double omega = 1.0;
    int np = 0;
    int max_m = 0;
    int64_t total_m = 0, total_inv = 0;
    int nunique = 0;                    // distinct patch operators (inverses stored)
    bool fast = true;                   // batched / shared-memory colour-step kernels (JFEM_SCHWARZ_FAST)
    int batch_max = 4;                  // patches per batch of k_schwarz_batch
    int batch_threads = 256;            // its threads per CTA (4 CTAs per SM)
    uint64_t uid = next_uid();
    DevBuf<int64_t> pptr, inv_off;      // patch p: dofs[pptr[p], pptr[p+1]), inverse at inv + inv_off[p]
    DevBuf<int> dofs;
    DevBuf<double> inv;                 // m_p x m_p inverses, column-major (transposed)
    DevBuf<float> inv32;                // FP32 copy for FP32 hierarchies (built on first use)
    DevBuf<int> seq;                    // multiplicative: patches forward then backward (2 np)
    DevBuf<int> cpat;                   // colour patch lists, concatenated
    DevBuf<int> touched;                // per colour (or all, additive): DOFs updated by the scatter
    DevBuf<int64_t> tptr;               // contributions of touched[t]: slots[tptr[t], tptr[t+1])
    DevBuf<int64_t> slots;              // indices into lsol, in ascending patch order
    DevBuf<double> lsol;                // local solutions of the patches of one sweep step
    DevBuf<int> flag;
    DevBuf<int> bpat, bptr;             // batches of patches sharing an inverse (colours with many patches)
    struct Colour {
        int start = 0, count = 0;       // range of cpat
        bool independent = false;       // patches neither share nor couple DOFs: one fused kernel
        int64_t t_start = 0, t_count = 0;   // range of touched
        int mcap = 0;                   // largest patch of the colour
        int b_start = 0, b_count = 0;   // batches bptr[b_start .. b_start + b_count] (0: one CTA per patch)
        int kern = 0;                   // 0: one CTA per patch, 1: k_schwarz_batch, 2 / 3: k_schwarz_colour
                                        // with the inverse in shared / global memory
        int rows_cap = 0;               // patch rows per batch at most (k_schwarz_colour)
        int grid = 0;                   // CTAs of the colour-step launch
    };
    std::vector<Colour> colours;
    Colour all;                         // additive: every patch in order

    void init(Context* ctx, Matrix* A, int kind, double omega, int np, const int64_t* pptr, const int* dofs,
              int ncolours, const int* colour_ptr, const int* colour_patches);
    // SubspaceCorrection.apply: x <- x + corrections (b - A x)
    template <typename T>
    void apply(const T* b, T* x, const Scratch& sc, const int* done, cudaStream_t st);
    // SubspaceCorrection.solve: out = corrections of b from a zero iterate
    template <typename T>
    void solve(const T* b, T* out, const Scratch& sc, const int* done, cudaStream_t st);
    // SchwarzSmoother.smooth: runs x apply
    template <typename T>
    void smooth(int runs, const T* b, T* x, const Scratch& sc, const int* done, cudaStream_t st)
    {
        for (int i = 0; i < runs; i++) apply<T>(b, x, sc, done, st);
    }
    const float* inverses32();

private:
    template <typename T>
    void colour_step(const Colour& col, const T* b, T* x, double om, const int* done, cudaStream_t st);
    void build_scatter(Colour& col, const std::vector<int64_t>& hp, const std::vector<int>& hd,
                       const std::vector<int>& patches, std::vector<int>& h_touched, std::vector<int64_t>& h_tptr,
                       std::vector<int64_t>& h_slots);
};

}  // namespace jfg

struct jfg_schwarz {
    jfg_ctx* ctx = nullptr;
    jfg::SchwarzImpl s;
};

namespace jfg {
SchwarzImpl* schwarz_of(jfg_schwarz* s);
}  // namespace jfg
