// Epilogue functors for the row-block SpMV, vector functors, and the launch
// helpers shared by the multigrid and Krylov code.
#pragma once
#include "jfg_kernels.cuh"

namespace jfg {

// Reduction scratch of one solve / one context: partial sums and a counter.
struct Scratch {
    double* partials = nullptr;   // >= 4 * max(grid) doubles
    unsigned* counter = nullptr;
};

inline int ilog2(int v)
{
    int l = 0;
    while ((1 << (l + 1)) <= v) l++;
    return l;
}

template <typename T> const T* vals_of(const Matrix* M);
// the SELL value copy of type VT and its stencil-layout twin
template <typename VT> struct LayoutVals;
template <> struct LayoutVals<double> {
    static const double* sell(const Matrix* M) { return M->val.p; }
    static const double* st(const Matrix* M) { return M->st_val.p; }
};
template <> struct LayoutVals<float> {
    static const float* sell(const Matrix* M) { return M->val32.p; }
    static const float* st(const Matrix* M) { return M->st_val32.p; }
};
template <> struct LayoutVals<__nv_bfloat16> {
    static const __nv_bfloat16* sell(const Matrix* M) { return M->val16.p; }
    static const __nv_bfloat16* st(const Matrix* M) { return M->st_val16.p; }
};
template <> struct LayoutVals<__half> {
    static const __half* sell(const Matrix* M) { return M->valh.p; }
    static const __half* st(const Matrix* M) { return M->st_valh.p; }
};
template <> inline const double* vals_of<double>(const Matrix* M) { return M->val.p; }
template <> inline const float* vals_of<float>(const Matrix* M) { return M->val32.p; }

// ---------------------------------------------------------------------------
// SpMV epilogues (row r, row sum s)
// ---------------------------------------------------------------------------
template <typename T>
struct EpiStore {  // y = A x
    T* y;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&)[K]) const { y[r] = (T)s; }
};

template <typename T>
struct EpiStoreDot {  // y = A p, acc += p . y
    T* y;
    const T* p;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&acc)[K]) const
    {
        y[r] = (T)s;
        acc[0] += (double)p[r] * (double)s;
    }
};

template <typename T>
struct EpiResid {  // y = b - A x, acc += y^2
    const T* b;
    T* y;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&acc)[K]) const
    {
        T v = b[r] - (T)s;
        y[r] = v;
        acc[0] += (double)v * (double)v;
    }
};

template <typename T>
struct EpiJacobi {  // xn = x + (dinv * (b - A x)) * omega   (JacobiSmoother.java:38-42)
    const T* x;
    const T* b;
    const T* dinv;
    T* xn;
    T omega;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&)[K]) const
    {
        xn[r] = x[r] + (dinv[r] * (b[r] - (T)s)) * omega;
    }
};

template <typename T>
struct EpiJacobiBc {  // EpiJacobi, then xn += v on the boundary rows (the MG mvMul's initial.add(iterate))
    const T* x;
    const T* b;
    const T* dinv;
    T* xn;
    T omega;
    const unsigned char* mask;
    const T* v;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&)[K]) const
    {
        const T o = x[r] + (dinv[r] * (b[r] - (T)s)) * omega;
        xn[r] = mask[r] ? v[r] + o : o;
    }
};

template <typename T>
struct EpiMasked {  // y = mask ? 0 : A x  (transfer followed by zero boundary values)
    const unsigned char* mask;
    T* y;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&)[K]) const { y[r] = mask[r] ? (T)0 : (T)s; }
};

template <typename T>
struct EpiMaskedAdd {  // x += mask ? 0 : A e   (prolongation + correction, MGPreconditionerInterface.java:171-174)
    const unsigned char* mask;
    T* x;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&)[K]) const
    {
        x[r] = x[r] + (mask[r] ? (T)0 : (T)s);
    }
};

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
// Kernel launch with the programmatic-stream-serialization attribute (PDL):
// the next kernel may be scheduled while this one drains; every solve-path
// kernel starts with griddepcontrol.wait.  JFEM_PDL=0 disables it.
bool use_pdl();

template <typename... KArgs, typename... Args>
void launch_ex(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = use_pdl() ? 1 : 0;
    JFG_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
    note_launch();
}

int sm_count();
// One-thread-per-row SpMVs with 16-bit columns use k_spmv_pipe (shared-memory
// stages) unless the environment variable JFEM_SPMV_PIPE=0 selects the
// register-only k_spmv.
bool spmv_pipe();
// k_spmv_pipe stage shape (measured on the Q2 512^2 level matrices): chunks of
// 8 entries for 2-byte values, 4 entries for FP32 and FP64 values; two stages.
template <typename VT>
constexpr int pipe_chunk() { return sizeof(VT) <= 2 ? 8 : 4; }
constexpr int kPipeStages = 2;

// The staged point-layout SpMV (k_spmv_pt) of a matrix with Matrix::st: a
// persistent grid of as many regular CTAs as stay resident beside the CTAs of
// the irregular rows (FP64 values: 2 CTAs per SM, others 4).
template <typename VT, typename XT, int NR, class Epi, class Fin, bool PF, int KIND>
void launch_pt_kind(cudaStream_t st, const Matrix* M, const VT* val, const XT* x, Epi epi, GridRed<NR, Fin> red,
                    const int* done)
{
    const int nreg = M->st_hi - M->st_lo;
    const int ntiles = (nreg + kPtRows - 1) / kPtRows;
    const int cps = sizeof(VT) == 8 ? 2 : kStCtasPerSm;
    const int nbr = std::max(1, std::min(ntiles, sm_count() * cps - M->st_nb_irr));
    const int smem = pt_smem<VT>(KIND == 1 ? 4 : 9);
    auto kern = k_spmv_pt<VT, XT, NR, Epi, Fin, PF, KIND>;
    if (smem > 48 * 1024) {
        static const bool set = [&] {
            JFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            return true;
        }();
        (void)set;
    }
    PtArgs a{M->st_S, M->st_S2, M->st_lo, nreg, M->st_ld, M->st_nirr, ntiles, M->st_irow.p, M->st_iptr.p,
             M->st_icol.p, std::is_same<VT, __half>::value ? M->hscale_inv : 1.0f, M->st_err.p};
    launch_ex(kern, dim3(nbr + M->st_nb_irr), dim3(kThreads), (size_t)smem, st, a, val, x, epi, red, done);
}

template <typename VT, typename XT, int NR, class Epi, class Fin, bool PF>
void launch_pt(cudaStream_t st, const Matrix* M, const VT* val, const XT* x, Epi epi, GridRed<NR, Fin> red,
               const int* done)
{
    switch (M->st_kind) {
    case 1: launch_pt_kind<VT, XT, NR, Epi, Fin, PF, 1>(st, M, val, x, epi, red, done); break;
    case 2: launch_pt_kind<VT, XT, NR, Epi, Fin, PF, 2>(st, M, val, x, epi, red, done); break;
    default: launch_pt_kind<VT, XT, NR, Epi, Fin, PF, 0>(st, M, val, x, epi, red, done); break;
    }
}

// PF: prefetch the matrix before the PDL wait (see k_spmv); only for
// matrices that are not written after set-up.
template <typename VT, typename XT, int NR, class Epi, class Fin = NoFin, bool PF = false>
void spmv_launch(cudaStream_t st, const Matrix* M, const VT* val, const XT* x, Epi epi, const Scratch& sc,
                 const int* done, Fin fin = Fin())
{
    if (M->rows == 0) return;
    GridRed<NR, Fin> red{sc.partials, sc.counter, fin};
    // the values-only point layouts, when the matrix has one in this value type:
    // transfers (kinds 1, 2) by the staged kernel for 4- and 2-byte values
    // (FP64 transfers measured faster in SELL-32), the 9-point kind by the
    // register kernel k_spmv_st (measured faster than the staged one) unless
    // the matrix was built with JFEM_ST_STAGED=1
    const bool pt_layout = M->st && val == LayoutVals<VT>::sell(M) && LayoutVals<VT>::st(M);
    if (pt_layout && ((M->st_kind != 0 && !std::is_same<VT, double>::value) || (M->st_kind == 0 && M->st_staged))) {
        launch_pt<VT, XT, NR, Epi, Fin, PF>(st, M, LayoutVals<VT>::st(M), x, epi, red, done);
        return;
    }
    if (pt_layout && M->st_kind == 0) {
        // persistent: as many regular CTAs as stay resident next to the irregular ones
        // (FP64 values: up to 128 registers, 2 CTAs per SM)
        const int nbr = std::max(1, std::min(M->st_nb_reg, sm_count() * (sizeof(VT) == 8 ? 2 : kStCtasPerSm) -
                                                                M->st_nb_irr));
        StArgs sa{M->st_S, M->st_lo, M->st_hi - M->st_lo, M->st_ld, M->st_nirr, nbr, M->st_irow.p, M->st_iptr.p,
                  M->st_icol.p, std::is_same<VT, __half>::value ? M->hscale_inv : 1.0f};
        launch_ex(k_spmv_st<VT, XT, NR, Epi, Fin, PF>, dim3(nbr + M->st_nb_irr), dim3(kThreads), 0, st, sa,
                  LayoutVals<VT>::st(M), x, epi, red, done);
        return;
    }
    SpmvArgs a{M->off.p, M->perm.p, M->col.p, M->nslices * kSliceRows, M->tpr_log2, M->col16.p,
               M->idx16 == 2 ? M->cbase.p : nullptr, std::is_same<VT, __half>::value ? M->hscale_inv : 1.0f};
    const dim3 g(M->nblocks), b(kThreads);
    if (M->idx16) {
        switch (M->tpr_log2) {
        case 0:
            if (spmv_pipe()) {
                launch_ex(k_spmv_pipe<VT, XT, NR, pipe_chunk<VT>(), kPipeStages, Epi, Fin>, g, b, 0, st, a, val, x,
                          epi, red, done);
                break;
            }
            launch_ex(k_spmv<VT, XT, NR, 1, Epi, Fin, true, false>, g, b, 0, st, a, val, x, epi, red, done);
            break;
        case 2: launch_ex(k_spmv<VT, XT, NR, 4, Epi, Fin, true, PF>, g, b, 0, st, a, val, x, epi, red, done); break;
        default: launch_ex(k_spmv<VT, XT, NR, 8, Epi, Fin, true, PF>, g, b, 0, st, a, val, x, epi, red, done); break;
        }
        return;
    }
    switch (M->tpr_log2) {
    case 0: launch_ex(k_spmv<VT, XT, NR, 1, Epi, Fin, false, false>, g, b, 0, st, a, val, x, epi, red, done); break;
    case 2: launch_ex(k_spmv<VT, XT, NR, 4, Epi, Fin, false, PF>, g, b, 0, st, a, val, x, epi, red, done); break;
    default: launch_ex(k_spmv<VT, XT, NR, 8, Epi, Fin, false, PF>, g, b, 0, st, a, val, x, epi, red, done); break;
    }
}

inline int vec_grid(int n)
{
    int g = (n + kThreads - 1) / kThreads;
    return g < 1 ? 1 : (g > kVecGrid ? kVecGrid : g);
}

template <int NR, class F, class Fin = NoFin>
void vec_launch(cudaStream_t st, int n, F f, const Scratch& sc, const int* done, Fin fin = Fin())
{
    GridRed<NR, Fin> red{sc.partials, sc.counter, fin};
    launch_ex(k_vec<NR, F, Fin>, dim3(vec_grid(n)), dim3(kThreads), 0, st, n, f, red, done);
}

template <class F>
void scalar_launch(cudaStream_t st, F f, const int* done)
{
    launch_ex(k_scalar<F>, dim3(1), dim3(1), 0, st, f, done);
}

// ---------------------------------------------------------------------------
// vector functors
// ---------------------------------------------------------------------------
template <typename T>
struct VCopy {
    const T* a;
    T* b;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { b[i] = a[i]; }
};
template <typename T>
struct VZero {
    T* a;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { a[i] = (T)0; }
};
template <typename T>
struct VDot {
    const T* a;
    const T* b;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const { acc[0] += (double)a[i] * (double)b[i]; }
};
template <typename T>
struct VScaleMul {  // y = (dinv * b) * omega      (first Jacobi sweep from a zero guess)
    const T* dinv;
    const T* b;
    T* y;
    T omega;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { y[i] = (T)0 + (dinv[i] * b[i]) * omega; }
};
template <typename T>
struct VCopyScaleMul {  // d = v and y = (dinv * v) * omega: the defect copy fused with the first sweep from zero
    const T* v;
    T* d;
    const T* dinv;
    T* y;
    T omega;
    template <int K> __device__ void operator()(int i, double (&)[K]) const
    {
        const T vi = v[i];
        d[i] = vi;
        y[i] = (T)0 + (dinv[i] * vi) * omega;
    }
};
template <typename A, typename B>
struct VCast {  // b = (B) a
    const A* a;
    B* b;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { b[i] = (B)a[i]; }
};
template <typename T>
struct VMul {  // y = d * x
    const T* d;
    const T* x;
    T* y;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { y[i] = d[i] * x[i]; }
};

}  // namespace jfg
