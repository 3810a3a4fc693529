// Multigrid V-cycle, FMG and smoothers on the device.
#include <cooperative_groups.h>

#include <algorithm>

#include "jfg_mg.cuh"
#include "jfg_gs.cuh"
#include "jfg_schwarz.cuh"

namespace cg = cooperative_groups;

namespace jfg {

namespace {

template <typename T>
__global__ void k_dinv(int n, const double* diag, T* dinv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = diag[i];
    if (fabs(d) < 1e-10) d = 1;          // JacobiSmoother.java:21-22
    dinv[i] = (T)(1.0 / d);
}

__global__ void k_mask(int nb, const int* bd, unsigned char* mask)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) mask[bd[i]] = 1;
}

template <typename T>
__global__ void k_cast(int64_t n, const double* a, T* b)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (T)a[i];
}

// x = Ainv * rhs with FP64 arithmetic; one warp per row.
template <typename T>
__global__ void k_coarse_gemv(int n, const double* __restrict__ ainv, const T* __restrict__ rhs, T* __restrict__ x,
                              const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0;
    for (int j = lane; j < n; j += 32) s += ainv[(size_t)row * n + j] * (double)rhs[j];
    s = warp_sum(s);
    if (lane == 0) x[row] = (T)s;
}

// defect rows touched by boundary columns: d[r] = v[r] - sum_j A[r, j] v[j]
template <typename T>
__global__ void k_bc_defect(int naff, const int* __restrict__ row, const int* __restrict__ ptr,
                            const int* __restrict__ col, const T* __restrict__ val, const T* __restrict__ v,
                            T* __restrict__ d, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= naff) return;
    int r = row[i];
    T s = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; k++) s += val[k] * v[col[k]];
    d[r] = v[r] - s;
}

// k_bc_defect, and the first Jacobi sweep from zero of those rows:
// y[r] = (dinv[r] * d[r]) * omega (the rest of y written by VCopyScaleMul)
template <typename T>
__global__ void k_bc_defect_scale(int naff, const int* __restrict__ row, const int* __restrict__ ptr,
                                  const int* __restrict__ col, const T* __restrict__ val, const T* __restrict__ v,
                                  T* __restrict__ d, const T* __restrict__ dinv, T* __restrict__ y, T omega,
                                  const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= naff) return;
    int r = row[i];
    T s = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; k++) s += val[k] * v[col[k]];
    const T dr = v[r] - s;
    d[r] = dr;
    y[r] = (T)0 + (dinv[r] * dr) * omega;
}

// out[bd] += v[bd]   (initial.add(iterate), initial = boundary copy of v)
template <typename T>
__global__ void k_bc_add(int nb, const int* __restrict__ bd, const T* __restrict__ v, T* __restrict__ out,
                         const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) out[bd[i]] = v[bd[i]] + out[bd[i]];
}

// Richardson update x += omega * r unless the level flag says "smooth"
template <typename T>
struct VRichardson {
    const T* r;
    T* x;
    T omega;
    const int* flag;
    template <int K> __device__ void operator()(int i, double (&)[K]) const
    {
        if (*flag) return;
        x[i] = x[i] + r[i] * omega;
    }
};

struct FinSmoothFlag {  // RichardsonSmoother.java:33-38: stop when ||r|| < 1e-10
    int* flag;
    __device__ void operator()(const double* t) const { *flag = sqrt(t[0]) < 1e-10 ? 1 : 0; }
};

inline unsigned nb(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Restriction whose epilogue also performs the first Jacobi sweep of the
// coarse level from a zero guess: b = mask ? 0 : R r ; xd = (dinv * b) * omega.
template <typename T>
struct EpiRestrictSweep {
    const unsigned char* mask;
    T* b;
    const T* dinv;
    T* xd;
    T omega;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&)[K]) const
    {
        T v = mask[r] ? (T)0 : (T)s;
        b[r] = v;
        xd[r] = (T)0 + (dinv[r] * v) * omega;
    }
};

// ---------------------------------------------------------------------------
// The tail of the V-cycle in one launch.  Below a few thousand rows every
// level's kernels are launch-latency bound (3.5-5 us each whatever their
// size), so the levels 0..tail run inside one thread-block cluster of
// C = 16 (or 8) CTAs that keeps the whole tail in distributed shared
// memory.  CTA c owns rows [c R_l, (c + 1) R_l) of level l (R_l =
// ceil(n_l / C)) and holds, in its shared memory:
//   * copied once per launch (before the wait for the preceding kernel):
//     its rows of every tail matrix -- A_l, the restriction R_l into level
//     l - 1 and the prolongation P_l from level l - 1 -- as ELL slices
//     (entry k of local row t at k * R + t, padding (column 0, value 0)),
//     and its rows of the Jacobi diagonal inverse and the Dirichlet mask;
//     a column is stored as (owning CTA << 12 | local row), so a product
//     reads x of another CTA straight from that CTA's shared memory
//     (mapa + ld.shared::cluster);
//   * the level vectors x, t, b, r of its rows.
// A phase (Jacobi sweep, residual, restriction with the fused first sweep of
// the coarser level, coarse FP64 solve, prolongation + correction) is one
// pass of each thread over its rows followed by a hardware cluster barrier
// (barrier.cluster arrive.release / wait.acquire): no software spin-wait,
// and no global-memory traffic inside the cycle.  The coarsest levels, when
// their rows fit next to the rest, are owned wholly by CTA 0 ("local"
// levels): a phase whose own level and the level the next phase reads are
// both local ends with a CTA barrier instead of a cluster barrier (the other
// CTAs have no rows there), and every CTA still meets every cluster barrier,
// so the sequence of cluster barriers is the same on all of them.  The level entered from
// above reads its restricted right-hand side from global memory and the
// result x of that level is written back at the end.  Row sums run in
// ascending column order from 0 with fused multiply-adds, as in the
// one-thread-per-row kernels.
constexpr int kTailMaxLevels = 8;         // coarse level included
constexpr int kTailMaxRowsPerCta = 4095;  // 12-bit local row of a packed column
constexpr int kTailThreads = 1024;
constexpr int kTailSmemBudget = 224 * 1024;
constexpr int kTailMetaInts = 23;         // per level: A, R, P (5 each), dinv, mask, rows per CTA, x, t, b, r, local
constexpr int kTailLocalRows = 1100;      // largest level owned wholly by CTA 0 (if the shared memory allows)

struct TailMat {
    int off_col, off_val;   // byte offsets of the column and value blocks in a CTA's shared memory
    int W, R, m;            // entries per row, rows per CTA, rows
    int xoff;               // byte offset of the vector the columns index (set per product)
};

template <typename T>
struct TailLevel {
    TailMat A, R, P;          // R: restriction into level l - 1, P: prolongation from level l - 1
    int Rl, n, runs;          // rows per CTA, rows, Jacobi sweeps
    int local;                // every row on CTA 0 (Rl == n)
    int off_dinv, off_mask, off_x, off_t, off_b, off_r;
    T omega;
};

template <typename T>
struct TailParams {
    TailLevel<T> lv[kTailMaxLevels];
    int top, n0;
    const double* ainv0;
    const T* b_top;           // the restricted right-hand side of level top (global)
    T* x_top;                 // its result (global)
    const int* done;
    const uint4* pkg;         // C blocks of pkg_bytes each
    int pkg_bytes;            // constant part per CTA, a multiple of 16
    int smem_bytes;           // package + vectors
};

__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, uint32_t rank)
{
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(local), "r"(rank));
    return a;
}
__device__ __forceinline__ float ld_cluster(uint32_t a, float)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ double ld_cluster(uint32_t a, double)
{
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
    return v;
}

// row sums of M times the distributed vector at byte offset M.xoff; f(t, s) per own row t
template <typename T, class F>
__device__ __forceinline__ void tail_spmv(unsigned char* sm, const TailMat& M, int c, F f)
{
    const uint16_t* col = reinterpret_cast<const uint16_t*>(sm + M.off_col);
    const T* val = reinterpret_cast<const T*>(sm + M.off_val);
    const uint32_t xb = smem_u32(sm + M.xoff);
    for (int t = threadIdx.x; t < M.R; t += blockDim.x) {
        if (c * M.R + t >= M.m) break;
        T s = 0;
        for (int k0 = 0; k0 < M.W; k0 += 9) {
            T v[9], xv[9];
#pragma unroll
            for (int u = 0; u < 9; u++) {
                const int k = k0 + u;
                if (k < M.W) {
                    const unsigned q = col[k * M.R + t];
                    v[u] = val[k * M.R + t];
                    xv[u] = ld_cluster(cluster_addr(xb + (q & 0xFFFu) * (unsigned)sizeof(T), q >> 12), T());
                } else {
                    v[u] = 0;
                    xv[u] = 0;
                }
            }
#pragma unroll
            for (int u = 0; u < 9; u++) s += v[u] * xv[u];
        }
        f(t, s);
    }
}

template <class F>
__device__ __forceinline__ void tail_own(int R, int n, int c, F f)
{
    for (int t = threadIdx.x; t < R; t += blockDim.x) {
        if (c * R + t >= n) break;
        f(t);
    }
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_mg_tail(const __grid_constant__ TailParams<T> P)
{
    extern __shared__ __align__(16) unsigned char sm[];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    // end of a phase: a CTA barrier when the phase's level and the level the
    // next phase reads are both local (CTA 0 alone), else a cluster barrier
    auto phase_end = [&](bool local) {
        if (local)
            __syncthreads();
        else
            cl.sync();
    };
    // the matrices, diagonals and masks do not change after set-up: copy them
    // before waiting for the preceding kernel
    {
        const uint4* src = P.pkg + (size_t)c * (P.pkg_bytes / 16);
        uint4* dst = reinterpret_cast<uint4*>(sm);
        for (int i = threadIdx.x; i < P.pkg_bytes / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    pdl_wait();
    if (P.done && *P.done) return;           // the same answer for every CTA of the cluster
    auto vec = [&](int off) { return reinterpret_cast<T*>(sm + off); };
    {   // the restricted right-hand side of the top level, own rows
        const TailLevel<T>& L = P.lv[P.top];
        T* b = vec(L.off_b);
        tail_own(L.Rl, L.n, c, [&](int t) { b[t] = P.b_top[c * L.Rl + t]; });
    }
    __syncthreads();
    for (int l = P.top; l >= 1; l--) {
        const TailLevel<T>& L = P.lv[l];
        const T* b = vec(L.off_b);
        const T* dinv = vec(L.off_dinv);
        const T om = L.omega;
        // the first sweep from the zero guess lands where the last one ends in x
        T* cur = vec((L.runs % 2 == 1) ? L.off_x : L.off_t);
        int cur_off = (L.runs % 2 == 1) ? L.off_x : L.off_t;
        const bool loc = L.local != 0;
        if (l == P.top) {   // below the top the restriction phase did it
            tail_own(L.Rl, L.n, c, [&](int t) { cur[t] = (T)0 + (dinv[t] * b[t]) * om; });
            phase_end(loc);
        }
        for (int k = 1; k < L.runs; k++) {
            const int alt_off = cur_off == L.off_x ? L.off_t : L.off_x;
            T* alt = vec(alt_off);
            TailMat A = L.A;
            A.xoff = cur_off;
            const T* cu = cur;
            tail_spmv<T>(sm, A, c, [&](int t, T s) { alt[t] = cu[t] + (dinv[t] * (b[t] - s)) * om; });
            phase_end(loc);
            cur = alt;
            cur_off = alt_off;
        }
        {   // residual r = b - A x
            T* r = vec(L.off_r);
            TailMat A = L.A;
            A.xoff = L.off_x;
            tail_spmv<T>(sm, A, c, [&](int t, T s) { r[t] = b[t] - s; });
            phase_end(loc);   // level l - 1 is local whenever level l is
        }
        {   // restriction into level l - 1 with zero boundary values (and its fused first sweep)
            const TailLevel<T>& Cl = P.lv[l - 1];
            TailMat R = L.R;
            R.xoff = L.off_r;
            T* bc = vec(Cl.off_b);
            const unsigned char* mask = sm + Cl.off_mask;
            if (l - 1 >= 1) {
                const T* dc = vec(Cl.off_dinv);
                T* xd = vec((Cl.runs % 2 == 1) ? Cl.off_x : Cl.off_t);
                const T oc = Cl.omega;
                tail_spmv<T>(sm, R, c, [&](int t, T s) {
                    const T v = mask[t] ? (T)0 : s;
                    bc[t] = v;
                    xd[t] = (T)0 + (dc[t] * v) * oc;
                });
            } else {
                tail_spmv<T>(sm, R, c, [&](int t, T s) { bc[t] = mask[t] ? (T)0 : s; });
            }
            // a local level l - 1 is read next by CTA 0 alone; the other CTAs
            // keep their r rows (read here remotely) until the next cluster
            // barrier, which comes before any of them writes level l again
            phase_end(Cl.local != 0);
        }
    }
    {   // coarsest level: x0 = Ainv * b0 in FP64, one warp per own row (the order of k_coarse_gemv)
        const TailLevel<T>& L0 = P.lv[0];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const uint32_t bb = smem_u32(sm + L0.off_b);
        T* x0 = vec(L0.off_x);
        for (int t = w; t < L0.Rl; t += blockDim.x >> 5) {
            const int row = c * L0.Rl + t;
            if (row >= P.n0) break;
            double s = 0;
            for (int j = lane; j < P.n0; j += 32) {
                const int owner = j / L0.Rl, loc = j - owner * L0.Rl;
                s += P.ainv0[(size_t)row * P.n0 + j] *
                     (double)ld_cluster(cluster_addr(bb + loc * (unsigned)sizeof(T), owner), T());
            }
            s = warp_sum(s);
            if (lane == 0) x0[t] = (T)s;
        }
        phase_end(L0.local != 0 && (P.top < 1 || P.lv[1].local != 0));
    }
    for (int l = 1; l <= P.top; l++) {
        const TailLevel<T>& L = P.lv[l];
        const T* b = vec(L.off_b);
        const T* dinv = vec(L.off_dinv);
        const T om = L.omega;
        {   // x += mask ? 0 : P x_{l-1}
            T* x = vec(L.off_x);
            const unsigned char* mask = sm + L.off_mask;
            TailMat Pm = L.P;
            Pm.xoff = P.lv[l - 1].off_x;
            tail_spmv<T>(sm, Pm, c, [&](int t, T s) { x[t] = x[t] + (mask[t] ? (T)0 : s); });
            phase_end(L.local != 0);
        }
        // the last phase of level l is read next by the prolongation into
        // level l + 1 (or, at the top, by the copy-out of the own rows)
        const bool loc_next = L.local != 0 && (l == P.top || P.lv[l + 1].local != 0);
        int cur_off = L.off_x;
        for (int k = 0; k < L.runs; k++) {
            const int alt_off = cur_off == L.off_x ? L.off_t : L.off_x;
            const T* cu = vec(cur_off);
            T* alt = vec(alt_off);
            TailMat A = L.A;
            A.xoff = cur_off;
            tail_spmv<T>(sm, A, c, [&](int t, T s) { alt[t] = cu[t] + (dinv[t] * (b[t] - s)) * om; });
            const bool last = k == L.runs - 1 && alt_off == L.off_x;
            phase_end(last ? loc_next : L.local != 0);
            cur_off = alt_off;
        }
        if (cur_off != L.off_x) {
            const T* cu = vec(cur_off);
            T* x = vec(L.off_x);
            tail_own(L.Rl, L.n, c, [&](int t) { x[t] = cu[t]; });
            phase_end(loc_next);
        }
    }
    {   // the result of the top level back to global memory
        const TailLevel<T>& L = P.lv[P.top];
        const T* x = vec(L.off_x);
        tail_own(L.Rl, L.n, c, [&](int t) { P.x_top[c * L.Rl + t] = x[t]; });
    }
}

template <typename T>
void launch_tail(const TailParams<T>& p, int ctas, cudaStream_t st)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = (size_t)p.smem_bytes;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    int na = 1;
    if (use_pdl()) {
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        na = 2;
    }
    cfg.attrs = at;
    cfg.numAttrs = na;
    JFG_CUDA(cudaLaunchKernelEx(&cfg, k_mg_tail<T>, p));
    note_launch();
}

// Largest cluster (16, else 8 CTAs) that can be resident with `smem` bytes
// of dynamic shared memory per CTA; 0 when none can.
template <typename T>
int tail_cluster_size(size_t smem)
{
    // the same cap for every hierarchy (the attribute belongs to the kernel, not to one launch)
    JFG_CUDA(cudaFuncSetAttribute(k_mg_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTailSmemBudget));
    JFG_CUDA(cudaFuncSetAttribute(k_mg_tail<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    for (int ctas : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ctas);
        cfg.blockDim = dim3(kTailThreads);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = ctas;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, k_mg_tail<T>, &cfg) == cudaSuccess && nc >= 1) return ctas;
        cudaGetLastError();
    }
    return 0;
}

}  // namespace

template <typename T>
void MGImpl<T>::init(Context* ctx, int levels, Matrix* const* As, Matrix* const* Ps, const int* const* bdry,
                     const int* nbdry, const SmootherDesc* sms, int cycles_, int use_fmg_, int vfmt)
{
    c = ctx;
    L = levels;
    cycles = cycles_;
    use_fmg = use_fmg_;
    cudaStream_t st = c->stream;
    A.assign(As, As + L);
    P.assign(L, nullptr);
    R.assign(L, nullptr);
    n.resize(L);
    sm.assign(sms, sms + L);
    x = std::vector<DevBuf<T>>(L);
    t = std::vector<DevBuf<T>>(L);
    b = std::vector<DevBuf<T>>(L);
    r = std::vector<DevBuf<T>>(L);
    fr = std::vector<DevBuf<T>>(L);
    dinv = std::vector<DevBuf<T>>(L);
    mask = std::vector<DevBuf<unsigned char>>(L);
    for (int l = 0; l < L; l++) {
        JFG_CHECK(A[l] && A[l]->rows == A[l]->cols, JFG_ERR_BAD_ARG, "level matrix missing or not square");
        n[l] = A[l]->rows;
        if (l < L - 1) {
            P[l] = Ps[l];
            JFG_CHECK(P[l], JFG_ERR_BAD_ARG, "prolongation missing");
            JFG_CHECK(P[l]->rows == As[l + 1]->rows && P[l]->cols == As[l]->rows, JFG_ERR_BAD_ARG,
                      "prolongation shape does not match the level sizes");
            R[l] = matrix_transpose(P[l]);
            // Q1 grids whose level matrices carry the 9-point layout with
            // strides S (coarse) and 2 S - 1 (fine): values-only transfers
            // (JFEM_MG_TRANSFER=0 keeps them in SELL-32)
            const Matrix* Ac = As[l];
            const Matrix* Af = As[l + 1];
            const char* et = getenv("JFEM_MG_TRANSFER");
            if (!(et && et[0] == '0') && Ac->st && Af->st && Ac->st_kind == 0 && Af->st_kind == 0 &&
                Af->st_S == 2 * Ac->st_S - 1) {
                matrix_build_transfer_layout(P[l], 1, Af->st_S, Ac->st_S);
                matrix_build_transfer_layout(R[l], 2, Ac->st_S, Af->st_S);
            }
        }
        if (std::is_same<T, float>::value) {
            vbf16 = vfmt == 1 ? 1 : 0;
            vfp16 = vfmt == 2 ? 1 : 0;
            auto ensure = vbf16 ? matrix_ensure_bf16 : (vfp16 ? matrix_ensure_fp16 : matrix_ensure_fp32);
            ensure(A[l]);
            if (l < L - 1) {
                ensure(P[l]);
                ensure(R[l]);
            }
        }
        size_t m = (size_t)n[l];
        x[l].alloc(m);
        t[l].alloc(m);
        b[l].alloc(m);
        r[l].alloc(m);
        fr[l].alloc(m);
        dinv[l].alloc(m);
        mask[l].alloc(m);
        if (m) {
            k_dinv<T><<<nb(m), 256, 0, st>>>((int)m, A[l]->diag.p, dinv[l].p);
            JFG_CUDA(cudaMemsetAsync(mask[l].p, 0, m, st));
            JFG_CUDA(cudaMemsetAsync(x[l].p, 0, m * sizeof(T), st));
        }
        JFG_CHECK(nbdry[l] >= 0 && (nbdry[l] == 0 || bdry[l]), JFG_ERR_BAD_ARG, "bad boundary list");
        for (int i = 0; i < nbdry[l]; i++)
            JFG_CHECK(bdry[l][i] >= 0 && bdry[l][i] < n[l], JFG_ERR_BAD_ARG, "boundary node out of range");
        if (nbdry[l]) {
            DevBuf<int> d_bd;
            d_bd.alloc(nbdry[l]);
            JFG_CUDA(cudaMemcpyAsync(d_bd.p, bdry[l], sizeof(int) * nbdry[l], cudaMemcpyHostToDevice, st));
            k_mask<<<nb(nbdry[l]), 256, 0, st>>>(nbdry[l], d_bd.p, mask[l].p);
            JFG_CUDA(cudaStreamSynchronize(st));
        }
        JFG_CUDA(cudaGetLastError());
    }
    // finest boundary list and the rows with entries in boundary columns
    int Lf = L - 1;
    nbd_fine = nbdry[Lf];
    bd_fine.alloc(nbd_fine ? nbd_fine : 1);
    if (nbd_fine)
        JFG_CUDA(cudaMemcpyAsync(bd_fine.p, bdry[Lf], sizeof(int) * nbd_fine, cudaMemcpyHostToDevice, st));
    {
        Matrix* Af = A[Lf];
        std::vector<int> hp(Af->rows + 1);
        std::vector<int> hc((size_t)Af->nnz + 1);
        std::vector<double> hv((size_t)Af->nnz + 1);
        JFG_CUDA(cudaMemcpyAsync(hp.data(), Af->csr_ptr.p, sizeof(int) * (Af->rows + 1), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(hc.data(), Af->csr_col.p, sizeof(int) * Af->nnz, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(hv.data(), Af->csr_val.p, sizeof(double) * Af->nnz, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        std::vector<char> isbd(Af->rows, 0);
        for (int i = 0; i < nbd_fine; i++) {
            if (isbd[bdry[Lf][i]]) bd_unique = false;
            isbd[bdry[Lf][i]] = 1;
        }
        std::vector<int> arow, aptr{0}, acol;
        std::vector<T> aval;
        for (int rr = 0; rr < Af->rows; rr++) {
            bool any = false;
            for (int k = hp[rr]; k < hp[rr + 1]; k++)
                if (hv[k] != 0.0 && isbd[hc[k]]) {
                    acol.push_back(hc[k]);
                    aval.push_back((T)hv[k]);
                    any = true;
                }
            if (any) {
                arow.push_back(rr);
                aptr.push_back((int)acol.size());
            }
        }
        naff = (int)arow.size();
        aff_row.alloc(naff ? naff : 1);
        aff_ptr.alloc(naff + 1);
        aff_col.alloc(acol.size() ? acol.size() : 1);
        aff_val.alloc(aval.size() ? aval.size() : 1);
        if (naff) {
            JFG_CUDA(cudaMemcpyAsync(aff_row.p, arow.data(), sizeof(int) * naff, cudaMemcpyHostToDevice, st));
            JFG_CUDA(cudaMemcpyAsync(aff_ptr.p, aptr.data(), sizeof(int) * (naff + 1), cudaMemcpyHostToDevice, st));
            JFG_CUDA(cudaMemcpyAsync(aff_col.p, acol.data(), sizeof(int) * acol.size(), cudaMemcpyHostToDevice, st));
            JFG_CUDA(cudaMemcpyAsync(aff_val.p, aval.data(), sizeof(T) * aval.size(), cudaMemcpyHostToDevice, st));
        }
        JFG_CUDA(cudaStreamSynchronize(st));
    }
    // coarsest level: dense inverse computed on the device in FP64
    int n0 = n[0];
    ainv0.alloc((size_t)n0 * n0);
    {
        DevBuf<double> dense;
        dense.alloc((size_t)n0 * n0);
        JFG_CUDA(cudaMemsetAsync(dense.p, 0, sizeof(double) * n0 * n0, st));
        // scatter the level-0 CSR into the dense array
        std::vector<int> hp(n0 + 1);
        std::vector<int> hc((size_t)A[0]->nnz + 1);
        std::vector<double> hv((size_t)A[0]->nnz + 1);
        JFG_CUDA(cudaMemcpyAsync(hp.data(), A[0]->csr_ptr.p, sizeof(int) * (n0 + 1), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(hc.data(), A[0]->csr_col.p, sizeof(int) * A[0]->nnz, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(hv.data(), A[0]->csr_val.p, sizeof(double) * A[0]->nnz, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        std::vector<double> hd((size_t)n0 * n0, 0.0);
        for (int rr = 0; rr < n0; rr++)
            for (int k = hp[rr]; k < hp[rr + 1]; k++) hd[(size_t)rr * n0 + hc[k]] += hv[k];
        JFG_CUDA(cudaMemcpyAsync(dense.p, hd.data(), sizeof(double) * hd.size(), cudaMemcpyHostToDevice, st));
        coarse_status = dense_inverse_device(c, n0, dense.p, ainv0.p);
    }
    flags.alloc(L);
    zero_flag.alloc(1);
    JFG_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(int) * L, st));
    JFG_CUDA(cudaMemsetAsync(zero_flag.p, 0, sizeof(int), st));
    build_tail();
    JFG_CUDA(cudaStreamSynchronize(st));
}

// Host copy of a matrix's merged CSR.
static void csr_to_host(const Matrix* M, std::vector<int>& hp, std::vector<int>& hc, std::vector<double>& hv,
                        cudaStream_t st)
{
    hp.assign(M->rows + 1, 0);
    hc.assign((size_t)M->nnz + 1, 0);
    hv.assign((size_t)M->nnz + 1, 0.0);
    JFG_CUDA(cudaMemcpyAsync(hp.data(), M->csr_ptr.p, sizeof(int) * (M->rows + 1), cudaMemcpyDeviceToHost, st));
    if (M->nnz) {
        JFG_CUDA(cudaMemcpyAsync(hc.data(), M->csr_col.p, sizeof(int) * M->nnz, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(hv.data(), M->csr_val.p, sizeof(double) * M->nnz, cudaMemcpyDeviceToHost, st));
    }
    JFG_CUDA(cudaStreamSynchronize(st));
}

// Picks the levels 0..tail of the one-launch V-cycle tail (k_mg_tail) and
// builds its shared-memory package: the largest top level such that the
// levels 1..top are Jacobi-smoothed and lie below the finest level, every
// level has at most kTailMaxRowsPerCta rows per CTA, and the package plus
// the level vectors fit kTailSmemBudget bytes per CTA of a resident
// cluster.  JFEM_MG_TAIL=0 turns it off.
template <typename T>
void MGImpl<T>::build_tail()
{
    tail = -1;
    const char* e = getenv("JFEM_MG_TAIL");
    if (e && e[0] == '0') return;
    cudaStream_t st = c->stream;
    int cand = -1;
    for (int l = 1; l < L - 1 && l < kTailMaxLevels; l++) {
        if (sm[l].kind != JFG_SMOOTH_JACOBI || sm[l].runs < 1 || (n[l] + 15) / 16 > kTailMaxRowsPerCta) break;
        cand = l;
    }
    if (cand < 1) return;
    struct HostMat {
        std::vector<int> p, c;
        std::vector<double> v;
        int rows = 0, W = 1;
    };
    auto rounded = [&](const Matrix* M, double a) -> double {   // the value the level's products read
        if constexpr (std::is_same<T, float>::value) {
            if (vbf16) return (double)__bfloat162float(__float2bfloat16_rn((float)a));
            if (vfp16) {
                const double sc = 1.0 / (double)M->hscale_inv;
                return (double)__half2float(__double2half(a * sc)) / sc;
            }
            return (double)(float)a;
        }
        return a;
    };
    std::vector<HostMat> hm(3 * (cand + 1));      // per level l >= 1: A_l, R (into l-1), P (from l-1)
    auto load = [&](HostMat& h, const Matrix* M) {
        csr_to_host(M, h.p, h.c, h.v, st);
        h.rows = M->rows;
        for (int r = 0; r < M->rows; r++) h.W = std::max(h.W, h.p[r + 1] - h.p[r]);
        for (int k = 0; k < (int)M->nnz; k++) h.v[k] = rounded(M, h.v[k]);
    };
    for (int l = 1; l <= cand; l++) {
        load(hm[3 * l], A[l]);
        load(hm[3 * l + 1], R[l - 1]);
        load(hm[3 * l + 2], P[l - 1]);
    }
    std::vector<double> hdinv;
    auto al16 = [](size_t b) { return (b + 15) / 16 * 16; };
    int loc_rows = 0;                                  // levels with at most this many rows are local (CTA 0)
    auto rows_per = [&](int l, int C) { return n[l] <= loc_rows ? n[l] : (n[l] + C - 1) / C; };
    // byte sizes: constant package, then vectors
    auto sizes = [&](int top, int C, size_t& pkg, size_t& total) {
        pkg = 0;
        for (int l = 0; l <= top; l++) {
            const size_t Rl = (size_t)rows_per(l, C);
            if (l >= 1) {
                const size_t Rc = (size_t)rows_per(l - 1, C);
                const HostMat &a = hm[3 * l], &r = hm[3 * l + 1], &p = hm[3 * l + 2];
                pkg += al16(Rl * a.W * 2) + al16(Rl * a.W * sizeof(T));
                pkg += al16(Rc * r.W * 2) + al16(Rc * r.W * sizeof(T));
                pkg += al16(Rl * p.W * 2) + al16(Rl * p.W * sizeof(T));
                pkg += al16(Rl * sizeof(T));                 // dinv
            }
            pkg += al16(Rl);                                 // mask
        }
        total = pkg;
        for (int l = 0; l <= top; l++) total += 4 * al16((size_t)rows_per(l, C) * sizeof(T));
    };
    int top = cand, C = 0;
    size_t pkg_b = 0, tot_b = 0;
    for (; top >= 1; top--) {
        for (int cs : {16, 8}) {
            if ((n[top] + cs - 1) / cs > kTailMaxRowsPerCta) continue;
            sizes(top, cs, pkg_b, tot_b);
            if (tot_b > (size_t)kTailSmemBudget) continue;
            if (tail_cluster_size<T>(tot_b) >= cs) {
                C = cs;
                break;
            }
        }
        if (C) break;
    }
    if (top < 1 || !C) return;
    {   // the largest set of coarsest levels that CTA 0 can own with the cluster still resident
        const char* le = getenv("JFEM_MG_TAIL_LOCAL");
        if (!(le && le[0] == '0')) {
            for (int l = top; l >= 0; l--) {
                if (n[l] > kTailLocalRows) continue;
                loc_rows = n[l];
                sizes(top, C, pkg_b, tot_b);
                if (tot_b <= (size_t)kTailSmemBudget && tail_cluster_size<T>(tot_b) >= C) break;
                loc_rows = 0;
            }
        }
    }
    sizes(top, C, pkg_b, tot_b);
    // host copies of the diagonal inverses and masks
    std::vector<std::vector<T>> dv(top + 1);
    std::vector<std::vector<unsigned char>> mk(top + 1);
    for (int l = 0; l <= top; l++) {
        dv[l].resize(n[l]);
        mk[l].resize(n[l]);
        if (n[l]) {
            JFG_CUDA(cudaMemcpyAsync(dv[l].data(), dinv[l].p, sizeof(T) * n[l], cudaMemcpyDeviceToHost, st));
            JFG_CUDA(cudaMemcpyAsync(mk[l].data(), mask[l].p, n[l], cudaMemcpyDeviceToHost, st));
        }
    }
    JFG_CUDA(cudaStreamSynchronize(st));
    std::vector<unsigned char> pkg(pkg_b * C, 0);
    tail_meta.assign(kTailMetaInts * (top + 1), 0);
    size_t off = 0;
    // one matrix: rows of `row_level` owned per CTA, columns packed in the ownership of `col_level`
    auto put_mat = [&](const HostMat& h, int row_level, int col_level, int* meta) {
        const int Rr = rows_per(row_level, C), Rc = rows_per(col_level, C);
        const size_t bc = al16((size_t)Rr * h.W * 2), bv = al16((size_t)Rr * h.W * sizeof(T));
        meta[0] = (int)off;
        meta[1] = (int)(off + bc);
        meta[2] = h.W;
        meta[3] = Rr;
        meta[4] = h.rows;
        for (int cc = 0; cc < C; cc++) {
            uint16_t* col = reinterpret_cast<uint16_t*>(pkg.data() + cc * pkg_b + off);
            T* val = reinterpret_cast<T*>(pkg.data() + cc * pkg_b + off + bc);
            for (int t = 0; t < Rr; t++) {
                const int r = cc * Rr + t;
                const int a = r < h.rows ? h.p[r] : 0, len = r < h.rows ? h.p[r + 1] - h.p[r] : 0;
                for (int k = 0; k < h.W; k++) {
                    uint16_t q = 0;
                    double v = 0.0;
                    if (k < len) {
                        const int j = h.c[a + k];
                        q = (uint16_t)(((j / Rc) << 12) | (j % Rc));
                        v = h.v[a + k];
                    }
                    col[(size_t)k * Rr + t] = q;
                    val[(size_t)k * Rr + t] = (T)v;
                }
            }
        }
        off += bc + bv;
    };
    for (int l = 0; l <= top; l++) {
        int* meta = &tail_meta[kTailMetaInts * l];
        const int Rl = rows_per(l, C);
        if (l >= 1) {
            put_mat(hm[3 * l], l, l, meta);
            put_mat(hm[3 * l + 1], l - 1, l, meta + 5);
            put_mat(hm[3 * l + 2], l, l - 1, meta + 10);
            meta[15] = (int)off;                          // dinv
            for (int cc = 0; cc < C; cc++) {
                T* d = reinterpret_cast<T*>(pkg.data() + cc * pkg_b + off);
                for (int t = 0; t < Rl && cc * Rl + t < n[l]; t++) d[t] = dv[l][cc * Rl + t];
            }
            off += al16((size_t)Rl * sizeof(T));
        }
        meta[16] = (int)off;                              // mask
        for (int cc = 0; cc < C; cc++)
            for (int t = 0; t < Rl && cc * Rl + t < n[l]; t++) pkg[cc * pkg_b + off + t] = mk[l][cc * Rl + t];
        off += al16((size_t)Rl);
        meta[17] = Rl;
        meta[22] = n[l] <= loc_rows ? 1 : 0;
    }
    JFG_CHECK(off == pkg_b, JFG_ERR_CUDA, "tail package layout mismatch");
    for (int l = 0; l <= top; l++) {                      // vectors x, t, b, r
        int* meta = &tail_meta[kTailMetaInts * l];
        const size_t vb = al16((size_t)rows_per(l, C) * sizeof(T));
        for (int q = 0; q < 4; q++) {
            meta[18 + q] = (int)off;
            off += vb;
        }
    }
    JFG_CHECK(off == tot_b, JFG_ERR_CUDA, "tail vector layout mismatch");
    tail_pkg.alloc(pkg.size() / 16);
    JFG_CUDA(cudaMemcpyAsync(tail_pkg.p, pkg.data(), pkg.size(), cudaMemcpyHostToDevice, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    tail_pkg_bytes = (int)pkg_b;
    tail_smem_bytes = (int)tot_b;
    tail_ctas = C;
    tail = top;
}

template <typename T>
int MGImpl<T>::max_blocks() const
{
    int m = kVecGrid;
    for (int l = 0; l < L; l++) {
        m = std::max(m, A[l]->nblocks);
        if (P[l]) m = std::max(m, P[l]->nblocks);
        if (R[l]) m = std::max(m, R[l]->nblocks);
    }
    return m;
}

// y-epilogue SpMV on a level matrix in the hierarchy's value type (FP64,
// FP32, or BF16 values with FP32 vectors)
template <typename T, int NR, class Epi, class Fin = NoFin>
static void mg_spmv(const MGImpl<T>& g, cudaStream_t st, const Matrix* M, const T* x, Epi epi, const Scratch& sc,
                    const int* done, Fin fin = Fin())
{
    // the hierarchy's matrices are fixed after init: prefetched before the PDL wait
    if constexpr (std::is_same<T, float>::value) {
        if (g.vbf16) {
            spmv_launch<__nv_bfloat16, float, NR, Epi, Fin, true>(st, M, M->val16.p, x, epi, sc, done, fin);
            return;
        }
        if (g.vfp16) {
            spmv_launch<__half, float, NR, Epi, Fin, true>(st, M, M->valh.p, x, epi, sc, done, fin);
            return;
        }
    }
    spmv_launch<T, T, NR, Epi, Fin, true>(st, M, vals_of<T>(M), x, epi, sc, done, fin);
}

template <typename T>
void MGImpl<T>::coarse(const T* rhs, T* out, const int* done, cudaStream_t st)
{
    int n0 = n[0];
    launch_ex(k_coarse_gemv<T>, dim3((n0 + 7) / 8), dim3(256), 0, st, n0, (const double*)ainv0.p, rhs, out, done);
}

// Smoother.smooth on level l with rhs; the result ends in x[l].
template <typename T>
void MGImpl<T>::smooth(int l, const T* rhs, bool xzero, const Scratch& sc, const int* done, cudaStream_t st,
                       bool first_sweep_done, T* dest)
{
    const SmootherDesc& d = sm[l];
    Matrix* M = A[l];
    int m = n[l];
    if (dest && d.kind == JFG_SMOOTH_JACOBI && d.runs >= 1 && !xzero) {
        // the result goes to dest instead of x[l]: the last sweep writes it there
        T om = (T)d.omega;
        T* cur = x[l].p;
        T* alt = t[l].p;
        for (int k = 0; k < d.runs; k++) {
            T* o = (k == d.runs - 1) ? dest : alt;
            if (k == d.runs - 1 && bc_src && l == L - 1) {
                mg_spmv<T, 0>(*this, st, M, cur, EpiJacobiBc<T>{cur, rhs, dinv[l].p, o, om, mask[l].p, bc_src}, sc,
                              done);
                bc_done = true;
            } else {
                mg_spmv<T, 0>(*this, st, M, cur, EpiJacobi<T>{cur, rhs, dinv[l].p, o, om}, sc, done);
            }
            alt = cur;
            cur = o;
        }
        return;
    }
    if (dest) {
        smooth(l, rhs, xzero, sc, done, st, first_sweep_done, nullptr);
        vec_launch<0>(st, m, VCopy<T>{x[l].p, dest}, sc, done);
        return;
    }
    if (d.runs <= 0) {
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[l].p}, sc, done);
        return;
    }
    if (d.kind == JFG_SMOOTH_JACOBI) {
        T om = (T)d.omega;
        int k = 0;
        T* cur = x[l].p;
        T* alt = t[l].p;
        if (xzero) {
            // first sweep from zero: x = (dinv * b) * omega; choose its target so
            // that the last sweep lands in x[l] (already done by the restriction
            // epilogue when first_sweep_done)
            T* dst = (d.runs % 2 == 1) ? x[l].p : t[l].p;
            if (!first_sweep_done) vec_launch<0>(st, m, VScaleMul<T>{dinv[l].p, rhs, dst, om}, sc, done);
            cur = dst;
            alt = (dst == x[l].p) ? t[l].p : x[l].p;
            k = 1;
        }
        for (; k < d.runs; k++) {
            mg_spmv<T, 0>(*this, st, M, cur, EpiJacobi<T>{cur, rhs, dinv[l].p, alt, om}, sc, done);
            std::swap(cur, alt);
        }
        if (cur != x[l].p) vec_launch<0>(st, m, VCopy<T>{cur, x[l].p}, sc, done);
    } else if (d.kind == JFG_SMOOTH_SCHWARZ) {
        // SchwarzSmoother.smooth (schwarz/SchwarzSmoother.java:21-43)
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[l].p}, sc, done);
        d.schwarz->smooth<T>(d.runs, rhs, x[l].p, sc, done, st);
    } else if (d.kind == JFG_SMOOTH_FBGS) {
        // ForwardBackwardGaussSeidelSmoother.smooth: x += L^-1 D U^-1 (b - A x)
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[l].p}, sc, done);
        for (int k = 0; k < d.runs; k++) {
            mg_spmv<T, 0>(*this, st, M, x[l].p, EpiResid<T>{rhs, r[l].p}, sc, done);
            d.gs->backward<T>(r[l].p, t[l].p, done, st);
            d.gs->forward_fbgs<T>(t[l].p, r[l].p, x[l].p, done, st);
        }
    } else if (d.kind == JFG_SMOOTH_GS) {
        // GaussSeidelSmoother.smooth: x = (L + D)^-1 (b - R x)
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[l].p}, sc, done);
        for (int k = 0; k < d.runs; k++) {
            d.gs->strict_upper<T>(rhs, x[l].p, t[l].p, done, st);
            d.gs->forward<T>(t[l].p, x[l].p, done, st);
        }
    } else {
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[l].p}, sc, done);
        for (int k = 0; k < d.runs; k++) {
            mg_spmv<T, 1>(*this, st, M, x[l].p, EpiResid<T>{rhs, r[l].p}, sc, done,
                                 FinSmoothFlag{flags.p + l});
            vec_launch<0>(st, m, VRichardson<T>{r[l].p, x[l].p, (T)d.omega, flags.p + l}, sc, done);
        }
    }
}

template <typename T>
void MGImpl<T>::run_tail(bool first_sweep_done, const int* done, cudaStream_t st)
{
    (void)first_sweep_done;     // the tail redoes the top level's first sweep from b
    TailParams<T> p = {};
    p.top = tail;
    p.n0 = n[0];
    p.ainv0 = ainv0.p;
    p.b_top = b[tail].p;
    p.x_top = x[tail].p;
    p.done = done;
    p.pkg = tail_pkg.p;
    p.pkg_bytes = tail_pkg_bytes;
    p.smem_bytes = tail_smem_bytes;
    for (int l = 0; l <= tail; l++) {
        const int* m = &tail_meta[kTailMetaInts * l];
        auto& Lv = p.lv[l];
        Lv.A = TailMat{m[0], m[1], m[2], m[3], m[4], 0};
        Lv.R = TailMat{m[5], m[6], m[7], m[8], m[9], 0};
        Lv.P = TailMat{m[10], m[11], m[12], m[13], m[14], 0};
        Lv.off_dinv = m[15];
        Lv.off_mask = m[16];
        Lv.Rl = m[17];
        Lv.local = m[22];
        Lv.off_x = m[18];
        Lv.off_t = m[19];
        Lv.off_b = m[20];
        Lv.off_r = m[21];
        Lv.n = n[l];
        Lv.runs = sm[l].runs;
        Lv.omega = (T)sm[l].omega;
    }
    launch_tail(p, tail_ctas, st);
}

// mgStepV (MGPreconditionerInterface.java:125-198): guess in x[l] (or zero),
// rhs given; result in x[l].
template <typename T>
void MGImpl<T>::vstep(int l, const T* rhs, bool xzero, const Scratch& sc, const int* done, cudaStream_t st,
                      bool first_sweep_done, T* dest)
{
    if (dest && l == 0) {
        vstep(l, rhs, xzero, sc, done, st, first_sweep_done, nullptr);
        vec_launch<0>(st, n[0], VCopy<T>{x[0].p, dest}, sc, done);
        return;
    }
    if (l == tail && xzero && rhs == b[l].p) {   // the whole tail of the cycle in one cluster launch
        run_tail(first_sweep_done, done, st);
        return;
    }
    if (l == 0) {
        coarse(rhs, x[0].p, done, st);
        return;
    }
    smooth(l, rhs, xzero, sc, done, st, first_sweep_done);
    coarse_correction(l, rhs, sc, done, st);
    smooth(l, rhs, false, sc, done, st, false, dest);
}

template <typename T>
void MGImpl<T>::coarse_correction(int l, const T* rhs, const Scratch& sc, const int* done, cudaStream_t st)
{
    mg_spmv<T, 0>(*this, st, A[l], x[l].p, EpiResid<T>{rhs, r[l].p}, sc, done);
    const int lc = l - 1;
    const bool fuse_sweep = lc >= 1 && sm[lc].kind == JFG_SMOOTH_JACOBI && sm[lc].runs > 0;
    if (fuse_sweep) {
        T* dst = (sm[lc].runs % 2 == 1) ? x[lc].p : t[lc].p;
        mg_spmv<T, 0>(*this, st, R[lc], r[l].p,
                             EpiRestrictSweep<T>{mask[lc].p, b[lc].p, dinv[lc].p, dst, (T)sm[lc].omega}, sc, done);
    } else {
        mg_spmv<T, 0>(*this, st, R[lc], r[l].p, EpiMasked<T>{mask[lc].p, b[lc].p}, sc, done);
    }
    vstep(lc, b[lc].p, true, sc, done, st, fuse_sweep);
    mg_spmv<T, 0>(*this, st, P[lc], x[lc].p, EpiMaskedAdd<T>{mask[l].p, x[l].p}, sc, done);
}

// mgStepW (MGPreconditionerInterface.java:200-291): pre-smoothing, two
// coarse-grid corrections in a row, each by mgStepV on level l-1 from a zero
// start, post-smoothing; result in x[l] (or dest).
template <typename T>
void MGImpl<T>::wstep(int l, const T* rhs, bool xzero, const Scratch& sc, const int* done, cudaStream_t st, T* dest)
{
    if (l == 0) {
        coarse(rhs, x[0].p, done, st);
        if (dest) vec_launch<0>(st, n[0], VCopy<T>{x[0].p, dest}, sc, done);
        return;
    }
    smooth(l, rhs, xzero, sc, done, st);
    coarse_correction(l, rhs, sc, done, st);
    coarse_correction(l, rhs, sc, done, st);
    smooth(l, rhs, false, sc, done, st, false, dest);
}

// fullVCycleCorrection (MGPreconditionerInterface.java:307-326); result in x[L-1].
template <typename T>
void MGImpl<T>::fmg_into_top(const T* defect, const Scratch& sc, const int* done, cudaStream_t st)
{
    std::vector<const T*> rh(L);
    rh[L - 1] = defect;
    for (int l = L - 2; l >= 0; l--) {
        mg_spmv<T, 0>(*this, st, R[l], rh[l + 1], EpiMasked<T>{mask[l].p, fr[l].p}, sc, done);
        rh[l] = fr[l].p;
    }
    for (int l = 0; l < L - 1; l++) {
        vstep(l, rh[l], false, sc, done, st);
        // raw prolongation without boundary zeroing (getProlongationMatrix, line 323)
        mg_spmv<T, 0>(*this, st, P[l], x[l].p, EpiStore<T>{x[l + 1].p}, sc, done);
    }
}

template <typename T>
void MGImpl<T>::apply(const T* v, T* out, const Scratch& sc, const int* done, cudaStream_t st)
{
    int Lf = L - 1, m = n[Lf];
    T* defect = b[Lf].p;
    // the defect copy fused with the finest level's first Jacobi sweep from zero
    // (a plain V-cycle whose finest level is not the cluster tail)
    const bool fuse_first = !use_fmg && !wcycle && L > 1 && cycles >= 1 && tail != Lf &&
                            sm[Lf].kind == JFG_SMOOTH_JACOBI && sm[Lf].runs >= 1;
    if (fuse_first) {
        const T om = (T)sm[Lf].omega;
        T* dst0 = (sm[Lf].runs % 2 == 1) ? x[Lf].p : t[Lf].p;
        vec_launch<0>(st, m, VCopyScaleMul<T>{v, defect, dinv[Lf].p, dst0, om}, sc, done);
        if (naff)
            launch_ex(k_bc_defect_scale<T>, dim3(nb(naff)), dim3(256), 0, st, naff, (const int*)aff_row.p,
                      (const int*)aff_ptr.p, (const int*)aff_col.p, (const T*)aff_val.p, v, defect,
                      (const T*)dinv[Lf].p, dst0, om, done);
    } else {
        vec_launch<0>(st, m, VCopy<T>{v, defect}, sc, done);
        if (naff) {
            launch_ex(k_bc_defect<T>, dim3(nb(naff)), dim3(256), 0, st, naff, (const int*)aff_row.p,
                      (const int*)aff_ptr.p, (const int*)aff_col.p, (const T*)aff_val.p, v, defect, done);
        }
    }
    // the boundary add folded into the last post-smoothing sweep when it writes out
    bc_src = (nbd_fine && bd_unique) ? v : nullptr;
    bc_done = false;
    bool xzero = true;
    if (use_fmg && L > 1) {
        fmg_into_top(defect, sc, done, st);
        xzero = false;
    } else if (use_fmg && L == 1) {
        coarse(defect, x[0].p, done, st);
        xzero = false;
    }
    if (L == 1) {
        for (int cyc = 0; cyc < cycles; cyc++) coarse(defect, x[0].p, done, st);
        if (cycles == 0 && xzero) vec_launch<0>(st, m, VZero<T>{x[0].p}, sc, done);
    } else {
        // the last cycle's post-smoothing writes the result straight into out
        for (int cyc = 0; cyc < cycles; cyc++) {
            // only the last cycle's post-smoothing writes out (bc_src applies there)
            const T* keep = bc_src;
            if (cyc != cycles - 1) bc_src = nullptr;
            if (wcycle)
                wstep(Lf, defect, xzero, sc, done, st, cyc == cycles - 1 ? out : nullptr);
            else
                vstep(Lf, defect, xzero, sc, done, st, fuse_first && cyc == 0, cyc == cycles - 1 ? out : nullptr);
            bc_src = keep;
            xzero = false;
        }
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[Lf].p}, sc, done);
    }
    if (L == 1 || cycles == 0) vec_launch<0>(st, m, VCopy<T>{x[Lf].p, out}, sc, done);
    if (nbd_fine && !bc_done) {
        launch_ex(k_bc_add<T>, dim3(nb(nbd_fine)), dim3(256), 0, st, nbd_fine, (const int*)bd_fine.p, v, out, done);
    }
    bc_src = nullptr;
    bc_done = false;
}

template <typename T>
void MGImpl<T>::vcycle(const T* x0, const T* rhs, T* out, const Scratch& sc, const int* done, cudaStream_t st)
{
    int Lf = L - 1, m = n[Lf];
    vec_launch<0>(st, m, VCopy<T>{rhs, b[Lf].p}, sc, done);
    vec_launch<0>(st, m, VCopy<T>{x0, x[Lf].p}, sc, done);
    vstep(Lf, b[Lf].p, false, sc, done, st);
    vec_launch<0>(st, m, VCopy<T>{x[Lf].p, out}, sc, done);
}

template <typename T>
void MGImpl<T>::wcycle_apply(const T* x0, const T* rhs, T* out, const Scratch& sc, const int* done,
                             cudaStream_t st)
{
    int Lf = L - 1, m = n[Lf];
    vec_launch<0>(st, m, VCopy<T>{rhs, b[Lf].p}, sc, done);
    vec_launch<0>(st, m, VCopy<T>{x0, x[Lf].p}, sc, done);
    wstep(Lf, b[Lf].p, false, sc, done, st);
    vec_launch<0>(st, m, VCopy<T>{x[Lf].p, out}, sc, done);
}

template <typename T>
void MGImpl<T>::fmg(const T* defect, T* out, const Scratch& sc, const int* done, cudaStream_t st)
{
    int Lf = L - 1, m = n[Lf];
    vec_launch<0>(st, m, VCopy<T>{defect, b[Lf].p}, sc, done);
    if (L == 1) {
        coarse(b[0].p, x[0].p, done, st);
    } else {
        fmg_into_top(b[Lf].p, sc, done, st);
    }
    vec_launch<0>(st, m, VCopy<T>{x[Lf].p, out}, sc, done);
}

template struct MGImpl<double>;
template struct MGImpl<float>;

void smooth_standalone(Context* c, Matrix* A, const SmootherDesc& d, const double* rhs, double* xv, const Scratch& sc)
{
    cudaStream_t st = c->stream;
    int m = A->rows;
    if (d.kind == JFG_SMOOTH_SCHWARZ) {
        d.schwarz->smooth<double>(d.runs, rhs, xv, sc, nullptr, st);
        JFG_CUDA(cudaStreamSynchronize(st));
        return;
    }
    DevBuf<double> dinv, t, r;
    DevBuf<int> flag;
    dinv.alloc(m);
    t.alloc(m);
    r.alloc(m);
    flag.alloc(1);
    if (d.kind == JFG_SMOOTH_FBGS || d.kind == JFG_SMOOTH_GS) {
        for (int k = 0; k < d.runs; k++) {
            if (d.kind == JFG_SMOOTH_FBGS) {
                spmv_launch<double, double, 0>(st, A, A->val.p, xv, EpiResid<double>{rhs, r.p}, sc, nullptr);
                d.gs->backward<double>(r.p, t.p, nullptr, st);
                d.gs->forward_fbgs<double>(t.p, r.p, xv, nullptr, st);
            } else {
                d.gs->strict_upper<double>(rhs, xv, t.p, nullptr, st);
                d.gs->forward<double>(t.p, xv, nullptr, st);
            }
        }
        JFG_CUDA(cudaStreamSynchronize(st));
        return;
    }
    if (m) k_dinv<double><<<nb(m), 256, 0, st>>>(m, A->diag.p, dinv.p);
    JFG_CUDA(cudaGetLastError());
    if (d.kind == JFG_SMOOTH_JACOBI) {
        double* cur = xv;
        double* alt = t.p;
        for (int k = 0; k < d.runs; k++) {
            spmv_launch<double, double, 0>(st, A, A->val.p, cur, EpiJacobi<double>{cur, rhs, dinv.p, alt, d.omega},
                                           sc, nullptr);
            std::swap(cur, alt);
        }
        if (cur != xv) vec_launch<0>(st, m, VCopy<double>{cur, xv}, sc, nullptr);
    } else {
        for (int k = 0; k < d.runs; k++) {
            spmv_launch<double, double, 1>(st, A, A->val.p, xv, EpiResid<double>{rhs, r.p}, sc, nullptr,
                                           FinSmoothFlag{flag.p});
            vec_launch<0>(st, m, VRichardson<double>{r.p, xv, d.omega, flag.p}, sc, nullptr);
        }
    }
    JFG_CUDA(cudaStreamSynchronize(st));
}

}  // namespace jfg

jfg::MGImpl<float>* jfg_mg::fp32()
{
    if (!d32) {
        std::vector<const int*> bp(levels);
        std::vector<int> nbp(levels);
        for (int l = 0; l < levels; l++) {
            bp[l] = bdry[l].data();
            nbp[l] = (int)bdry[l].size();
        }
        d32.reset(new jfg::MGImpl<float>());
        const char* e = getenv("JFEM_MG_BF16");
        const int vfmt = precision == 3 ? 2 : ((precision == 2 || (e && e[0] == '1')) ? 1 : 0);
        d32->init(ctx, levels, A.data(), P.data(), bp.data(), nbp.data(), sm.data(), cycles, use_fmg, vfmt);
        d32->wcycle = wcycle;
    }
    return d32.get();
}
