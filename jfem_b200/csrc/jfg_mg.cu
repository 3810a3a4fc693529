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
// The bottom of the V-cycle in one launch.  Below a few thousand rows every
// level's kernels are launch-latency bound (a few microseconds each whatever
// their size), so the levels 0..bot run inside one thread-block cluster:
// every phase (Jacobi sweep, residual, restriction with the fused first
// sweep, coarse solve, prolongation + correction) is a cluster-wide loop over
// the level's SELL slots followed by a cluster barrier.  Row sums use the
// SpMV kernel's order (same lanes per row, same unrolling and shuffle tree),
// so the result is bit-identical to the per-kernel V-cycle; vectors written
// inside the kernel are read with coherent loads.
constexpr int kBotMax = 6;                // levels handled by the cluster kernel, coarse level included
constexpr int kBotRows = 4500;            // largest level taken into the cluster kernel
constexpr int kBotCtas = 8;               // portable cluster size
constexpr int kBotThreads = 1024;

template <typename VT>
struct BotMat {
    const int* off;
    const int* perm;
    const int* col;
    const int16_t* col16;
    const VT* val;
    int nslots, tpr_log2, idx16;
};

template <typename T, typename VT>
struct BotLevel {
    BotMat<VT> A, R, P;       // R: restriction to level l - 1, P: prolongation from level l - 1
    T *x, *t, *b, *r;
    const T* dinv;
    const unsigned char* mask;
    int n, runs;
    T omega;
};

template <typename T, typename VT>
struct BotParams {
    BotLevel<T, VT> lv[kBotMax];
    int top, n0, fsd;
    const double* ainv0;
    const int* done;
};

template <typename VT>
BotMat<VT> bot_mat(const Matrix* M, const VT* val)
{
    return BotMat<VT>{M->off.p, M->perm.p, M->col.p, M->col16.p, val, M->nslices * kSliceRows, M->tpr_log2,
                      M->idx16};
}

template <typename VT, typename XT, int TPR, bool I16>
__device__ __forceinline__ typename AccOf<VT>::T bot_row(const BotMat<VT>& m, const XT* x, int slot, int sub, int& r)
{
    using AT = typename AccOf<VT>::T;
    AT sum = 0;
    r = -1;
    if (slot < m.nslots) {
        const int s = slot >> 5, lane = slot & 31;
        const int o = __ldg(m.off + s);
        const int len = (__ldg(m.off + s + 1) - o) >> 5;
        r = __ldg(m.perm + slot);
        const VT* vp = m.val + o + lane;
        const int st = 32 * TPR;
        int k = sub;
        if constexpr (I16) {
            const int base = r < 0 ? 0 : r;
            const int16_t* cp = m.col16 + o + lane;
            for (; k + 3 * TPR < len; k += 4 * TPR) {
                const int c0 = base + __ldg(cp + 32 * k), c1 = base + __ldg(cp + 32 * k + st);
                const int c2 = base + __ldg(cp + 32 * k + 2 * st), c3 = base + __ldg(cp + 32 * k + 3 * st);
                const AT v0 = to_acc(__ldg(vp + 32 * k)), v1 = to_acc(__ldg(vp + 32 * k + st));
                const AT v2 = to_acc(__ldg(vp + 32 * k + 2 * st)), v3 = to_acc(__ldg(vp + 32 * k + 3 * st));
                const AT x0 = (AT)x[c0], x1 = (AT)x[c1], x2 = (AT)x[c2], x3 = (AT)x[c3];
                sum += v0 * x0;
                sum += v1 * x1;
                sum += v2 * x2;
                sum += v3 * x3;
            }
            for (; k < len; k += TPR) sum += to_acc(__ldg(vp + 32 * k)) * (AT)x[base + __ldg(cp + 32 * k)];
        } else {
            const int* cp = m.col + o + lane;
            for (; k + 3 * TPR < len; k += 4 * TPR) {
                const int c0 = __ldg(cp + 32 * k), c1 = __ldg(cp + 32 * k + st);
                const int c2 = __ldg(cp + 32 * k + 2 * st), c3 = __ldg(cp + 32 * k + 3 * st);
                const AT v0 = to_acc(__ldg(vp + 32 * k)), v1 = to_acc(__ldg(vp + 32 * k + st));
                const AT v2 = to_acc(__ldg(vp + 32 * k + 2 * st)), v3 = to_acc(__ldg(vp + 32 * k + 3 * st));
                const AT x0 = (AT)x[c0], x1 = (AT)x[c1], x2 = (AT)x[c2], x3 = (AT)x[c3];
                sum += v0 * x0;
                sum += v1 * x1;
                sum += v2 * x2;
                sum += v3 * x3;
            }
            for (; k < len; k += TPR) sum += to_acc(__ldg(vp + 32 * k)) * (AT)x[__ldg(cp + 32 * k)];
        }
    }
    for (int o = TPR >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    return sum;
}

template <int TPR, bool I16, typename VT, typename XT, class Epi>
__device__ __forceinline__ void bot_spmv_t(const BotMat<VT>& m, const XT* x, Epi epi, int gtid, int gthreads)
{
    const int total = m.nslots * TPR;
    for (int base = 0; base < total; base += gthreads) {      // warp-uniform trip count
        const int gid = base + gtid;
        int r;
        const auto sum = bot_row<VT, XT, TPR, I16>(m, x, gid / TPR, gid % TPR, r);
        double acc[1] = {0.0};
        if (gid % TPR == 0 && r >= 0) epi(r, sum, acc);
    }
}

template <typename VT, typename XT, class Epi>
__device__ void bot_spmv(const BotMat<VT>& m, const XT* x, Epi epi, int gtid, int gthreads)
{
    if (m.idx16) {
        switch (m.tpr_log2) {
        case 0: bot_spmv_t<1, true>(m, x, epi, gtid, gthreads); break;
        case 2: bot_spmv_t<4, true>(m, x, epi, gtid, gthreads); break;
        default: bot_spmv_t<8, true>(m, x, epi, gtid, gthreads); break;
        }
    } else {
        switch (m.tpr_log2) {
        case 0: bot_spmv_t<1, false>(m, x, epi, gtid, gthreads); break;
        case 2: bot_spmv_t<4, false>(m, x, epi, gtid, gthreads); break;
        default: bot_spmv_t<8, false>(m, x, epi, gtid, gthreads); break;
        }
    }
}

template <typename T, typename VT>
__global__ void __launch_bounds__(kBotThreads, 1) k_mg_bottom(const __grid_constant__ BotParams<T, VT> P)
{
    pdl_wait();
    if (P.done && *P.done) return;           // the same answer for every CTA of the cluster
    cg::cluster_group cl = cg::this_cluster();
    const int gthreads = (int)cl.num_blocks() * blockDim.x;
    const int gtid = (int)cl.block_rank() * blockDim.x + threadIdx.x;
    bool fsd = P.fsd != 0;
    for (int l = P.top; l >= 1; l--) {
        const BotLevel<T, VT>& L = P.lv[l];
        const T* rhs = L.b;
        T* dst = (L.runs % 2 == 1) ? L.x : L.t;
        if (!fsd) {                           // first sweep from the zero guess
            for (int i = gtid; i < L.n; i += gthreads) dst[i] = (T)0 + (L.dinv[i] * rhs[i]) * L.omega;
            cl.sync();
        }
        T* cur = dst;
        T* alt = (dst == L.x) ? L.t : L.x;
        for (int k = 1; k < L.runs; k++) {
            bot_spmv(L.A, cur, EpiJacobi<T>{cur, rhs, L.dinv, alt, L.omega}, gtid, gthreads);
            cl.sync();
            T* tmp = cur;
            cur = alt;
            alt = tmp;
        }
        if (cur != L.x) {
            for (int i = gtid; i < L.n; i += gthreads) L.x[i] = cur[i];
            cl.sync();
        }
        bot_spmv(L.A, L.x, EpiResid<T>{rhs, L.r}, gtid, gthreads);
        cl.sync();
        const BotLevel<T, VT>& Cl = P.lv[l - 1];
        if (l - 1 >= 1) {
            T* dc = (Cl.runs % 2 == 1) ? Cl.x : Cl.t;
            bot_spmv(L.R, L.r, EpiRestrictSweep<T>{Cl.mask, Cl.b, Cl.dinv, dc, Cl.omega}, gtid, gthreads);
            fsd = true;
        } else {
            bot_spmv(L.R, L.r, EpiMasked<T>{Cl.mask, Cl.b}, gtid, gthreads);
        }
        cl.sync();
    }
    {   // coarsest level: x0 = Ainv * b0 in FP64, one warp per row (the order of k_coarse_gemv)
        const int lane = threadIdx.x & 31;
        const int nw = gthreads >> 5;
        for (int row = gtid >> 5; row < P.n0; row += nw) {
            double s = 0;
            for (int j = lane; j < P.n0; j += 32) s += P.ainv0[(size_t)row * P.n0 + j] * (double)P.lv[0].b[j];
            s = warp_sum(s);
            if (lane == 0) P.lv[0].x[row] = (T)s;
        }
        cl.sync();
    }
    for (int l = 1; l <= P.top; l++) {
        const BotLevel<T, VT>& L = P.lv[l];
        bot_spmv(L.P, P.lv[l - 1].x, EpiMaskedAdd<T>{L.mask, L.x}, gtid, gthreads);
        cl.sync();
        T* cur = L.x;
        T* alt = L.t;
        for (int k = 0; k < L.runs; k++) {
            bot_spmv(L.A, cur, EpiJacobi<T>{cur, L.b, L.dinv, alt, L.omega}, gtid, gthreads);
            cl.sync();
            T* tmp = cur;
            cur = alt;
            alt = tmp;
        }
        if (cur != L.x) {
            for (int i = gtid; i < L.n; i += gthreads) L.x[i] = cur[i];
            cl.sync();
        }
    }
}

template <typename T, typename VT>
void launch_bottom(const BotParams<T, VT>& p, cudaStream_t st)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kBotCtas);
    cfg.blockDim = dim3(kBotThreads);
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kBotCtas;
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
    JFG_CUDA(cudaLaunchKernelEx(&cfg, k_mg_bottom<T, VT>, p));
    note_launch();
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
        for (int i = 0; i < nbd_fine; i++) isbd[bdry[Lf][i]] = 1;
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
    // JFEM_MG_BOTTOM=1: levels 1..bot (all small, Jacobi-smoothed) and the
    // coarse solve run as one cluster kernel.  Off by default: on the Q2 512^2
    // hierarchy it replaces ~19 launches per V-cycle but is ~26 us slower per
    // V-cycle, because one 8-SM cluster hides far less load latency than the
    // whole GPU does per launch.
    bot = -1;
    const char* eb = getenv("JFEM_MG_BOTTOM");
    if (eb && eb[0] == '1' && !vfp16) {
        for (int l = 1; l < L - 1 && l < kBotMax; l++) {
            if (n[l] > kBotRows || sm[l].kind != JFG_SMOOTH_JACOBI || sm[l].runs < 1) break;
            bot = l;
        }
    }
    JFG_CUDA(cudaStreamSynchronize(st));
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
            mg_spmv<T, 0>(*this, st, M, cur, EpiJacobi<T>{cur, rhs, dinv[l].p, o, om}, sc, done);
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
void MGImpl<T>::bottom(bool first_sweep_done, const int* done, cudaStream_t st)
{
    auto fill = [&](auto& p, auto vals) {
        p.top = bot;
        p.n0 = n[0];
        p.fsd = first_sweep_done ? 1 : 0;
        p.ainv0 = ainv0.p;
        p.done = done;
        for (int l = 0; l <= bot; l++) {
            auto& L = p.lv[l];
            L.A = bot_mat(A[l], vals(A[l]));
            if (l >= 1) {
                L.R = bot_mat(R[l - 1], vals(R[l - 1]));
                L.P = bot_mat(P[l - 1], vals(P[l - 1]));
            }
            L.x = x[l].p;
            L.t = t[l].p;
            L.b = b[l].p;
            L.r = r[l].p;
            L.dinv = dinv[l].p;
            L.mask = mask[l].p;
            L.n = n[l];
            L.runs = sm[l].runs;
            L.omega = (T)sm[l].omega;
        }
    };
    if constexpr (std::is_same<T, float>::value) {
        if (vbf16) {
            BotParams<float, __nv_bfloat16> p = {};
            fill(p, [](const Matrix* M) { return (const __nv_bfloat16*)M->val16.p; });
            launch_bottom(p, st);
            return;
        }
    }
    BotParams<T, T> p = {};
    fill(p, [](const Matrix* M) { return vals_of<T>(M); });
    launch_bottom(p, st);
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
    if (l == bot && xzero && rhs == b[l].p) {    // the whole bottom of the cycle in one cluster launch
        bottom(first_sweep_done, done, st);
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
    vec_launch<0>(st, m, VCopy<T>{v, defect}, sc, done);
    if (naff) {
        launch_ex(k_bc_defect<T>, dim3(nb(naff)), dim3(256), 0, st, naff, (const int*)aff_row.p,
                  (const int*)aff_ptr.p, (const int*)aff_col.p, (const T*)aff_val.p, v, defect, done);
    }
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
            if (wcycle)
                wstep(Lf, defect, xzero, sc, done, st, cyc == cycles - 1 ? out : nullptr);
            else
                vstep(Lf, defect, xzero, sc, done, st, false, cyc == cycles - 1 ? out : nullptr);
            xzero = false;
        }
        if (xzero) vec_launch<0>(st, m, VZero<T>{x[Lf].p}, sc, done);
    }
    if (L == 1 || cycles == 0) vec_launch<0>(st, m, VCopy<T>{x[Lf].p, out}, sc, done);
    if (nbd_fine) {
        launch_ex(k_bc_add<T>, dim3(nb(nbd_fine)), dim3(256), 0, st, nbd_fine, (const int*)bd_fine.p, v, out, done);
    }
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
