// Batched implicit-Euler time stepping of many independent systems in one
// persistent launch (the HeatEquation time loop, Examples/src/HeatEquation.java:81-94,
// for a whole batch).
//
// Layout: every system keeps its own K = M + dt A (SELL-32-sigma, FP64 and
// FP32 values) and M (FP64) as built by jfg_matrix_from_coo; a device
// descriptor table holds the pointers plus per-system work vectors carved
// from one pool.  A cluster of C CTAs owns one system at a time: the CTA of
// rank c owns a contiguous range of SELL slots (rows), cluster barriers
// separate the phases, and dot products are reduced across the cluster
// through distributed shared memory (fixed order, deterministic).  Clusters
// take systems from a global counter over a largest-first order.
//
// Per step:  rhs = M u + f;  repeat  r = rhs - K u (FP64);  stop when
// ||r|| <= rtol ||rhs||;  solve K e = r/||r|| by FP32 Jacobi-PCG to
// inner_rtol;  u += ||r|| e.
// The inner PCG folds the direction update into the product:
// A p_new = A z + beta A p_old, so one iteration needs two cluster barriers.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "jfg_ops.cuh"

namespace cg = cooperative_groups;

struct jfg_ctx;
struct jfg_mat;

namespace jfg {
cudaStream_t ctx_stream(jfg_ctx* ctx);
int ctx_device(jfg_ctx* ctx);
void ctx_set_error(jfg_ctx* ctx, const std::string& msg);
Matrix* mat_of(jfg_mat* m);
jfg_ctx* mat_ctx(jfg_mat* m);
}  // namespace jfg

namespace {

using namespace jfg;

struct SysDesc {
    int n, nslots;
    const int *k_off, *k_perm, *k_col;
    const int16_t* k_col16;      // 16-bit column offsets from the row, or null
    const double* k_v64;
    const float* k_v32;
    const int *m_off, *m_perm, *m_col;
    const double* m_v64;
    const float* dinv;
    double *u, *rhs, *r64;
    const double* f;
    float *e, *r, *z, *p, *Ap;
};

struct BatchParams {
    const SysDesc* sys;
    const int* order;
    int nsys;
    int steps;
    double rtol, inner_rtol;
    int inner_max, max_refine;
    unsigned* queue;
    int* iters;
    double* relres;
    int* refines;
    int* status;
};

// Block sum of two values; result valid in every thread.
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh)
{
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (l == 0) {
        sh[2 * w] = a;
        sh[2 * w + 1] = b;
    }
    __syncthreads();
    double ta = 0, tb = 0;
    for (int i = 0; i < nw; i++) {
        ta += sh[2 * i];
        tb += sh[2 * i + 1];
    }
    a = ta;
    b = tb;
    __syncthreads();
}

// Cluster-wide sum of two values (deterministic: rank order).  slot is a
// double-buffered shared array [2][2] of every CTA.
__device__ __forceinline__ void cluster_sum2(cg::cluster_group& cl, double& a, double& b, double* sh, double* slot,
                                             int& parity)
{
    block_sum2(a, b, sh);
    if (threadIdx.x == 0) {
        slot[2 * parity] = a;
        slot[2 * parity + 1] = b;
    }
    cl.sync();
    double ta = 0, tb = 0;
    const unsigned nb = cl.num_blocks();
    for (unsigned r = 0; r < nb; r++) {
        const double* rs = cl.map_shared_rank(slot, r);
        ta += rs[2 * parity];
        tb += rs[2 * parity + 1];
    }
    a = ta;
    b = tb;
    parity ^= 1;
}

template <typename V, typename X>
__device__ __forceinline__ double sell_row(const int* off, const int* col, const V* val, const X* x, int slot)
{
    const int s = slot >> 5, lane = slot & 31;
    const int o = off[s];
    const int len = (off[s + 1] - o) >> 5;
    double sum = 0;
    for (int k = 0; k < len; k++) sum += (double)val[o + 32 * k + lane] * (double)x[col[o + 32 * k + lane]];
    return sum;
}
// The two passes of an inner PCG iteration take U rows of a thread
// at once (slots t, t + B, t + 2B, ... as in a plain strided loop): all loads
// of those rows are issued before any of their results is used, so a thread
// has several rows' gathers in flight instead of one dependent chain per row.
// Row sums keep the entry order and partial dot products the row order of the
// one-row-at-a-time loop, so the results are the same bits.
constexpr int kRowChunk = 3;     // entries of each row loaded together

template <int U, int CH, bool I16>
__device__ __forceinline__ void sell_rows32(const SysDesc& S, const int (&slot)[U], const int (&row)[U],
                                            float (&q)[U])
{
    const int* __restrict__ off = S.k_off;
    const float* __restrict__ val = S.k_v32;
    const float* x = S.z;                 // written inside the kernel: coherent loads
    int o[U], len[U];
    int maxlen = 0;
#pragma unroll
    for (int u = 0; u < U; u++) {
        q[u] = 0.f;
        o[u] = 0;
        len[u] = 0;
        if (row[u] >= 0) {
            const int s = slot[u] >> 5;
            const int a = __ldg(off + s);
            o[u] = a + (slot[u] & 31);
            len[u] = (__ldg(off + s + 1) - a) >> 5;
        }
        maxlen = max(maxlen, len[u]);
    }
    for (int k = 0; k < maxlen; k += CH) {
        int c[U][CH];
        float v[U][CH], xv[U][CH];
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int j = 0; j < CH; j++) {
                const bool ok = k + j < len[u];
                const int idx = o[u] + 32 * (k + j);
                if constexpr (I16)
                    c[u][j] = ok ? row[u] + (int)__ldg(S.k_col16 + idx) : 0;
                else
                    c[u][j] = ok ? __ldg(S.k_col + idx) : 0;
                v[u][j] = ok ? __ldg(val + idx) : 0.f;
            }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int j = 0; j < CH; j++) xv[u][j] = k + j < len[u] ? x[c[u][j]] : 0.f;
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int j = 0; j < CH; j++)
                if (k + j < len[u]) q[u] += v[u][j] * xv[u][j];
    }
}

// p = z + beta p ; Ap = K z + beta Ap ; returns this thread's part of p.Ap.
template <int U, bool I16>
__device__ __forceinline__ double pass_direction(const SysDesc& S, int s0, int s1, float bf)
{
    const int B = blockDim.x;
    double pap = 0;
    for (int b0 = s0 + threadIdx.x; b0 < s1; b0 += U * B) {
        int slot[U], row[U];
        float zr[U], pr[U], ar[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            slot[u] = b0 + u * B;
            row[u] = slot[u] < s1 ? __ldg(S.k_perm + slot[u]) : -1;
            zr[u] = pr[u] = ar[u] = 0.f;
            if (row[u] >= 0) {
                zr[u] = S.z[row[u]];
                pr[u] = S.p[row[u]];
                ar[u] = S.Ap[row[u]];
            }
        }
        float q[U];
        sell_rows32<U, kRowChunk, I16>(S, slot, row, q);
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (row[u] < 0) continue;
            const float pn = zr[u] + bf * pr[u];
            const float apn = q[u] + bf * ar[u];
            S.p[row[u]] = pn;
            S.Ap[row[u]] = apn;
            pap += (double)pn * apn;
        }
    }
    return pap;
}

// e += alpha p ; r -= alpha Ap ; z = dinv r ; adds r.z and r.r of this thread.
template <int U>
__device__ __forceinline__ void pass_update(const SysDesc& S, int s0, int s1, float alpha, double& rzn,
                                            double& rrn)
{
    const int B = blockDim.x;
    for (int b0 = s0 + threadIdx.x; b0 < s1; b0 += U * B) {
        int row[U];
        float ev[U], pv[U], rv[U], av[U], dv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int sl = b0 + u * B;
            row[u] = sl < s1 ? __ldg(S.k_perm + sl) : -1;
            ev[u] = pv[u] = rv[u] = av[u] = dv[u] = 0.f;
            if (row[u] >= 0) {
                ev[u] = S.e[row[u]];
                pv[u] = S.p[row[u]];
                rv[u] = S.r[row[u]];
                av[u] = S.Ap[row[u]];
                dv[u] = S.dinv[row[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (row[u] < 0) continue;
            S.e[row[u]] = ev[u] + alpha * pv[u];
            const float rn = rv[u] - alpha * av[u];
            const float zn = dv[u] * rn;
            S.r[row[u]] = rn;
            S.z[row[u]] = zn;
            rzn += (double)rn * zn;
            rrn += (double)rn * rn;
        }
    }
}

// U: rows of a thread in flight per pass (2, 3 or 4; picked by the autotuner)
template <int U>
__global__ void __launch_bounds__(512, 2) k_batch_heat(BatchParams P)
{
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double sh[64];
    __shared__ double slot[4];
    __shared__ int sys_sh;
    const unsigned rank = cl.block_rank();
    const unsigned C = cl.num_blocks();
    int parity = 0;
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            unsigned t = atomicAdd(P.queue, 1u);
            sys_sh = t < (unsigned)P.nsys ? P.order[t] : -1;
        }
        cl.sync();
        const int si = *cl.map_shared_rank(&sys_sh, 0);
        cl.sync();   // everyone has read the leader's slot before it is reused
        if (si < 0) break;
        const SysDesc& S = P.sys[si];   // fields re-read from L1 rather than pinned in registers
        // this CTA's slots
        const int chunk = ((S.nslots / 32 + C - 1) / C) * 32;
        const int s0 = min(S.nslots, (int)rank * chunk), s1 = min(S.nslots, s0 + chunk);
        int total_inner = 0, refines_max = 0, status = JFG_OK;
        double last_rel = 0;
        for (int step = 0; step < P.steps; step++) {
            // rhs = M u + f
            double bb = 0, dummy = 0;
            for (int slot_i = s0 + threadIdx.x; slot_i < s1; slot_i += blockDim.x) {
                const int row = S.m_perm[slot_i];
                if (row < 0) continue;
                double v = sell_row(S.m_off, S.m_col, S.m_v64, S.u, slot_i);
                if (S.f) v += S.f[row];
                S.rhs[row] = v;
                bb += v * v;
            }
            cluster_sum2(cl, bb, dummy, sh, slot, parity);
            const double bnorm = sqrt(bb);
            int ref = 0;
            for (;; ref++) {
                // r = rhs - K u (FP64) and its norm
                double rr = 0, d2 = 0;
                for (int slot_i = s0 + threadIdx.x; slot_i < s1; slot_i += blockDim.x) {
                    const int row = S.k_perm[slot_i];
                    if (row < 0) continue;
                    double v = S.rhs[row] - sell_row(S.k_off, S.k_col, S.k_v64, S.u, slot_i);
                    S.r64[row] = v;
                    rr += v * v;
                }
                cluster_sum2(cl, rr, d2, sh, slot, parity);
                const double rn = sqrt(rr);
                last_rel = bnorm > 0 ? rn / bnorm : rn;
                if (!isfinite(rn)) {
                    status = JFG_NONFINITE;
                    break;
                }
                if (rn <= P.rtol * bnorm || rn == 0.0) break;
                if (ref >= P.max_refine) {
                    status = JFG_NOT_CONVERGED;
                    break;
                }
                // inner FP32 Jacobi-PCG on K e = r / ||r||, e0 = 0
                const float inv = (float)(1.0 / rn);
                double rz = 0, rr32 = 0;
                for (int slot_i = s0 + threadIdx.x; slot_i < s1; slot_i += blockDim.x) {
                    const int row = S.k_perm[slot_i];
                    if (row < 0) continue;
                    const float rv = (float)S.r64[row] * inv;
                    const float zv = S.dinv[row] * rv;
                    S.r[row] = rv;
                    S.z[row] = zv;
                    S.e[row] = 0.f;
                    S.p[row] = 0.f;
                    S.Ap[row] = 0.f;
                    rz += (double)rv * zv;
                    rr32 += (double)rv * rv;
                }
                cluster_sum2(cl, rz, rr32, sh, slot, parity);
                double beta = 0;
                int it = 0;
                while (sqrt(rr32) > P.inner_rtol && it < P.inner_max) {
                    // p = z + beta p ; Ap = K z + beta Ap ; pAp
                    double d3 = 0;
                    const float bf = (float)beta;
                    double pap = S.k_col16 ? pass_direction<U, true>(S, s0, s1, bf)
                                           : pass_direction<U, false>(S, s0, s1, bf);
                    cluster_sum2(cl, pap, d3, sh, slot, parity);
                    const float alpha = (float)(rz / pap);
                    // e += alpha p ; r -= alpha Ap ; z = dinv r
                    double rzn = 0, rrn = 0;
                    pass_update<U>(S, s0, s1, alpha, rzn, rrn);
                    cluster_sum2(cl, rzn, rrn, sh, slot, parity);
                    beta = rzn / rz;
                    rz = rzn;
                    rr32 = rrn;
                    it++;
                    if (!isfinite(rr32)) break;
                }
                total_inner += it;
                // u += ||r|| e
                for (int slot_i = s0 + threadIdx.x; slot_i < s1; slot_i += blockDim.x) {
                    const int row = S.k_perm[slot_i];
                    if (row < 0) continue;
                    S.u[row] += rn * (double)S.e[row];
                }
                cl.sync();
            }
            refines_max = max(refines_max, ref);
            if (status != JFG_OK) break;
        }
        if (rank == 0 && threadIdx.x == 0) {
            P.iters[si] = total_inner;
            P.relres[si] = last_rel;
            P.refines[si] = refines_max;
            P.status[si] = status;
        }
        cl.sync();
    }
}

__global__ void k_dinv32(int n, const double* diag, float* dinv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = diag[i];
    dinv[i] = (float)(fabs(d) < 1e-300 ? 1.0 : 1.0 / d);
}

}  // namespace

struct jfg_batch {
    jfg_ctx* ctx = nullptr;
    int nsys = 0;
    std::vector<jfg::Matrix*> K, M;
    std::vector<int64_t> offs;       // packed offsets, nsys + 1
    std::vector<int> order;          // largest first
    jfg::DevBuf<double> pool64;      // u, rhs, r64
    jfg::DevBuf<float> pool32;       // e, r, z, p, Ap, dinv
    jfg::DevBuf<double> f;
    jfg::DevBuf<SysDesc> desc;
    jfg::DevBuf<int> d_order, iters, refines, status;
    jfg::DevBuf<double> relres;
    jfg::DevBuf<unsigned> queue;
    int tuned_cluster = 0, tuned_threads = 0, tuned_rows = 0;
};

namespace {

void build_desc(jfg_batch* b, bool with_f)
{
    std::vector<SysDesc> h(b->nsys);
    int64_t tot = b->offs[b->nsys];
    for (int s = 0; s < b->nsys; s++) {
        jfg::Matrix* K = b->K[s];
        jfg::Matrix* M = b->M[s];
        int64_t o = b->offs[s];
        SysDesc& d = h[s];
        d.n = K->rows;
        d.nslots = K->nslices * jfg::kSliceRows;
        d.k_off = K->off.p;
        d.k_perm = K->perm.p;
        d.k_col = K->col.p;
        d.k_col16 = K->idx16 == 1 ? K->col16.p : nullptr;   // offsets from the row only
        d.k_v64 = K->val.p;
        d.k_v32 = K->val32.p;
        d.m_off = M->off.p;
        d.m_perm = M->perm.p;
        d.m_col = M->col.p;
        d.m_v64 = M->val.p;
        d.u = b->pool64.p + o;
        d.rhs = b->pool64.p + tot + o;
        d.r64 = b->pool64.p + 2 * tot + o;
        d.f = with_f ? b->f.p + o : nullptr;
        d.e = b->pool32.p + o;
        d.r = b->pool32.p + tot + o;
        d.z = b->pool32.p + 2 * tot + o;
        d.p = b->pool32.p + 3 * tot + o;
        d.Ap = b->pool32.p + 4 * tot + o;
        d.dinv = b->pool32.p + 5 * tot + o;
    }
    JFG_CUDA(cudaMemcpyAsync(b->desc.p, h.data(), sizeof(SysDesc) * b->nsys, cudaMemcpyHostToDevice,
                             jfg::ctx_stream(b->ctx)));
}

// One persistent launch with cluster size C and T threads per CTA.
float launch(jfg_batch* b, int C, int T, int U, int steps, const jfg_batch_opts& o)
{
    void (*kern)(BatchParams) = U == 2 ? k_batch_heat<2> : (U == 4 ? k_batch_heat<4> : k_batch_heat<3>);
    cudaStream_t st = jfg::ctx_stream(b->ctx);
    BatchParams P;
    P.sys = b->desc.p;
    P.order = b->d_order.p;
    P.nsys = b->nsys;
    P.steps = steps;
    P.rtol = o.rtol;
    P.inner_rtol = o.inner_rtol;
    P.inner_max = o.inner_max;
    P.max_refine = o.max_refine;
    P.queue = b->queue.p;
    P.iters = b->iters.p;
    P.relres = b->relres.p;
    P.refines = b->refines.p;
    P.status = b->status.p;
    JFG_CUDA(cudaMemsetAsync(b->queue.p, 0, sizeof(unsigned), st));
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(T);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int max_clusters = 0;
    cfg.gridDim = dim3(C);
    JFG_CUDA(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg));
    if (max_clusters < 1) max_clusters = 1;
    int nclusters = std::min(max_clusters, b->nsys);
    cfg.gridDim = dim3(nclusters * C);
    cudaEvent_t e0, e1;
    JFG_CUDA(cudaEventCreate(&e0));
    JFG_CUDA(cudaEventCreate(&e1));
    JFG_CUDA(cudaEventRecord(e0, st));
    JFG_CUDA(cudaLaunchKernelEx(&cfg, kern, P));
    jfg::note_launch();
    JFG_CUDA(cudaEventRecord(e1, st));
    JFG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    JFG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

}  // namespace

extern "C" {

void jfg_batch_opts_default(jfg_batch_opts* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->rtol = 1e-10;
    o->inner_rtol = 1e-5;
    o->inner_max = 500;
    o->max_refine = 6;
}

int jfg_batch_create(jfg_ctx* ctx, int nsys, jfg_mat* const* K, jfg_mat* const* M, jfg_batch** out)
{
    if (!ctx || !out || nsys < 1 || !K || !M) return JFG_ERR_BAD_ARG;
    *out = nullptr;
    auto* b = new jfg_batch();
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(ctx)));
        b->ctx = ctx;
        b->nsys = nsys;
        b->offs.assign(nsys + 1, 0);
        for (int s = 0; s < nsys; s++) {
            JFG_CHECK(K[s] && M[s] && jfg::mat_ctx(K[s]) == ctx && jfg::mat_ctx(M[s]) == ctx, JFG_ERR_BAD_ARG,
                      "batch matrix missing or from another context");
            jfg::Matrix* k = jfg::mat_of(K[s]);
            jfg::Matrix* m = jfg::mat_of(M[s]);
            JFG_CHECK(k->rows == k->cols && m->rows == m->cols && k->rows == m->rows, JFG_ERR_BAD_ARG,
                      "K and M must be square and of equal size");
            jfg::matrix_ensure_fp32(k);
            b->K.push_back(k);
            b->M.push_back(m);
            b->offs[s + 1] = b->offs[s] + k->rows;
        }
        int64_t tot = b->offs[nsys];
        b->order.resize(nsys);
        for (int s = 0; s < nsys; s++) b->order[s] = s;
        std::stable_sort(b->order.begin(), b->order.end(),
                         [&](int x, int y) { return b->K[x]->nnz > b->K[y]->nnz; });
        cudaStream_t st = jfg::ctx_stream(ctx);
        b->pool64.alloc((size_t)std::max<int64_t>(1, 3 * tot));
        b->pool32.alloc((size_t)std::max<int64_t>(1, 6 * tot));
        b->desc.alloc(nsys);
        b->d_order.alloc(nsys);
        b->iters.alloc(nsys);
        b->refines.alloc(nsys);
        b->status.alloc(nsys);
        b->relres.alloc(nsys);
        b->queue.alloc(1);
        JFG_CUDA(cudaMemcpyAsync(b->d_order.p, b->order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, st));
        for (int s = 0; s < nsys; s++) {
            int n = b->K[s]->rows;
            if (n)
                k_dinv32<<<(n + 255) / 256, 256, 0, st>>>(n, b->K[s]->diag.p, b->pool32.p + 5 * tot + b->offs[s]);
        }
        JFG_CUDA(cudaGetLastError());
        build_desc(b, false);
        JFG_CUDA(cudaStreamSynchronize(st));
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(ctx, e.msg);
        delete b;
        return e.status;
    }
    *out = b;
    return JFG_OK;
}

int jfg_batch_free(jfg_batch* b)
{
    if (!b) return JFG_ERR_BAD_ARG;
    cudaStreamSynchronize(jfg::ctx_stream(b->ctx));
    delete b;
    return JFG_OK;
}

int jfg_batch_layout(jfg_batch* b, int64_t* total, int64_t* offsets)
{
    if (!b) return JFG_ERR_BAD_ARG;
    if (total) *total = b->offs[b->nsys];
    if (offsets)
        for (int s = 0; s <= b->nsys; s++) offsets[s] = b->offs[s];
    return JFG_OK;
}

int jfg_batch_heat(jfg_batch* b, int steps, const double* h_f, double* h_u, const jfg_batch_opts* opts,
                   jfg_batch_info* info)
{
    if (!b || !h_u || steps < 0) return JFG_ERR_BAD_ARG;
    jfg_batch_opts o;
    if (opts)
        o = *opts;
    else
        jfg_batch_opts_default(&o);
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(b->ctx)));
        JFG_CHECK(o.cluster == 0 || o.cluster == 1 || o.cluster == 2 || o.cluster == 4 || o.cluster == 8,
                  JFG_ERR_BAD_ARG, "cluster must be 1, 2, 4 or 8");
        JFG_CHECK(o.threads == 0 || o.threads == 256 || o.threads == 512, JFG_ERR_BAD_ARG,
                  "threads must be 256 or 512");
        JFG_CHECK(o.rows_per_thread == 0 || (o.rows_per_thread >= 2 && o.rows_per_thread <= 4), JFG_ERR_BAD_ARG,
                  "rows_per_thread must be 2, 3 or 4");
        JFG_CHECK(o.rtol > 0 && o.inner_rtol > 0 && o.inner_max > 0 && o.max_refine >= 0, JFG_ERR_BAD_ARG,
                  "bad tolerances or caps");
        cudaStream_t st = jfg::ctx_stream(b->ctx);
        int64_t tot = b->offs[b->nsys];
        if (h_f) {
            b->f.alloc((size_t)tot);
            JFG_CUDA(cudaMemcpyAsync(b->f.p, h_f, sizeof(double) * tot, cudaMemcpyHostToDevice, st));
        }
        build_desc(b, h_f != nullptr);
        int C = o.cluster, T = o.threads, U = o.rows_per_thread;
        if (C == 0 || T == 0 || U == 0) {
            // autotune once: one step of every configuration (cluster size x
            // threads per CTA x rows per thread in flight) from the given states
            if (!b->tuned_cluster) {
                float best = 1e30f;
                for (int c : {1, 2, 4, 8})
                    for (int t : {256, 512})
                        for (int u : {2, 3, 4}) {
                            JFG_CUDA(cudaMemcpyAsync(b->pool64.p, h_u, sizeof(double) * tot, cudaMemcpyHostToDevice,
                                                     st));
                            float ms = launch(b, c, t, u, 1, o);
                            if (ms < best) {
                                best = ms;
                                b->tuned_cluster = c;
                                b->tuned_threads = t;
                                b->tuned_rows = u;
                            }
                        }
            }
            if (C == 0) C = b->tuned_cluster;
            if (T == 0) T = b->tuned_threads;
            if (U == 0) U = b->tuned_rows;
        }
        JFG_CUDA(cudaMemcpyAsync(b->pool64.p, h_u, sizeof(double) * tot, cudaMemcpyHostToDevice, st));
        float ms = launch(b, C, T, U, steps, o);
        JFG_CUDA(cudaMemcpyAsync(h_u, b->pool64.p, sizeof(double) * tot, cudaMemcpyDeviceToHost, st));
        std::vector<int> it(b->nsys), rf(b->nsys), stt(b->nsys);
        std::vector<double> rr(b->nsys);
        JFG_CUDA(cudaMemcpyAsync(it.data(), b->iters.p, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(rf.data(), b->refines.p, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(stt.data(), b->status.p, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(rr.data(), b->relres.p, sizeof(double) * b->nsys, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        int worst = JFG_OK, failed = 0;
        jfg_batch_info inf{};
        for (int s = 0; s < b->nsys; s++) {
            inf.total_inner_iterations += it[s];
            inf.max_refine_used = std::max(inf.max_refine_used, rf[s]);
            inf.max_rel_residual = std::max(inf.max_rel_residual, rr[s]);
            if (stt[s] != JFG_OK) {
                failed++;
                worst = stt[s];
            }
        }
        inf.failed = failed;
        inf.cluster = C;
        inf.threads = T;
        inf.rows_per_thread = U;
        inf.ms = ms;
        if (info) *info = inf;
        return worst;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(b->ctx, e.msg);
        return e.status;
    }
}

}  // extern "C"
