// Gauss-Seidel family smoothers on the device:
//   ForwardBackwardGaussSeidelSmoother (multigrid/ForwardBackwardGaussSeidelSmoother.java:23-44)
//     runs x { x += L^-1 D U^-1 (b - A x) }
//   GaussSeidelSmoother (multigrid/GaussSeidelSmoother.java:24-32)
//     runs x { x = (L + D)^-1 (b - R x) }
// with L / U the lower / upper triangles including the diagonal
// (linalg/LowerTriangularSparseMatrix.java:22-41, linalg/UpperTriangularSparseMatrix.java:36-55),
// D the diagonal and R the strict upper triangle, all relative to an ordering
// of the rows.
//
// A triangular solve is a sequence of dependency levels (rows of one level
// read solution entries of earlier levels only).  Row i computes, in the
// reference's arithmetic (LowerTriangularSparseMatrix.backsubstituteRow,
// :188-212), sol_i = rhs_i / d_i and then sol_i += (-sol_j / d_i) * a_ij for
// its off-diagonal entries j in ascending column order, each operation
// rounded on its own (no fused multiply-add).  Runs of small levels go to one
// CTA (levels of at most 512 rows) or one 8-CTA cluster (at most 4,096) that
// steps through them with a barrier between levels; a large level is one
// grid launch.  The natural ordering reproduces the reference's
// sequential algorithm (as many steps as the longest dependency chain); the
// multicolour ordering (greedy colouring of the graph of A + A^T) is the same
// algorithm on the symmetrically permuted system and has one step per colour.
#include <cooperative_groups.h>

#include <algorithm>
#include <numeric>

#include "jfg_gs.cuh"

namespace jfg {

namespace {

inline unsigned nb(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

constexpr int kCtaThreads = 512;
constexpr int kClusterCtas = 8;
constexpr int kCtaMaxRows = kCtaThreads * kClusterCtas;   // levels up to this size run inside the cluster kernel

__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// one row of a triangular solve; slot q of a level with cnt rows, its ELL
// entries at col/val + k * cnt + q.  Entries are taken in chunks of kChunk:
// the chunk's column, value and solution loads are all issued before its
// arithmetic, so a row costs one memory round trip per chunk rather than
// one per entry; the arithmetic keeps the entry order.
template <typename T, bool SCALE, bool ADDX, int kChunk>
__device__ __forceinline__ void trsv_row(int q, int cnt, int width, const int* __restrict__ rows,
                                         const int* __restrict__ col, const T* __restrict__ val,
                                         const T* __restrict__ diag, const T* __restrict__ rhs, T* sol, T* x)
{
    const int i = rows[q];
    const T d = diag[i];
    T r = rhs[i];
    if (SCALE) r = mul_rn(d, r);     // D.mvMul(y)
    T s = div_rn(r, d);
    for (int k0 = 0; k0 < width; k0 += kChunk) {
        int js[kChunk];
        T vs[kChunk], xs[kChunk];
#pragma unroll
        for (int u = 0; u < kChunk; u++) js[u] = k0 + u < width ? col[(int64_t)(k0 + u) * cnt + q] : -1;
#pragma unroll
        for (int u = 0; u < kChunk; u++) {
            vs[u] = js[u] >= 0 ? val[(int64_t)(k0 + u) * cnt + q] : (T)0;
            xs[u] = js[u] >= 0 ? sol[js[u]] : (T)0;
        }
#pragma unroll
        for (int u = 0; u < kChunk; u++)
            if (js[u] >= 0) s = add_rn(s, mul_rn(div_rn(-xs[u], d), vs[u]));
        if (js[kChunk - 1] < 0) break;
    }
    sol[i] = s;
    if (ADDX) x[i] = add_rn(x[i], s);
}

template <typename T, bool SCALE, bool ADDX>
__global__ void k_trsv_level(int cnt, int width, const int* __restrict__ rows, const int* __restrict__ col,
                             const T* __restrict__ val, const T* __restrict__ diag, const T* __restrict__ rhs, T* sol,
                             T* x, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= cnt) return;
    trsv_row<T, SCALE, ADDX, 8>(q, cnt, width, rows, col, val, diag, rhs, sol, x);
}

// Levels [l0, l1) in one CTA or one cluster of kClusterCtas CTAs, one row per
// thread (every level of the run fits the threads).  A thread loads the next
// level's row data (row, diagonal, right-hand side, the first 8 entries)
// before the barrier that ends the current level, so a level costs one round
// trip for the solution entries it reads.  In a cluster the barrier
// (release / acquire at cluster scope) orders the level's solution stores
// before the next level's loads, which read through L2 (ld.global.cg) so that
// no CTA sees a line its own L1 cached before another CTA wrote it.
template <typename T>
struct RowPre {
    int i = -1;          // row, -1 when this thread has none in the level
    int cnt = 0, w = 0, q = 0;
    int64_t b = 0;
    T d = 0, r = 0;
    int js[8];
    T vs[8];
};

template <typename T, bool SCALE>
__device__ __forceinline__ void row_prefetch(RowPre<T>& p, int l, int tid, const int* __restrict__ lstart,
                                             const int* __restrict__ lwidth, const int64_t* __restrict__ lbase,
                                             const int* __restrict__ rows, const int* __restrict__ col,
                                             const T* __restrict__ val, const T* __restrict__ diag,
                                             const T* __restrict__ rhs)
{
    const int s0 = lstart[l];
    p.cnt = lstart[l + 1] - s0;
    p.w = lwidth[l];
    p.b = lbase[l];
    p.q = tid;
    p.i = tid < p.cnt ? rows[s0 + tid] : -1;
    if (p.i < 0) return;
    p.d = diag[p.i];
    p.r = rhs[p.i];
    if (SCALE) p.r = mul_rn(p.d, p.r);
#pragma unroll
    for (int u = 0; u < 8; u++) {
        p.js[u] = u < p.w ? col[p.b + (int64_t)u * p.cnt + tid] : -1;
        p.vs[u] = p.js[u] >= 0 ? val[p.b + (int64_t)u * p.cnt + tid] : (T)0;
    }
}

// the loop of the level-run kernels; CL = 1: one CTA, __syncthreads between
// levels (same SM: block-scope visibility); CL = kClusterCtas: a cluster
// barrier between levels and solution loads through L2
template <typename T, bool SCALE, bool ADDX, int CL>
__device__ __forceinline__ void level_run(int l0, int l1, int tid, const int* __restrict__ lstart,
                                          const int* __restrict__ lwidth, const int64_t* __restrict__ lbase,
                                          const int* __restrict__ rows, const int* __restrict__ col,
                                          const T* __restrict__ val, const T* __restrict__ diag,
                                          const T* __restrict__ rhs, T* sol, T* x)
{
    auto ld = [&](int j) -> T { return CL > 1 ? __ldcg(sol + j) : sol[j]; };
    RowPre<T> p;
    row_prefetch<T, SCALE>(p, l0, tid, lstart, lwidth, lbase, rows, col, val, diag, rhs);
    for (int l = l0; l < l1; l++) {
        if (p.i >= 0) {
            T xs[8];
#pragma unroll
            for (int u = 0; u < 8; u++) xs[u] = p.js[u] >= 0 ? ld(p.js[u]) : (T)0;
            T s = div_rn(p.r, p.d);
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (p.js[u] >= 0) s = add_rn(s, mul_rn(div_rn(-xs[u], p.d), p.vs[u]));
            for (int k0 = 8; k0 < p.w && p.js[7] >= 0; k0 += 8) {   // rows longer than the prefetched chunk
                int js[8];
                T vs[8], ys[8];
#pragma unroll
                for (int u = 0; u < 8; u++) js[u] = k0 + u < p.w ? col[p.b + (int64_t)(k0 + u) * p.cnt + p.q] : -1;
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    vs[u] = js[u] >= 0 ? val[p.b + (int64_t)(k0 + u) * p.cnt + p.q] : (T)0;
                    ys[u] = js[u] >= 0 ? ld(js[u]) : (T)0;
                }
#pragma unroll
                for (int u = 0; u < 8; u++)
                    if (js[u] >= 0) s = add_rn(s, mul_rn(div_rn(-ys[u], p.d), vs[u]));
                if (js[7] < 0) break;
            }
            sol[p.i] = s;
            if (ADDX) x[p.i] = add_rn(x[p.i], s);
        }
        if (l + 1 < l1) row_prefetch<T, SCALE>(p, l + 1, tid, lstart, lwidth, lbase, rows, col, val, diag, rhs);
        if (CL > 1) {
            cooperative_groups::this_cluster().sync();
        } else {
            __syncthreads();
        }
    }
}

template <typename T, bool SCALE, bool ADDX>
__global__ void __cluster_dims__(kClusterCtas, 1, 1) __launch_bounds__(kCtaThreads, 1)
    k_trsv_levels_cluster(int l0, int l1, const int* __restrict__ lstart, const int* __restrict__ lwidth,
                          const int64_t* __restrict__ lbase, const int* __restrict__ rows,
                          const int* __restrict__ col, const T* __restrict__ val, const T* __restrict__ diag,
                          const T* __restrict__ rhs, T* sol, T* x, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;      // uniform over the cluster: no barrier is left waiting
    const int tid = (int)cooperative_groups::this_cluster().block_rank() * blockDim.x + threadIdx.x;
    level_run<T, SCALE, ADDX, kClusterCtas>(l0, l1, tid, lstart, lwidth, lbase, rows, col, val, diag, rhs, sol, x);
}

template <typename T, bool SCALE, bool ADDX>
__global__ void __launch_bounds__(kCtaThreads, 1)
    k_trsv_levels_cta(int l0, int l1, const int* __restrict__ lstart, const int* __restrict__ lwidth,
                      const int64_t* __restrict__ lbase, const int* __restrict__ rows, const int* __restrict__ col,
                      const T* __restrict__ val, const T* __restrict__ diag, const T* __restrict__ rhs, T* sol, T* x,
                      const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    level_run<T, SCALE, ADDX, 1>(l0, l1, threadIdx.x, lstart, lwidth, lbase, rows, col, val, diag, rhs, sol, x);
}

// t = b - R x over the strict upper triangle (CSR in row order, ascending columns)
template <typename T>
__global__ void k_strict_upper(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                               const T* __restrict__ val, const T* __restrict__ b, const T* __restrict__ x,
                               T* __restrict__ t, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T s = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; k++) s = add_rn(s, mul_rn(val[k], x[col[k]]));
    t[i] = b[i] - s;
}

__global__ void k_gs_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// set-up (host): ordering, dependency levels, ELL arrays per level
// ---------------------------------------------------------------------------
static void build_tri(GSImpl::Tri& tri, int n, bool is_lower, const std::vector<int>& rank,
                      const std::vector<int>& order, const std::vector<int>& ptr, const std::vector<int>& col,
                      const std::vector<double>& val, cudaStream_t st)
{
    auto in_tri = [&](int i, int j) { return j != i && (is_lower ? rank[j] < rank[i] : rank[j] > rank[i]); };
    // level of each row: 1 + the deepest level it reads
    std::vector<int> lev(n, 0);
    int nl = 0;
    for (int p = 0; p < n; p++) {
        const int i = order[is_lower ? p : n - 1 - p];
        int L = 0;
        for (int k = ptr[i]; k < ptr[i + 1]; k++)
            if (in_tri(i, col[k])) L = std::max(L, lev[col[k]] + 1);
        lev[i] = L;
        nl = std::max(nl, L + 1);
    }
    if (n == 0) nl = 0;
    tri.nlevels = nl;
    // rows grouped by level, in ordering order inside a level
    tri.start.assign(nl + 1, 0);
    for (int i = 0; i < n; i++) tri.start[lev[i] + 1]++;
    for (int l = 0; l < nl; l++) tri.start[l + 1] += tri.start[l];
    std::vector<int> rows(n ? n : 1), fill(tri.start.begin(), tri.start.end() - (nl ? 1 : 0));
    for (int p = 0; p < n; p++) {
        const int i = order[is_lower ? p : n - 1 - p];
        rows[fill[lev[i]]++] = i;
    }
    // ELL per level
    tri.width.assign(nl, 0);
    tri.base.assign(nl + 1, 0);
    for (int l = 0; l < nl; l++) {
        int w = 0;
        for (int q = tri.start[l]; q < tri.start[l + 1]; q++) {
            const int i = rows[q];
            int c = 0;
            for (int k = ptr[i]; k < ptr[i + 1]; k++) c += in_tri(i, col[k]);
            w = std::max(w, c);
        }
        tri.width[l] = w;
        tri.base[l + 1] = tri.base[l] + (int64_t)w * (tri.start[l + 1] - tri.start[l]);
    }
    const int64_t total = nl ? tri.base[nl] : 0;
    std::vector<int> ecol(total ? total : 1, -1);
    std::vector<double> eval(total ? total : 1, 0.0);
    for (int l = 0; l < nl; l++) {
        const int cnt = tri.start[l + 1] - tri.start[l];
        for (int q = 0; q < cnt; q++) {
            const int i = rows[tri.start[l] + q];
            int k2 = 0;
            for (int k = ptr[i]; k < ptr[i + 1]; k++) {
                if (!in_tri(i, col[k])) continue;
                const int64_t at = tri.base[l] + (int64_t)k2 * cnt + q;
                ecol[at] = col[k];
                eval[at] = val[k];
                k2++;
            }
        }
    }
    // launch segments
    tri.segs.clear();
    for (int l = 0; l < nl;) {
        GSImpl::Tri::Seg sg;
        sg.l0 = l;
        if (tri.start[l + 1] - tri.start[l] > kCtaMaxRows) {
            sg.l1 = l + 1;
            sg.cta = false;
        } else {
            int e = l + 1, mx = tri.start[l + 1] - tri.start[l];
            while (e < nl && tri.start[e + 1] - tri.start[e] <= kCtaMaxRows) {
                mx = std::max(mx, tri.start[e + 1] - tri.start[e]);
                e++;
            }
            sg.l1 = e;
            sg.cta = true;
            sg.cluster = mx > kCtaThreads;
        }
        tri.segs.push_back(sg);
        l = sg.l1;
    }
    tri.rows.alloc((size_t)std::max(n, 1));
    tri.col.alloc((size_t)std::max<int64_t>(total, 1));
    tri.val.alloc((size_t)std::max<int64_t>(total, 1));
    tri.d_start.alloc((size_t)nl + 1);
    tri.d_width.alloc((size_t)std::max(nl, 1));
    tri.d_base.alloc((size_t)nl + 1);
    if (n) JFG_CUDA(cudaMemcpyAsync(tri.rows.p, rows.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    if (total) {
        JFG_CUDA(cudaMemcpyAsync(tri.col.p, ecol.data(), sizeof(int) * total, cudaMemcpyHostToDevice, st));
        JFG_CUDA(cudaMemcpyAsync(tri.val.p, eval.data(), sizeof(double) * total, cudaMemcpyHostToDevice, st));
    }
    JFG_CUDA(cudaMemcpyAsync(tri.d_start.p, tri.start.data(), sizeof(int) * (nl + 1), cudaMemcpyHostToDevice, st));
    if (nl) {
        JFG_CUDA(cudaMemcpyAsync(tri.d_width.p, tri.width.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
        JFG_CUDA(cudaMemcpyAsync(tri.d_base.p, tri.base.data(), sizeof(int64_t) * (nl + 1), cudaMemcpyHostToDevice,
                                 st));
    }
    JFG_CUDA(cudaStreamSynchronize(st));   // the host vectors above go out of scope
}

void GSImpl::init(Context* ctx, Matrix* M, int ord)
{
    JFG_CHECK(M->rows == M->cols, JFG_ERR_BAD_ARG, "must be square");
    JFG_CHECK(ord == JFG_GS_NATURAL || ord == JFG_GS_MULTICOLOR, JFG_ERR_BAD_ARG, "unknown Gauss-Seidel ordering");
    c = ctx;
    A = M;
    n = M->rows;
    ordering = ord;
    cudaStream_t st = ctx->stream;
    const int64_t nnz = M->nnz;
    std::vector<int> ptr(n + 1), col(nnz ? nnz : 1);
    std::vector<double> val(nnz ? nnz : 1), diag(n ? n : 1);
    JFG_CUDA(cudaMemcpyAsync(ptr.data(), M->csr_ptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (nnz) {
        JFG_CUDA(cudaMemcpyAsync(col.data(), M->csr_col.p, sizeof(int) * nnz, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(val.data(), M->csr_val.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost, st));
    }
    if (n) JFG_CUDA(cudaMemcpyAsync(diag.data(), M->diag.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; i++) JFG_CHECK(diag[i] != 0.0, JFG_ERR_SINGULAR, "Singular Matrix");

    // ordering
    rank.resize(n);
    std::vector<int> order(n);
    if (ord == JFG_GS_NATURAL) {
        std::iota(rank.begin(), rank.end(), 0);
        colours = 0;
    } else {
        // pattern of A^T for the symmetric adjacency
        std::vector<int> tptr(n + 1, 0), tcol(nnz ? nnz : 1);
        for (int64_t k = 0; k < nnz; k++) tptr[col[k] + 1]++;
        for (int i = 0; i < n; i++) tptr[i + 1] += tptr[i];
        {
            std::vector<int> f(tptr.begin(), tptr.end() - 1);
            for (int i = 0; i < n; i++)
                for (int k = ptr[i]; k < ptr[i + 1]; k++) tcol[f[col[k]]++] = i;
        }
        std::vector<int> colour(n, -1), seen;
        int nc = 0;
        for (int i = 0; i < n; i++) {
            auto mark = [&](int j) {
                if (j == i || colour[j] < 0) return;
                if ((int)seen.size() <= colour[j]) seen.resize(colour[j] + 1, -1);
                seen[colour[j]] = i;
            };
            for (int k = ptr[i]; k < ptr[i + 1]; k++) mark(col[k]);
            for (int k = tptr[i]; k < tptr[i + 1]; k++) mark(tcol[k]);
            int cc = 0;
            while (cc < (int)seen.size() && seen[cc] == i) cc++;
            colour[i] = cc;
            nc = std::max(nc, cc + 1);
        }
        colours = nc;
        std::vector<int> cstart(nc + 1, 0);
        for (int i = 0; i < n; i++) cstart[colour[i] + 1]++;
        for (int k = 0; k < nc; k++) cstart[k + 1] += cstart[k];
        for (int i = 0; i < n; i++) rank[i] = cstart[colour[i]]++;
    }
    for (int i = 0; i < n; i++) order[rank[i]] = i;
    build_tri(lower, n, true, rank, order, ptr, col, val, st);
    build_tri(upper, n, false, rank, order, ptr, col, val, st);

    // strict upper triangle in row order for GaussSeidelSmoother's b - R x
    std::vector<int> sp(n + 1, 0);
    std::vector<int> sc;
    std::vector<double> sv;
    for (int i = 0; i < n; i++) {
        for (int k = ptr[i]; k < ptr[i + 1]; k++)
            if (col[k] != i && rank[col[k]] > rank[i]) {
                sc.push_back(col[k]);
                sv.push_back(val[k]);
            }
        sp[i + 1] = (int)sc.size();
    }
    sup_ptr.alloc((size_t)n + 1);
    sup_col.alloc(std::max<size_t>(sc.size(), 1));
    sup_val.alloc(std::max<size_t>(sv.size(), 1));
    JFG_CUDA(cudaMemcpyAsync(sup_ptr.p, sp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    if (!sc.empty()) {
        JFG_CUDA(cudaMemcpyAsync(sup_col.p, sc.data(), sizeof(int) * sc.size(), cudaMemcpyHostToDevice, st));
        JFG_CUDA(cudaMemcpyAsync(sup_val.p, sv.data(), sizeof(double) * sv.size(), cudaMemcpyHostToDevice, st));
    }
    JFG_CUDA(cudaStreamSynchronize(st));
    sup_nnz = (int64_t)sc.size();
}

// ---------------------------------------------------------------------------
// precision copies
// ---------------------------------------------------------------------------
template <>
const double* GSImpl::tvals<double>(Tri& tri)
{
    return tri.val.p;
}
template <>
const float* GSImpl::tvals<float>(Tri& tri)
{
    if (!tri.val32.p) {
        const int64_t m = tri.nlevels ? tri.base[tri.nlevels] : 0;
        tri.val32.alloc((size_t)std::max<int64_t>(m, 1));
        if (m) k_gs_to_f32<<<nb(m), 256, 0, c->stream>>>(m, tri.val.p, tri.val32.p);
        JFG_CUDA(cudaGetLastError());
    }
    return tri.val32.p;
}
template <>
const double* GSImpl::dvals<double>()
{
    return A->diag.p;
}
template <>
const float* GSImpl::dvals<float>()
{
    if (!diag32.p) {
        diag32.alloc((size_t)std::max(n, 1));
        if (n) k_gs_to_f32<<<nb(n), 256, 0, c->stream>>>(n, A->diag.p, diag32.p);
        JFG_CUDA(cudaGetLastError());
    }
    return diag32.p;
}
template <>
const double* GSImpl::svals<double>()
{
    return sup_val.p;
}
template <>
const float* GSImpl::svals<float>()
{
    if (!sup_val32.p) {
        sup_val32.alloc((size_t)std::max<int64_t>(sup_nnz, 1));
        if (sup_nnz) k_gs_to_f32<<<nb(sup_nnz), 256, 0, c->stream>>>(sup_nnz, sup_val.p, sup_val32.p);
        JFG_CUDA(cudaGetLastError());
    }
    return sup_val32.p;
}

// ---------------------------------------------------------------------------
// solves
// ---------------------------------------------------------------------------
template <typename T, bool SCALE, bool ADDX>
void GSImpl::solve(Tri& tri, const T* rhs, T* sol, T* x, const int* done, cudaStream_t st)
{
    const T* v = tvals<T>(tri);
    const T* d = dvals<T>();
    for (const auto& sg : tri.segs) {
        if (sg.cta) {
            launch_ex(sg.cluster ? k_trsv_levels_cluster<T, SCALE, ADDX> : k_trsv_levels_cta<T, SCALE, ADDX>,
                      dim3(sg.cluster ? kClusterCtas : 1), dim3(kCtaThreads), 0, st, sg.l0, sg.l1,
                      (const int*)tri.d_start.p, (const int*)tri.d_width.p, (const int64_t*)tri.d_base.p,
                      (const int*)tri.rows.p, (const int*)tri.col.p, v, d, rhs, sol, x, done);
        } else {
            const int l = sg.l0;
            const int cnt = tri.start[l + 1] - tri.start[l];
            launch_ex(k_trsv_level<T, SCALE, ADDX>, dim3(nb(cnt)), dim3(256), 0, st, cnt, tri.width[l],
                      (const int*)(tri.rows.p + tri.start[l]), (const int*)(tri.col.p + tri.base[l]), v + tri.base[l],
                      d, rhs, sol, x, done);
        }
    }
}

template <typename T>
void GSImpl::backward(const T* rhs, T* sol, const int* done, cudaStream_t st)
{
    solve<T, false, false>(upper, rhs, sol, (T*)nullptr, done, st);
}

template <typename T>
void GSImpl::forward_fbgs(const T* y, T* sol, T* x, const int* done, cudaStream_t st)
{
    solve<T, true, true>(lower, y, sol, x, done, st);
}

template <typename T>
void GSImpl::forward(const T* rhs, T* sol, const int* done, cudaStream_t st)
{
    solve<T, false, false>(lower, rhs, sol, (T*)nullptr, done, st);
}

template <typename T>
void GSImpl::strict_upper(const T* b, const T* x, T* t, const int* done, cudaStream_t st)
{
    launch_ex(k_strict_upper<T>, dim3(nb(std::max(n, 1))), dim3(256), 0, st, n, (const int*)sup_ptr.p,
              (const int*)sup_col.p, svals<T>(), b, x, t, done);
}

template void GSImpl::backward<double>(const double*, double*, const int*, cudaStream_t);
template void GSImpl::backward<float>(const float*, float*, const int*, cudaStream_t);
template void GSImpl::forward_fbgs<double>(const double*, double*, double*, const int*, cudaStream_t);
template void GSImpl::forward_fbgs<float>(const float*, float*, float*, const int*, cudaStream_t);
template void GSImpl::forward<double>(const double*, double*, const int*, cudaStream_t);
template void GSImpl::forward<float>(const float*, float*, const int*, cudaStream_t);
template void GSImpl::strict_upper<double>(const double*, const double*, double*, const int*, cudaStream_t);
template void GSImpl::strict_upper<float>(const float*, const float*, float*, const int*, cudaStream_t);

GSImpl* gs_of(jfg_gs* g) { return g ? &g->g : nullptr; }

}  // namespace jfg

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct jfg_mat;
namespace jfg {
cudaStream_t ctx_stream(jfg_ctx* ctx);
int ctx_device(jfg_ctx* ctx);
void ctx_set_error(jfg_ctx* ctx, const std::string& msg);
Context* ctx_context(jfg_ctx* ctx);
Matrix* mat_of(jfg_mat* m);
jfg_ctx* mat_ctx(jfg_mat* m);
}  // namespace jfg

namespace {
template <typename F>
int gguard(jfg_ctx* ctx, F&& f)
{
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(ctx)));
        return f();
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(ctx, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        jfg::ctx_set_error(ctx, "host out of memory");
        return JFG_ERR_CUDA;
    }
}
}  // namespace

extern "C" {

int jfg_gs_create(jfg_ctx* ctx, jfg_mat* A, int ordering, jfg_gs** out)
{
    if (!ctx || !A || !out) return JFG_ERR_BAD_ARG;
    *out = nullptr;
    return gguard(ctx, [&]() -> int {
        JFG_CHECK(jfg::mat_ctx(A) == ctx, JFG_ERR_BAD_ARG, "matrix from another context");
        auto* g = new jfg_gs();
        g->ctx = ctx;
        try {
            g->g.init(jfg::ctx_context(ctx), jfg::mat_of(A), ordering);
        } catch (...) {
            delete g;
            throw;
        }
        *out = g;
        return JFG_OK;
    });
}

int jfg_gs_free(jfg_gs* g)
{
    if (!g) return JFG_ERR_BAD_ARG;
    cudaStreamSynchronize(jfg::ctx_stream(g->ctx));
    delete g;
    return JFG_OK;
}

int jfg_gs_info(jfg_gs* g, int* forward_levels, int* backward_levels, int* colours)
{
    if (!g) return JFG_ERR_BAD_ARG;
    if (forward_levels) *forward_levels = g->g.lower.nlevels;
    if (backward_levels) *backward_levels = g->g.upper.nlevels;
    if (colours) *colours = g->g.colours;
    return JFG_OK;
}

int jfg_gs_ranks(jfg_gs* g, int* h_rank)
{
    if (!g || (!h_rank && g->g.n)) return JFG_ERR_BAD_ARG;
    std::copy(g->g.rank.begin(), g->g.rank.end(), h_rank);
    return JFG_OK;
}

}  // extern "C"
