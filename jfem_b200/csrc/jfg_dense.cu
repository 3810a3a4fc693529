// Dense FP64 LU with partial pivoting on the device: the coarsest multigrid
// level, the drop-in dense solve and dense inverses.
//
// Right-looking LU: for each column k one CTA picks the pivot (largest |a_ik|,
// lowest index on ties), swaps rows and scales the column; a grid then applies
// the rank-1 update to the trailing block.  Triangular solves run one CTA per
// right-hand side, column-oriented.
//
// Matrices of more than kNb columns are factored in panels of kNb columns
// (the same arithmetic in the same order, so the factors and pivots are those
// of the column-by-column loop bit for bit):
//   1. one CTA factors the panel (rows k0 .. n-1, one warp per row and one lane
//      per panel column): pivot, swap inside the panel, scale, rank-1 update
//      of the panel's remaining columns, for each of its kNb columns;
//   2. the panel's row interchanges are applied to every other column, in
//      order (one thread per column);
//   3. U12 = L11^-1 A12 for the panel's rows right of it (one thread per
//      column, L11 in shared memory; subtractions in ascending k);
//   4. A22 -= L21 U12 by 64 x 64 tiles, each entry subtracting the kNb
//      products in ascending k from its current value, one rounding each, as
//      the rank-1 updates of the column loop do.
// Four launches per kNb columns instead of two per column, and the trailing
// block is read and written once per panel instead of once per column.
#include <cooperative_groups.h>

#include "jfg_mg.cuh"

namespace cg = cooperative_groups;

namespace jfg {

namespace {

__global__ void k_lu_pivot(int n, double* A, int* piv, int k, int* info)
{
    __shared__ double best[1024];
    __shared__ int bidx[1024];
    double b = -1.0;
    int bi = k;
    for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
        double v = fabs(A[(size_t)i * n + k]);
        if (v > b) { b = v; bi = i; }
    }
    best[threadIdx.x] = b;
    bidx[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            double o = best[threadIdx.x + s];
            int oi = bidx[threadIdx.x + s];
            if (o > best[threadIdx.x] || (o == best[threadIdx.x] && oi < bidx[threadIdx.x])) {
                best[threadIdx.x] = o;
                bidx[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    int p = bidx[0];
    if (threadIdx.x == 0) {
        piv[k] = p;
        if (!(best[0] > 0.0)) *info = 1;
    }
    if (!(best[0] > 0.0)) return;
    if (p != k)
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            double t = A[(size_t)k * n + j];
            A[(size_t)k * n + j] = A[(size_t)p * n + j];
            A[(size_t)p * n + j] = t;
        }
    __syncthreads();
    double inv = 1.0 / A[(size_t)k * n + k];
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + k] *= inv;
}

__global__ void k_lu_update(int n, double* A, int k, const int* info)
{
    if (*info) return;
    int m = n - k - 1;
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m * m) return;
    int i = k + 1 + (int)(idx / m);
    int j = k + 1 + (int)(idx % m);
    A[(size_t)i * n + j] = __fma_rn(-A[(size_t)i * n + k], A[(size_t)k * n + j], A[(size_t)i * n + j]);
}

// (|a|, row) argmax over a CTA: the largest value, the lowest row on ties.
// The rule is associative and commutative, so any reduction order picks the
// same pivot as a sequential scan.  red_v / red_i hold one entry per warp.
__device__ __forceinline__ void argmax_step(double& b, int& bi, double o, int oi)
{
    if (o > b || (o == b && oi < bi)) {
        b = o;
        bi = oi;
    }
}
__device__ __forceinline__ void cta_argmax(double& b, int& bi, double* red_v, int* red_i)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) argmax_step(b, bi, __shfl_xor_sync(0xffffffffu, b, o), __shfl_xor_sync(0xffffffffu, bi, o));
    if (lane == 0) {
        red_v[warp] = b;
        red_i[warp] = bi;
    }
    __syncthreads();
    b = lane < nw ? red_v[lane] : -1.0;
    bi = lane < nw ? red_i[lane] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) argmax_step(b, bi, __shfl_xor_sync(0xffffffffu, b, o), __shfl_xor_sync(0xffffffffu, bi, o));
}

constexpr int kNb = 32;          // panel width (one lane per panel column)
constexpr int kPanelThreads = 512;
constexpr int kPanelRows = 8;    // panel rows per warp in flight

// Step 1: the panel of columns k0 .. k0 + nb - 1 (nb <= kNb), rows k0 .. n-1.
__global__ void __launch_bounds__(kPanelThreads)
k_lu_panel(int n, double* A, int* piv, int k0, int nb, int* info)
{
    __shared__ double red_v[32];
    __shared__ int red_i[32];
    __shared__ double urow[kNb];
    if (*info) return;                         // an earlier panel was singular
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = k0; k < k0 + nb; k++) {
        double b = -1.0;
        int bi = INT_MAX;
        for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
            const double v = fabs(A[(size_t)i * n + k]);
            if (v > b) { b = v; bi = i; }
        }
        cta_argmax(b, bi, red_v, red_i);
        const int p = bi;
        const bool ok = b > 0.0;
        if (threadIdx.x == 0) {
            piv[k] = p;
            if (!ok) *info = 1;
        }
        if (!ok) return;                       // the same decision on every thread
        if (warp == 0 && lane < nb) {          // swap rows k and p inside the panel
            const int c = k0 + lane;
            const double t = A[(size_t)k * n + c];
            const double u = A[(size_t)p * n + c];
            A[(size_t)k * n + c] = u;
            A[(size_t)p * n + c] = t;
            urow[lane] = u;
        }
        __syncthreads();
        const double inv = 1.0 / urow[k - k0];
        const int lk = k - k0;
        const bool upd = lane > lk && lane < nb;
        const double uk = upd ? urow[lane] : 0.0;
        // scale and rank-1 update of the panel rows below k: a warp takes
        // kPanelRows rows at a time with all their loads issued first
        for (int i0 = k + 1 + warp * kPanelRows; i0 < n; i0 += nw * kPanelRows) {
            double av[kPanelRows], cv[kPanelRows];
#pragma unroll
            for (int u = 0; u < kPanelRows; u++) {
                const int i = i0 + u;
                av[u] = i < n ? A[(size_t)i * n + k] : 0.0;
                cv[u] = (i < n && upd) ? A[(size_t)i * n + k0 + lane] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kPanelRows; u++) {
                const int i = i0 + u;
                if (i < n) {
                    const double l = av[u] * inv;
                    if (lane == lk) A[(size_t)i * n + k] = l;
                    if (upd) A[(size_t)i * n + k0 + lane] = __fma_rn(-l, uk, cv[u]);
                }
            }
        }
        __syncthreads();
    }
}

// Step 1 on a cluster of kPcCtas CTAs, the panel held in distributed shared
// memory: CTA c owns the panel rows k0 + c * rc .. + rc - 1 (rows padded to
// kNb + 1 doubles, so a column walk is free of bank conflicts).  Per column:
// each CTA finds its candidate pivot, a cluster barrier, every CTA picks the
// same pivot from the kPcCtas candidates (largest |a|, lowest row on ties),
// reads the pivot row (and the owner of row p the old row k) from the
// owners, a cluster barrier, the two rows are exchanged, and every CTA scales
// and updates its own rows.  The arithmetic of k_lu_panel, entry by entry.
constexpr int kPcCtas = 16;
constexpr int kPcThreads = 512;
constexpr int kPcStride = kNb + 1;

__global__ void __launch_bounds__(kPcThreads)
k_lu_panel_cl(int n, double* A, int* piv, int k0, int nb, int rc, int* info)
{
    extern __shared__ double P[];                 // rc x kPcStride
    __shared__ double cval[2];
    __shared__ int cidx[2];
    __shared__ double red_v[32];
    __shared__ int red_i[32];
    __shared__ double urow[kNb], krow[kNb];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int r0 = k0 + c * rc;                   // first global row of this CTA
    const int rn = max(0, min(rc, n - r0));       // rows owned
    const bool bad = *info != 0;                  // the same answer on every CTA
    if (!bad)
        for (int t = threadIdx.x; t < rn * 32; t += blockDim.x) {
            const int lr = t >> 5, cc = t & 31;
            if (cc < nb) P[lr * kPcStride + cc] = A[(size_t)(r0 + lr) * n + k0 + cc];
        }
    cl.sync();
    if (bad) return;
    for (int k = k0; k < k0 + nb; k++) {
        const int lk = k - k0, par = lk & 1;
        double b = -1.0;
        int bi = INT_MAX;
        for (int lr = max(0, k - r0) + threadIdx.x; lr < rn; lr += blockDim.x) {
            const double v = fabs(P[lr * kPcStride + lk]);
            if (v > b) { b = v; bi = r0 + lr; }
        }
        cta_argmax(b, bi, red_v, red_i);
        if (threadIdx.x == 0) {
            cval[par] = b;
            cidx[par] = bi;
        }
        cl.sync();
        // every warp: lane q reads CTA q's candidate, then the same pick on every thread
        double gb = lane < kPcCtas ? *cl.map_shared_rank(&cval[par], lane) : -1.0;
        int p = lane < kPcCtas ? *cl.map_shared_rank(&cidx[par], lane) : INT_MAX;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            argmax_step(gb, p, __shfl_xor_sync(0xffffffffu, gb, o), __shfl_xor_sync(0xffffffffu, p, o));
        const bool ok = gb > 0.0;
        if (c == 0 && threadIdx.x == 0) {
            piv[k] = ok ? p : k;
            if (!ok) *info = 1;
        }
        if (!ok) {
            cl.sync();                             // nobody leaves while others read its shared memory
            return;
        }
        const int ck = (k - k0) / rc, cp = (p - k0) / rc;
        if (warp == 0 && lane < nb) {
            const double* Pp = cl.map_shared_rank(P, cp);
            urow[lane] = Pp[(p - k0 - cp * rc) * kPcStride + lane];
            if (c == cp) {
                const double* Pk = cl.map_shared_rank(P, ck);
                krow[lane] = Pk[(k - k0 - ck * rc) * kPcStride + lane];
            }
        }
        cl.sync();
        if (warp == 0 && lane < nb) {
            if (c == ck) P[(k - r0) * kPcStride + lane] = urow[lane];
            if (c == cp && p != k) P[(p - r0) * kPcStride + lane] = krow[lane];
        }
        __syncthreads();
        const double inv = 1.0 / urow[lk];
        const bool upd = lane > lk && lane < nb;
        const double uk = upd ? urow[lane] : 0.0;
        for (int lr = max(0, k + 1 - r0) + warp; lr < rn; lr += nw) {
            const double l = P[lr * kPcStride + lk] * inv;
            if (lane == lk) P[lr * kPcStride + lk] = l;
            if (upd) P[lr * kPcStride + lane] = __fma_rn(-l, uk, P[lr * kPcStride + lane]);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < rn * 32; t += blockDim.x) {
        const int lr = t >> 5, cc = t & 31;
        if (cc < nb) A[(size_t)(r0 + lr) * n + k0 + cc] = P[lr * kPcStride + cc];
    }
    cl.sync();                                     // no CTA leaves while others may read its rows
}

// Step 2: the panel's interchanges on the columns outside it, in order.
__global__ void k_lu_swap(int n, double* A, const int* piv, int k0, int nb, const int* info)
{
    if (*info) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n - nb) return;
    if (c >= k0) c += nb;
    for (int k = k0; k < k0 + nb; k++) {
        const int p = piv[k];
        if (p != k) {
            const double t = A[(size_t)k * n + c];
            A[(size_t)k * n + c] = A[(size_t)p * n + c];
            A[(size_t)p * n + c] = t;
        }
    }
}

// Step 3: rows k0 .. k0 + nb - 1 of the columns right of the panel,
// U12 = L11^-1 A12 (unit lower L11).
__global__ void k_lu_trsm(int n, double* A, int k0, int nb, const int* info)
{
    if (*info) return;
    __shared__ double L[kNb][kNb + 1];
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) L[t / nb][t % nb] = A[(size_t)(k0 + t / nb) * n + k0 + t % nb];
    __syncthreads();
    const int c = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double x[kNb];
#pragma unroll
    for (int r = 0; r < kNb; r++)
        if (r < nb) {
            double v = A[(size_t)(k0 + r) * n + c];
#pragma unroll
            for (int q = 0; q < kNb; q++)
                if (q < r) v = __fma_rn(-L[r][q], x[q], v);
            x[r] = v;
            A[(size_t)(k0 + r) * n + c] = v;
        }
}

// Step 4: A22 -= L21 U12 on 64 x 64 tiles (256 threads, 4 x 4 entries each).
constexpr int kGT = 64;
__global__ void __launch_bounds__(256) k_lu_gemm(int n, double* A, int k0, int nb, const int* info)
{
    if (*info) return;
    __shared__ double Ls[kNb][kGT + 1];    // L21 tile, transposed: Ls[q][row]
    __shared__ double Us[kNb][kGT];        // U12 tile: Us[q][col]
    const int s = k0 + nb;                 // first row / column of A22
    const int r0 = s + blockIdx.y * kGT, c0 = s + blockIdx.x * kGT;
    for (int t = threadIdx.x; t < kGT * kNb; t += blockDim.x) {
        const int rr = t / kNb, q = t % kNb;
        Ls[q][rr] = (q < nb && r0 + rr < n) ? A[(size_t)(r0 + rr) * n + k0 + q] : 0.0;
        const int qq = t / kGT, cc = t % kGT;
        Us[qq][cc] = (qq < nb && c0 + cc < n) ? A[(size_t)(k0 + qq) * n + c0 + cc] : 0.0;
    }
    __syncthreads();
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;   // rows tr + 16 a, columns tc + 16 b
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int r = r0 + tr + 16 * a, c = c0 + tc + 16 * b;
            acc[a][b] = (r < n && c < n) ? A[(size_t)r * n + c] : 0.0;
        }
    for (int q = 0; q < nb; q++) {
        double l[4], u[4];
#pragma unroll
        for (int a = 0; a < 4; a++) l[a] = Ls[q][tr + 16 * a];
#pragma unroll
        for (int b = 0; b < 4; b++) u[b] = Us[q][tc + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[a][b] = __fma_rn(-l[a], u[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int r = r0 + tr + 16 * a, c = c0 + tc + 16 * b;
            if (r < n && c < n) A[(size_t)r * n + c] = acc[a][b];
        }
}

// One CTA per right-hand side column c: B[:, c] <- A^-1 B[:, c], with B
// row-major n x nrhs (column c strided by nrhs).
__global__ void k_lu_solve(int n, const double* LU, const int* piv, double* B, int nrhs)
{
    int c = blockIdx.x;
    double* x = B + c;
    if (threadIdx.x == 0)
        for (int k = 0; k < n; k++)
            if (piv[k] != k) {
                double t = x[(size_t)k * nrhs];
                x[(size_t)k * nrhs] = x[(size_t)piv[k] * nrhs];
                x[(size_t)piv[k] * nrhs] = t;
            }
    __syncthreads();
    for (int k = 0; k < n; k++) {           // forward, unit lower
        double xk = x[(size_t)k * nrhs];
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x)
            x[(size_t)i * nrhs] = __fma_rn(-LU[(size_t)i * n + k], xk, x[(size_t)i * nrhs]);
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; k--) {      // backward
        if (threadIdx.x == 0) x[(size_t)k * nrhs] /= LU[(size_t)k * n + k];
        __syncthreads();
        double xk = x[(size_t)k * nrhs];
        for (int i = threadIdx.x; i < k; i += blockDim.x)
            x[(size_t)i * nrhs] = __fma_rn(-LU[(size_t)i * n + k], xk, x[(size_t)i * nrhs]);
        __syncthreads();
    }
}

// The same solve by blocks of 32 unknowns, x in shared memory (n doubles of
// dynamic shared memory): warp 0 solves the block's triangle (lane = row,
// the solved entries passed by shuffles), then every thread applies the
// block's columns to the rows beyond it.  Each x_i receives its updates in
// the column loop's order (ascending k forward, descending k backward), one
// rounding each, so the result is the same bit for bit, with 2 n / 32
// barriers instead of 3 n.
__global__ void __launch_bounds__(512) k_lu_solve_blk(int n, const double* LU, const int* piv, double* B, int nrhs)
{
    extern __shared__ double xs[];
    const int c = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = B[(size_t)i * nrhs + c];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < n; k++)
            if (piv[k] != k) {
                const double t = xs[k];
                xs[k] = xs[piv[k]];
                xs[piv[k]] = t;
            }
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 32) {                 // forward, unit lower
        const int nb = min(32, n - b0);
        if (warp == 0) {
            const int i = b0 + lane;
            double xi = lane < nb ? xs[i] : 0.0;
            double lr[32];                                  // the row's entries of the block, loaded first
#pragma unroll
            for (int k = 0; k < 32; k++) lr[k] = (k < lane && lane < nb) ? LU[(size_t)i * n + b0 + k] : 0.0;
#pragma unroll
            for (int k = 0; k < 32; k++) {
                if (k < nb) {
                    const double xk = __shfl_sync(0xffffffffu, xi, k);
                    if (lane > k && lane < nb) xi = __fma_rn(-lr[k], xk, xi);
                }
            }
            if (lane < nb) xs[i] = xi;
        }
        __syncthreads();
        for (int i = b0 + nb + threadIdx.x; i < n; i += blockDim.x) {
            double xi = xs[i];
            const double* Li = LU + (size_t)i * n + b0;
            for (int h = 0; h < nb; h += 16) {           // 16 loads in flight, then the ordered sums
                double lv[16];
#pragma unroll
                for (int u = 0; u < 16; u++) lv[u] = h + u < nb ? Li[h + u] : 0.0;
#pragma unroll
                for (int u = 0; u < 16; u++)
                    if (h + u < nb) xi = __fma_rn(-lv[u], xs[b0 + h + u], xi);
            }
            xs[i] = xi;
        }
        __syncthreads();
    }
    for (int b1 = n; b1 > 0; b1 -= 32) {                 // backward, rows [b0, b1)
        const int b0 = max(0, b1 - 32), nb = b1 - b0;
        if (warp == 0) {
            const int i = b0 + lane;
            double xi = lane < nb ? xs[i] : 0.0;
            const double dii = lane < nb ? LU[(size_t)i * n + i] : 1.0;
            double ur[32];                                  // the row's entries of the block, loaded first
#pragma unroll
            for (int k = 0; k < 32; k++) ur[k] = (lane < k && k < nb) ? LU[(size_t)i * n + b0 + k] : 0.0;
#pragma unroll
            for (int k = 31; k >= 0; k--) {
                if (k < nb) {
                    if (lane == k) xi = xi / dii;
                    const double xk = __shfl_sync(0xffffffffu, xi, k);
                    if (lane < k) xi = __fma_rn(-ur[k], xk, xi);
                }
            }
            if (lane < nb) xs[i] = xi;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < b0; i += blockDim.x) {
            double xi = xs[i];
            const double* Ui = LU + (size_t)i * n + b0;
            for (int h = nb - 1; h >= 0; h -= 16) {      // 16 loads in flight, then the ordered sums
                double uv[16];
#pragma unroll
                for (int u = 0; u < 16; u++) uv[u] = h - u >= 0 ? Ui[h - u] : 0.0;
#pragma unroll
                for (int u = 0; u < 16; u++)
                    if (h - u >= 0) xi = __fma_rn(-uv[u], xs[b0 + h - u], xi);
            }
            xs[i] = xi;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) B[(size_t)i * nrhs + c] = xs[i];
}

constexpr size_t kSolveSmemMax = 200 * 1024;

// x <- A^-1 x for nrhs columns of the row-major n x nrhs block B, from the LU
// factors; the blocked kernel when x fits in shared memory.
void lu_solve_launch(int n, const double* LU, const int* piv, double* B, int nrhs, cudaStream_t st)
{
    const char* e = getenv("JFEM_LU_BLOCKED");
    const size_t smem = (size_t)n * sizeof(double);
    if (smem <= kSolveSmemMax && !(e && e[0] == '0')) {
        static bool attr = false;
        if (!attr) {
            JFG_CUDA(cudaFuncSetAttribute(k_lu_solve_blk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kSolveSmemMax));
            attr = true;
        }
        k_lu_solve_blk<<<nrhs, 512, smem, st>>>(n, LU, piv, B, nrhs);
    } else {
        k_lu_solve<<<nrhs, nrhs == 1 ? 1024 : 256, 0, st>>>(n, LU, piv, B, nrhs);
    }
    JFG_CUDA(cudaGetLastError());
}

__global__ void k_identity(int n, double* B)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * n) return;
    B[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

// Whether a 16-CTA cluster of k_lu_panel_cl with the largest dynamic shared
// memory it is launched with (200 KB per CTA) can be resident; asked once per
// process, on the first device that factors a large enough matrix.
bool panel_cluster_ok()
{
    static int cached = -1;
    if (cached >= 0) return cached == 1;
    constexpr size_t kMax = 200 * 1024;
    cached = 0;
    if (cudaFuncSetAttribute(k_lu_panel_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMax) != cudaSuccess ||
        cudaFuncSetAttribute(k_lu_panel_cl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kPcCtas);
    cfg.blockDim = dim3(kPcThreads);
    cfg.dynamicSmemBytes = kMax;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kPcCtas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, k_lu_panel_cl, &cfg) == cudaSuccess && nc >= 1) cached = 1;
    cudaGetLastError();
    return cached == 1;
}

void launch_panel(int n, double* A, int* piv, int k0, int nb, int* info, cudaStream_t st)
{
    const int R = n - k0;
    const int rc = (R + kPcCtas - 1) / kPcCtas;
    const size_t smem = (size_t)rc * kPcStride * sizeof(double);
    if (R >= 512 && smem <= 200 * 1024 && panel_cluster_ok()) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kPcCtas);
        cfg.blockDim = dim3(kPcThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kPcCtas;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        JFG_CUDA(cudaLaunchKernelEx(&cfg, k_lu_panel_cl, n, A, piv, k0, nb, rc, info));
    } else {
        k_lu_panel<<<1, kPanelThreads, 0, st>>>(n, A, piv, k0, nb, info);
    }
}

int lu_factor(Context* c, int n, double* A, int* piv, int* info)
{
    cudaStream_t st = c->stream;
    JFG_CUDA(cudaMemsetAsync(info, 0, sizeof(int), st));
    const char* e = getenv("JFEM_LU_BLOCKED");
    if (n > kNb && !(e && e[0] == '0')) {
        for (int k0 = 0; k0 < n; k0 += kNb) {
            const int nb = std::min(kNb, n - k0);
            launch_panel(n, A, piv, k0, nb, info, st);
            if (n - nb > 0) k_lu_swap<<<(unsigned)((n - nb + 255) / 256), 256, 0, st>>>(n, A, piv, k0, nb, info);
            const int m = n - k0 - nb;
            if (m > 0) {
                k_lu_trsm<<<(unsigned)((m + 127) / 128), 128, 0, st>>>(n, A, k0, nb, info);
                const unsigned g = (unsigned)((m + kGT - 1) / kGT);
                k_lu_gemm<<<dim3(g, g), 256, 0, st>>>(n, A, k0, nb, info);
            }
            JFG_CUDA(cudaGetLastError());
            note_launch(m > 0 ? 4 : 2);
        }
    } else {
        for (int k = 0; k < n; k++) {
            k_lu_pivot<<<1, 1024, 0, st>>>(n, A, piv, k, info);
            int m = n - k - 1;
            if (m > 0) {
                int64_t tot = (int64_t)m * m;
                k_lu_update<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, A, k, info);
            }
        }
    }
    JFG_CUDA(cudaGetLastError());
    int h = 0;
    JFG_CUDA(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    return h ? JFG_ERR_SINGULAR : JFG_OK;
}

}  // namespace

int dense_inverse_device(Context* c, int n, double* d_A, double* d_inv)
{
    if (n == 0) return JFG_OK;
    DevBuf<int> piv, info;
    piv.alloc(n);
    info.alloc(1);
    int st = lu_factor(c, n, d_A, piv.p, info.p);
    if (st != JFG_OK) return st;
    int64_t tot = (int64_t)n * n;
    k_identity<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(n, d_inv);
    lu_solve_launch(n, d_A, piv.p, d_inv, n, c->stream);
    JFG_CUDA(cudaGetLastError());
    JFG_CUDA(cudaStreamSynchronize(c->stream));
    return JFG_OK;
}

int dense_solve_device(Context* c, int n, double* d_A, const double* d_b, double* d_x)
{
    if (n == 0) return JFG_OK;
    DevBuf<int> piv, info;
    piv.alloc(n);
    info.alloc(1);
    int st = lu_factor(c, n, d_A, piv.p, info.p);
    if (st != JFG_OK) return st;
    if (d_x != d_b) JFG_CUDA(cudaMemcpyAsync(d_x, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    lu_solve_launch(n, d_A, piv.p, d_x, 1, c->stream);
    JFG_CUDA(cudaGetLastError());
    JFG_CUDA(cudaStreamSynchronize(c->stream));
    return JFG_OK;
}

}  // namespace jfg
