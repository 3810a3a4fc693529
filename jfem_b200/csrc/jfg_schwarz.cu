// Overlapping Schwarz smoothers on the device: patch-local dense inverses
// (DirectSolver), multiplicative / coloured multiplicative / additive
// subspace corrections (schwarz/*.java).
//
// Layout in HBM: patch p's sorted DOF list is dofs[pptr[p] .. pptr[p+1]) and
// the transpose of the m_p x m_p inverse of R_p A R_p^T sits at inv + inv_off[p]
// (column-major inverse).  Patches whose local operators are identical (the
// interior patches of a structured grid) share one inverse, found by hashing
// the local matrices, so the inverses the sweeps stream stay in L2.
// One sweep step over a colour is one launch with a CTA per patch: the CTA
// gathers the patch rows of b - A x straight from A's CSR rows (no global
// residual vector), multiplies by the patch inverse (warp per row, coalesced
// along the row) and adds omega * correction into x.  That fusion is exact
// when the colour's patches share no DOF and no matrix entry couples one
// patch's rows to another's DOFs (checked on the device at setup); other
// colours, and the additive variant, write local solutions to a buffer and a
// second kernel adds them per DOF in ascending patch order, so every sum
// keeps the reference's order of additions.
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>

#include "jfg_krylov.cuh"
#include "jfg_schwarz.cuh"

namespace jfg {
namespace {

constexpr int kSchThreads = 256;
constexpr int kMaxPatch = 1024;       // DOFs per patch
// patches up to this size are inverted in shared memory: 8 m^2 + 24 m bytes
// (229,824 at m = 168) plus ~100 static bytes stay under the 227 KB opt-in limit
constexpr int kSmemInvMax = 168;

struct CsrView {
    const int* rp;
    const int* col;
    const double* val;
};

// R A R^T of one patch into M (m x m, row-major), then Gauss-Jordan inversion
// in place with partial pivoting (largest |pivot|, first index on ties) and
// the column interchanges undone in reverse order at the end.
template <bool SMEM>
__global__ void __launch_bounds__(kSchThreads)
    k_patch_inverse(int mcap, CsrView A, const int* __restrict__ plist, const int64_t* __restrict__ pptr,
                    const int* __restrict__ dofs, const int64_t* __restrict__ inv_off, double* __restrict__ inv,
                    int* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    double* Ms = reinterpret_cast<double*>(smraw);
    double* rowk = Ms + (SMEM ? (size_t)mcap * mcap : 0);
    double* fac = rowk + mcap;
    int* sdof = reinterpret_cast<int*>(fac + mcap);
    int* piv = sdof + mcap;
    __shared__ double wv[kSchThreads / 32];
    __shared__ int wi[kSchThreads / 32];
    __shared__ int s_sing;
    const int p = plist[blockIdx.x];
    const int64_t off = pptr[p];
    const int m = (int)(pptr[p + 1] - off);
    double* M = SMEM ? Ms : inv + inv_off[p];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int i = tid; i < m; i += blockDim.x) sdof[i] = dofs[off + i];
    for (int64_t e = tid; e < (int64_t)m * m; e += blockDim.x) M[e] = 0.0;
    if (tid == 0) s_sing = 0;
    __syncthreads();
    // RestrictionMatrix.selectFrom: keep the entries whose row and column are both in the patch
    for (int i = tid; i < m; i += blockDim.x) {
        const int g = sdof[i];
        for (int k = A.rp[g]; k < A.rp[g + 1]; k++) {
            const int c = A.col[k];
            int lo = 0, hi = m - 1, j = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                const int v = sdof[mid];
                if (v == c) {
                    j = mid;
                    break;
                }
                if (v < c)
                    lo = mid + 1;
                else
                    hi = mid - 1;
            }
            if (j >= 0) M[(size_t)i * m + j] = A.val[k];
        }
    }
    __syncthreads();
    for (int k = 0; k < m; k++) {
        double bv = -1.0;
        int bi = m;
        for (int r = k + tid; r < m; r += blockDim.x) {
            const double v = fabs(M[(size_t)r * m + k]);
            if (v > bv) {
                bv = v;
                bi = r;
            }
        }
        for (int o = 16; o; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            wv[warp] = bv;
            wi[warp] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double b = wv[0];
            int ii = wi[0];
            for (int w = 1; w < nw; w++)
                if (wv[w] > b || (wv[w] == b && wi[w] < ii)) {
                    b = wv[w];
                    ii = wi[w];
                }
            piv[k] = ii;
            if (!(b > 0.0) || !isfinite(b)) s_sing = 1;
        }
        __syncthreads();
        if (s_sing) break;
        const int pr = piv[k];
        if (pr != k)
            for (int j = tid; j < m; j += blockDim.x) {
                const double a = M[(size_t)k * m + j];
                M[(size_t)k * m + j] = M[(size_t)pr * m + j];
                M[(size_t)pr * m + j] = a;
            }
        __syncthreads();
        const double d = 1.0 / M[(size_t)k * m + k];
        __syncthreads();
        for (int j = tid; j < m; j += blockDim.x) {
            const double v = (j == k ? 1.0 : M[(size_t)k * m + j]) * d;
            rowk[j] = v;
            M[(size_t)k * m + j] = v;
        }
        for (int i = tid; i < m; i += blockDim.x) fac[i] = (i == k) ? 0.0 : M[(size_t)i * m + k];
        __syncthreads();
        for (int i = warp; i < m; i += nw) {
            if (i == k) continue;
            const double f = fac[i];
            double* Mi = M + (size_t)i * m;
            for (int j = lane; j < m; j += 32) {
                const double a = (j == k) ? 0.0 : Mi[j];
                Mi[j] = a - f * rowk[j];
            }
        }
        __syncthreads();
    }
    if (!s_sing) {
        // each thread owns fixed rows, so the interchanges need no barrier between steps
        for (int k = m - 1; k >= 0; k--) {
            const int pr = piv[k];
            if (pr == k) continue;
            for (int i = tid; i < m; i += blockDim.x) {
                const double a = M[(size_t)i * m + k];
                M[(size_t)i * m + k] = M[(size_t)i * m + pr];
                M[(size_t)i * m + pr] = a;
            }
        }
    }
    __syncthreads();
    // stored transposed (the apply kernels read it column by column)
    if (SMEM) {
        double* out = inv + inv_off[p];
        for (int64_t e = tid; e < (int64_t)m * m; e += blockDim.x) {
            const int j = (int)(e / m), i = (int)(e - (int64_t)j * m);
            out[e] = Ms[(size_t)i * m + j];
        }
    } else {
        for (int64_t e = tid; e < (int64_t)m * m; e += blockDim.x) {
            const int i = (int)(e / m), j = (int)(e - (int64_t)i * m);
            if (i < j) {
                const double a = M[(size_t)i * m + j];
                M[(size_t)i * m + j] = M[(size_t)j * m + i];
                M[(size_t)j * m + i] = a;
            }
        }
    }
    if (tid == 0) status[blockIdx.x] = s_sing;
}

// Two 64-bit hashes of R A R^T per patch (entries in row order, columns
// ascending), so that patches with identical local operators share one
// inverse: on structured grids every interior patch has the same matrix.
__device__ __forceinline__ uint64_t mix64(uint64_t h, uint64_t v, uint64_t k1, uint64_t k2)
{
    h ^= v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    h ^= h >> 31;
    h *= k1;
    h ^= h >> 29;
    h *= k2;
    h ^= h >> 32;
    return h;
}

__global__ void __launch_bounds__(kSchThreads)
    k_patch_hash(CsrView A, const int64_t* __restrict__ pptr, const int* __restrict__ dofs, uint64_t* __restrict__ out)
{
    __shared__ int sdof[kMaxPatch];
    __shared__ uint64_t rh[2][kMaxPatch];
    const int p = blockIdx.x;
    const int64_t off = pptr[p];
    const int m = (int)(pptr[p + 1] - off);
    for (int i = threadIdx.x; i < m; i += blockDim.x) sdof[i] = dofs[off + i];
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        uint64_t h1 = 0x1234567ULL + (uint64_t)i, h2 = 0x89abcdefULL ^ ((uint64_t)i << 20);
        const int g = sdof[i];
        for (int k = A.rp[g]; k < A.rp[g + 1]; k++) {
            const int c = A.col[k];
            int lo = 0, hi = m - 1, j = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                const int v = sdof[mid];
                if (v == c) {
                    j = mid;
                    break;
                }
                if (v < c)
                    lo = mid + 1;
                else
                    hi = mid - 1;
            }
            if (j < 0) continue;
            const uint64_t bits = (uint64_t)__double_as_longlong(A.val[k]);
            const uint64_t key = ((uint64_t)(uint32_t)j << 32) ^ (uint64_t)(uint32_t)i;
            h1 = mix64(mix64(h1, key, 0xbf58476d1ce4e5b9ULL, 0x94d049bb133111ebULL), bits, 0xbf58476d1ce4e5b9ULL,
                       0x94d049bb133111ebULL);
            h2 = mix64(mix64(h2, bits, 0x7fb5d329728ea185ULL, 0x81dadef4bc2dd44dULL), key, 0x7fb5d329728ea185ULL,
                       0x81dadef4bc2dd44dULL);
        }
        rh[0][i] = h1;
        rh[1][i] = h2;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        const uint64_t k1 = threadIdx.x ? 0x7fb5d329728ea185ULL : 0xbf58476d1ce4e5b9ULL;
        const uint64_t k2 = threadIdx.x ? 0x81dadef4bc2dd44dULL : 0x94d049bb133111ebULL;
        uint64_t h = (uint64_t)m * 0x100000001b3ULL;
        for (int i = 0; i < m; i++) h = mix64(h, rh[threadIdx.x][i], k1, k2);
        out[2 * (size_t)p + threadIdx.x] = h;
    }
}

// One patch: local residual rows of b - A x, times the patch inverse; either
// x += omega * correction (direct) or the correction into lsol[pptr[p] + i].
// Built for memory-level parallelism: the row ranges of all patch rows are
// fetched in one pass, the residual rows are summed by groups of 8 lanes (32
// rows in flight per CTA), and the inverse is stored transposed so that
// thread i walks column j of row i with every warp reading 32 consecutive
// entries per j (coalesced, many independent loads in flight per thread).
constexpr int kRowLanes = 4;     // lanes per residual row: 64 rows in flight per CTA
constexpr int kRowUnroll = 8;    // entries per lane fetched before any product (rows <= 32 entries in one shot)

// sr[i] = b[sdof[i]] - (A x)[sdof[i]] for the m staged rows (row ranges in
// srs / sre): kRowLanes lanes per row, lane `sub` summing the entries sub,
// sub + kRowLanes, ... in order, then a butterfly over the lanes.  Every row
// is summed the same way whatever the block size.
template <typename T>
__device__ __forceinline__ void residual_rows(const CsrView& A, int m, const int* sdof, const int* srs,
                                              const int* sre, const T* b, const T* x, double* sr)
{
    const int tid = threadIdx.x;
    const int sub = tid & (kRowLanes - 1);
    const int per_pass = blockDim.x / kRowLanes;
    for (int i0 = 0; i0 < m; i0 += per_pass) {          // uniform trip count: the shuffles see full warps
        const int i = i0 + tid / kRowLanes;
        double acc = 0.0;
        if (i < m) {
            const int k0 = srs[i] + sub, k1 = sre[i];
            int c[kRowUnroll];
            double v[kRowUnroll];
#pragma unroll
            for (int u = 0; u < kRowUnroll; u++) {      // all index/value loads first
                const int k = k0 + u * kRowLanes;
                c[u] = k < k1 ? __ldg(A.col + k) : -1;
                v[u] = k < k1 ? __ldg(A.val + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kRowUnroll; u++)
                if (c[u] >= 0) acc += v[u] * (double)x[c[u]];
            for (int k = k0 + kRowUnroll * kRowLanes; k < k1; k += kRowLanes) acc += A.val[k] * (double)x[A.col[k]];
        }
#pragma unroll
        for (int o = 1; o < kRowLanes; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (i < m && sub == 0) sr[i] = (double)b[sdof[i]] - acc;
    }
}

template <typename T, typename IT>
__device__ __forceinline__ void patch_correct(const CsrView& A, int p, const int64_t* __restrict__ pptr,
                                              const int* __restrict__ dofs, const int64_t* __restrict__ inv_off,
                                              const IT* __restrict__ inv, const T* b, T* x, double om,
                                              double* lsol, bool direct, int* sdof, int* srs, int* sre, double* sr)
{
    const int tid = threadIdx.x;
    const int64_t off = pptr[p];
    const int m = (int)(pptr[p + 1] - off);
    for (int i = tid; i < m; i += blockDim.x) {
        const int g = dofs[off + i];
        sdof[i] = g;
        srs[i] = A.rp[g];
        sre[i] = A.rp[g + 1];
    }
    __syncthreads();
    residual_rows<T>(A, m, sdof, srs, sre, b, x, sr);
    __syncthreads();
    const IT* At = inv + inv_off[p];                    // transposed: At[j * m + i] = inverse(i, j)
    for (int i = tid; i < m; i += blockDim.x) {
        double acc = 0.0;
#pragma unroll 16
        for (int j = 0; j < m; j++) acc += (double)__ldg(At + (size_t)j * m + i) * sr[j];
        if (direct) {
            const int g = sdof[i];
            x[g] = (T)((double)x[g] + acc * om);
        } else {
            lsol[off + i] = acc;
        }
    }
    __syncthreads();
}

template <typename T, typename IT>
__global__ void __launch_bounds__(kSchThreads, 5)
    k_schwarz_patches(CsrView A, const int* __restrict__ plist, const int64_t* __restrict__ pptr,
                      const int* __restrict__ dofs, const int64_t* __restrict__ inv_off, const IT* __restrict__ inv,
                      const T* b, T* x, double om, double* lsol, int direct, const int* done)
{
    if (done && *done) return;
    __shared__ int sdof[kMaxPatch], srs[kMaxPatch], sre[kMaxPatch];
    __shared__ double sr[kMaxPatch];
    patch_correct<T, IT>(A, plist[blockIdx.x], pptr, dofs, inv_off, inv, b, x, om, lsol, direct != 0, sdof, srs, sre,
                         sr);
}

// Fast colour steps of independent colours (the fused direct step).  Both
// kernels walk batches of up to kMaxBatch patches that share one inverse (the
// interior patches of a structured grid; batch q holds the patches
// bpat[bptr[q] .. bptr[q + 1])): the residual rows of all patches of a batch
// are gathered together, then each inverse entry is read once and applied to
// every patch of the batch.  Per patch the sums are those of patch_correct in
// the same order, so the result is the same bit for bit.
//   k_schwarz_batch (colours with many more patches than SMs, e.g. the finest
//     level): four CTAs of 256 threads per SM (measured best of 2-4 patches
//     per batch x 256 / 512 threads), the inverse read from L2;
//   k_schwarz_colour (the other colours, about one batch per SM): the batch's
//     inverse is copied into shared memory by cp.async in the background of
//     its DOF staging and residual rows, so the inverse product reads shared
//     memory; a CTA with several batches reloads it only when the inverse
//     changes (the batches are sorted by inverse).
constexpr int kMaxBatch = 4;
constexpr int kBatchThreads = 512;
constexpr int kBatchRows = 1024;      // patch rows per batch of k_schwarz_batch
constexpr int kColThreads = 1024;
constexpr size_t kColSmemMax = 226 * 1024;

template <typename T, typename IT, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
    k_schwarz_batch(CsrView A, const int* __restrict__ bpat, const int* __restrict__ bptr,
                    const int64_t* __restrict__ pptr, const int* __restrict__ dofs,
                    const int64_t* __restrict__ inv_off, const IT* __restrict__ inv, const T* b, T* x, double om,
                    const int* done)
{
    if (done && *done) return;
    __shared__ int sdof[kBatchRows], srs[kBatchRows], sre[kBatchRows];
    __shared__ double sr[kBatchRows];
    const int tid = threadIdx.x;
    const int q0 = bptr[blockIdx.x];
    const int np_ = bptr[blockIdx.x + 1] - q0;
    const int p0 = bpat[q0];
    const int m = (int)(pptr[p0 + 1] - pptr[p0]);      // the same for every patch of the batch
    const int rows = np_ * m;
    for (int k = tid; k < rows; k += blockDim.x) {
        const int pi = k / m, i = k - pi * m;
        const int g = dofs[pptr[bpat[q0 + pi]] + i];
        sdof[k] = g;
        srs[k] = A.rp[g];
        sre[k] = A.rp[g + 1];
    }
    __syncthreads();
    residual_rows<T>(A, rows, sdof, srs, sre, b, x, sr);
    __syncthreads();
    const IT* At = inv + inv_off[p0];                   // transposed: At[j * m + i] = inverse(i, j)
    for (int i = tid; i < m; i += blockDim.x) {
        double acc[kMaxBatch];
#pragma unroll
        for (int q = 0; q < kMaxBatch; q++) acc[q] = 0.0;
#pragma unroll 16
        for (int j = 0; j < m; j++) {
            const double a = (double)__ldg(At + (size_t)j * m + i);
#pragma unroll
            for (int q = 0; q < kMaxBatch; q++)
                if (q < np_) acc[q] += a * sr[q * m + j];
        }
#pragma unroll
        for (int q = 0; q < kMaxBatch; q++)
            if (q < np_) {
                const int g = sdof[q * m + i];
                x[g] = (T)((double)x[g] + acc[q] * om);
            }
    }
}

__device__ __forceinline__ void cp_async_bytes(void* sdst, const void* gsrc, int bytes)
{
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}

// Dynamic shared memory of k_schwarz_colour: one inverse (mcap x mcap, IT),
// then rows_cap ints x 3 and rows_cap doubles.
template <typename IT>
__host__ __device__ constexpr size_t col_smem_inv(int mcap) { return ((size_t)mcap * mcap * sizeof(IT) + 15) / 16 * 16; }
__host__ __device__ constexpr size_t col_smem_rows(int rows_cap)
{
    return ((size_t)3 * rows_cap * sizeof(int) + 15) / 16 * 16 + (size_t)rows_cap * sizeof(double);
}

// SM = false (patches whose inverse does not fit shared memory): the inverse
// is read from global memory, the rest is the same.
template <typename T, typename IT, bool SM>
__global__ void __launch_bounds__(kColThreads, 1)
    k_schwarz_colour(CsrView A, const int* __restrict__ bpat, const int* __restrict__ bptr, int nbatch,
                     const int64_t* __restrict__ pptr, const int* __restrict__ dofs,
                     const int64_t* __restrict__ inv_off, const IT* __restrict__ inv, int mcap, int rows_cap,
                     const T* b, T* x, double om, const int* done)
{
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char col_smem[];
    const int tid = threadIdx.x;
    IT* sAt = reinterpret_cast<IT*>(col_smem);
    const size_t inv_bytes = SM ? col_smem_inv<IT>(mcap) : 0;
    int* sdof = reinterpret_cast<int*>(col_smem + inv_bytes);
    int* srs = sdof + rows_cap;
    int* sre = srs + rows_cap;
    double* sr = reinterpret_cast<double*>(col_smem + inv_bytes + (((size_t)3 * rows_cap * sizeof(int) + 15) / 16 * 16));
    int64_t loaded = -1;                                           // the inverse in shared memory
    for (int qb = blockIdx.x; qb < nbatch; qb += gridDim.x) {     // the same trip count on every thread
        const int q0 = bptr[qb];
        const int np_ = bptr[qb + 1] - q0;
        const int p0 = bpat[q0];
        const int m = (int)(pptr[p0 + 1] - pptr[p0]);             // the same for every patch of the batch
        const int rows = np_ * m;
        const int64_t off = inv_off[p0];
        if (SM && off != loaded) {   // this batch's inverse into shared memory, in the background
            const size_t bytes = (size_t)m * m * sizeof(IT);
            const unsigned char* src = reinterpret_cast<const unsigned char*>(inv + off);
            unsigned char* dst = reinterpret_cast<unsigned char*>(sAt);
            const int g = ((reinterpret_cast<uintptr_t>(src) | bytes) & 15) == 0 ? 16 : (int)sizeof(IT);
            for (size_t k = (size_t)tid * g; k < bytes; k += (size_t)blockDim.x * g) cp_async_bytes(dst + k, src + k, g);
            loaded = off;
        }
        cp_async_commit();
        for (int k = tid; k < rows; k += blockDim.x) {
            const int pi = k / m, i = k - pi * m;
            const int g = dofs[pptr[bpat[q0 + pi]] + i];
            sdof[k] = g;
            srs[k] = A.rp[g];
            sre[k] = A.rp[g + 1];
        }
        __syncthreads();
        residual_rows<T>(A, rows, sdof, srs, sre, b, x, sr);
        cp_async_wait<0>();
        __syncthreads();
        const IT* Ag = inv + off;
        for (int i = tid; i < m; i += blockDim.x) {               // sAt[j * m + i] = inverse(i, j)
            double acc[kMaxBatch];
#pragma unroll
            for (int q = 0; q < kMaxBatch; q++) acc[q] = 0.0;
#pragma unroll 16
            for (int j = 0; j < m; j++) {
                const double a = SM ? (double)sAt[(size_t)j * m + i] : (double)__ldg(Ag + (size_t)j * m + i);
#pragma unroll
                for (int q = 0; q < kMaxBatch; q++)
                    if (q < np_) acc[q] += a * sr[q * m + j];
            }
#pragma unroll
            for (int q = 0; q < kMaxBatch; q++)
                if (q < np_) {
                    const int g = sdof[q * m + i];
                    x[g] = (T)((double)x[g] + acc[q] * om);
                }
        }
        __syncthreads();   // the next batch overwrites the staged rows (and perhaps the inverse)
    }
}

// MultiplicativeSubspaceCorrection: the patches of plist one after another
// in a single CTA (each step sees the previous steps' updates).
template <typename T, typename IT>
__global__ void __launch_bounds__(kSchThreads)
    k_schwarz_seq(CsrView A, const int* __restrict__ plist, int count, const int64_t* __restrict__ pptr,
                  const int* __restrict__ dofs, const int64_t* __restrict__ inv_off, const IT* __restrict__ inv,
                  const T* b, T* x, const int* done)
{
    if (done && *done) return;
    __shared__ int sdof[kMaxPatch], srs[kMaxPatch], sre[kMaxPatch];
    __shared__ double sr[kMaxPatch];
    for (int q = 0; q < count; q++)
        patch_correct<T, IT>(A, plist[q], pptr, dofs, inv_off, inv, b, x, 1.0, nullptr, true, sdof, srs, sre, sr);
}

// x[d] = x[d] + omega * c_1 + omega * c_2 + ... (coloured) or
// x[d] = x[d] + (0 + omega * c_1 + omega * c_2 + ...) (additive), contributions
// in ascending patch order.
template <typename T, bool ADDFIRST>
__global__ void k_schwarz_scatter(int64_t nt, const int* __restrict__ touched, const int64_t* __restrict__ tptr,
                                  const int64_t* __restrict__ slots, const double* __restrict__ lsol, double om,
                                  T* x, const int* done)
{
    if (done && *done) return;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
        const int d = touched[t];
        if (ADDFIRST) {
            double s = 0.0;
            for (int64_t k = tptr[t]; k < tptr[t + 1]; k++) s = s + lsol[slots[k]] * om;
            x[d] = (T)((double)x[d] + s);
        } else {
            double v = (double)x[d];
            for (int64_t k = tptr[t]; k < tptr[t + 1]; k++) v = v + lsol[slots[k]] * om;
            x[d] = (T)v;
        }
    }
}

__global__ void k_mark(const int* __restrict__ plist, const int64_t* __restrict__ pptr, const int* __restrict__ dofs,
                       int* owner, int* flag)
{
    const int p = plist[blockIdx.x];
    for (int64_t i = pptr[p] + threadIdx.x; i < pptr[p + 1]; i += blockDim.x) {
        const int old = atomicCAS(&owner[dofs[i]], -1, p);
        if (old != -1 && old != p) atomicOr(flag, 1);
    }
}

__global__ void k_check(CsrView A, const int* __restrict__ plist, const int64_t* __restrict__ pptr,
                        const int* __restrict__ dofs, const int* __restrict__ owner, int* flag)
{
    const int p = plist[blockIdx.x];
    for (int64_t i = pptr[p] + threadIdx.x; i < pptr[p + 1]; i += blockDim.x) {
        const int g = dofs[i];
        for (int k = A.rp[g]; k < A.rp[g + 1]; k++) {
            const int o = owner[A.col[k]];
            if (o != -1 && o != p) atomicOr(flag, 1);
        }
    }
}

__global__ void k_unmark(const int* __restrict__ plist, const int64_t* __restrict__ pptr, const int* __restrict__ dofs,
                         int* owner)
{
    const int p = plist[blockIdx.x];
    for (int64_t i = pptr[p] + threadIdx.x; i < pptr[p + 1]; i += blockDim.x) owner[dofs[i]] = -1;
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

CsrView csr_of(Matrix* A) { return CsrView{A->csr_ptr.p, A->csr_col.p, A->csr_val.p}; }

}  // namespace

void SchwarzImpl::build_scatter(Colour& col, const std::vector<int64_t>& hp, const std::vector<int>& hd,
                                const std::vector<int>& patches, std::vector<int>& h_touched,
                                std::vector<int64_t>& h_tptr, std::vector<int64_t>& h_slots)
{
    std::vector<std::pair<int, int64_t>> e;   // (dof, slot) in ascending patch order
    for (int p : patches)
        for (int64_t i = hp[p]; i < hp[p + 1]; i++) e.emplace_back(hd[i], i);
    std::stable_sort(e.begin(), e.end(),
                     [](const std::pair<int, int64_t>& a, const std::pair<int, int64_t>& b) { return a.first < b.first; });
    col.t_start = (int64_t)h_touched.size();
    for (size_t k = 0; k < e.size(); k++) {
        if (k == 0 || e[k].first != e[k - 1].first) {
            h_touched.push_back(e[k].first);
            h_tptr.push_back((int64_t)h_slots.size());
        }
        h_slots.push_back(e[k].second);
    }
    col.t_count = (int64_t)h_touched.size() - col.t_start;
}

void SchwarzImpl::init(Context* ctx, Matrix* Am, int kind_, double omega_, int np_, const int64_t* h_pptr,
                       const int* h_dofs, int ncolours, const int* colour_ptr, const int* colour_patches)
{
    c = ctx;
    A = Am;
    n = Am->rows;
    kind = kind_;
    omega = omega_;
    np = np_;
    cudaStream_t st = c->stream;
    JFG_CHECK(Am->rows == Am->cols, JFG_ERR_BAD_ARG, "Schwarz needs a square matrix");
    JFG_CHECK(kind >= JFG_SCHWARZ_MULTIPLICATIVE && kind <= JFG_SCHWARZ_ADDITIVE, JFG_ERR_BAD_ARG,
              "unknown subspace correction");
    JFG_CHECK(np >= 1 && h_pptr && h_dofs && h_pptr[0] == 0, JFG_ERR_BAD_ARG, "no patches");
    JFG_CHECK(std::isfinite(omega), JFG_ERR_BAD_ARG, "bad omega");
    // sorted patch DOF lists (the TreeSet order of CartesianUpFrontSchwarz.buildRestrictionMatrix)
    std::vector<int64_t> hp(h_pptr, h_pptr + np + 1);
    std::vector<int> hd;
    std::vector<int64_t> hoff(np + 1, 0);
    max_m = 0;
    for (int p = 0; p < np; p++) {
        JFG_CHECK(hp[p + 1] > hp[p], JFG_ERR_BAD_ARG, "empty patch");
        int64_t m = hp[p + 1] - hp[p];
        JFG_CHECK(m <= kMaxPatch, JFG_ERR_UNSUPPORTED, "patch larger than 1024 DOFs");
        std::vector<int> d(h_dofs + hp[p], h_dofs + hp[p + 1]);
        std::sort(d.begin(), d.end());
        for (size_t i = 0; i < d.size(); i++) {
            JFG_CHECK(d[i] >= 0 && d[i] < n, JFG_ERR_BAD_ARG, "patch DOF out of range");
            JFG_CHECK(i == 0 || d[i] != d[i - 1], JFG_ERR_BAD_ARG, "repeated DOF in a patch");
        }
        hd.insert(hd.end(), d.begin(), d.end());
        max_m = std::max<int>(max_m, (int)m);
        hoff[p + 1] = hoff[p] + m * m;
    }
    total_m = hp[np];
    pptr.alloc(np + 1);
    inv_off.alloc(np);
    dofs.alloc(total_m);
    flag.alloc(1);
    JFG_CUDA(cudaMemcpyAsync(pptr.p, hp.data(), sizeof(int64_t) * (np + 1), cudaMemcpyHostToDevice, st));
    JFG_CUDA(cudaMemcpyAsync(dofs.p, hd.data(), sizeof(int) * total_m, cudaMemcpyHostToDevice, st));
    // DirectSolver: every distinct patch operator is inverted once, up front
    std::vector<int> reps;                     // patches whose inverse is computed
    std::vector<int64_t> hoff2(np);
    const char* ed = getenv("JFEM_SCHWARZ_DEDUP");
    if (!(ed && ed[0] == '0')) {
        DevBuf<uint64_t> hh;
        hh.alloc(2 * (size_t)np);
        k_patch_hash<<<np, kSchThreads, 0, st>>>(csr_of(A), pptr.p, dofs.p, hh.p);
        JFG_CUDA(cudaGetLastError());
        note_launch();
        std::vector<uint64_t> h(2 * (size_t)np);
        JFG_CUDA(cudaMemcpyAsync(h.data(), hh.p, sizeof(uint64_t) * h.size(), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        std::map<std::tuple<int64_t, uint64_t, uint64_t>, int64_t> seen;
        int64_t tot = 0;
        for (int p = 0; p < np; p++) {
            const int64_t m = hp[p + 1] - hp[p];
            auto key = std::make_tuple(m, h[2 * (size_t)p], h[2 * (size_t)p + 1]);
            auto it = seen.find(key);
            if (it == seen.end()) {
                seen.emplace(key, tot);
                hoff2[p] = tot;
                reps.push_back(p);
                tot += m * m;
            } else {
                hoff2[p] = it->second;
            }
        }
        total_inv = tot;
    } else {
        for (int p = 0; p < np; p++) {
            hoff2[p] = hoff[p];
            reps.push_back(p);
        }
        total_inv = hoff[np];
    }
    nunique = (int)reps.size();
    inv.alloc(total_inv);
    JFG_CUDA(cudaMemcpyAsync(inv_off.p, hoff2.data(), sizeof(int64_t) * np, cudaMemcpyHostToDevice, st));
    DevBuf<int> pstat, d_reps;
    pstat.alloc(reps.size());
    d_reps.alloc(reps.size());
    JFG_CUDA(cudaMemcpyAsync(d_reps.p, reps.data(), sizeof(int) * reps.size(), cudaMemcpyHostToDevice, st));
    const bool smem = max_m <= kSmemInvMax;
    const int mcap = max_m;
    const unsigned nr = (unsigned)reps.size();
    size_t dyn = (smem ? (size_t)mcap * mcap * sizeof(double) : 0) + 2 * (size_t)mcap * sizeof(double) +
                 2 * (size_t)mcap * sizeof(int);
    if (smem) {
        JFG_CUDA(cudaFuncSetAttribute(k_patch_inverse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        k_patch_inverse<true><<<nr, kSchThreads, dyn, st>>>(mcap, csr_of(A), d_reps.p, pptr.p, dofs.p, inv_off.p,
                                                            inv.p, pstat.p);
    } else {
        JFG_CUDA(cudaFuncSetAttribute(k_patch_inverse<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        k_patch_inverse<false><<<nr, kSchThreads, dyn, st>>>(mcap, csr_of(A), d_reps.p, pptr.p, dofs.p, inv_off.p,
                                                             inv.p, pstat.p);
    }
    JFG_CUDA(cudaGetLastError());
    note_launch();
    std::vector<int> hs(reps.size());
    JFG_CUDA(cudaMemcpyAsync(hs.data(), pstat.p, sizeof(int) * hs.size(), cudaMemcpyDeviceToHost, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    for (size_t q = 0; q < reps.size(); q++)
        JFG_CHECK(hs[q] == 0, JFG_ERR_SINGULAR, "a patch matrix is singular (patch " + std::to_string(reps[q]) + ")");

    std::vector<int> h_touched;
    std::vector<int64_t> h_tptr, h_slots;
    bool need_buffer = false;
    if (kind == JFG_SCHWARZ_MULTIPLICATIVE) {
        std::vector<int> s(2 * (size_t)np);
        for (int p = 0; p < np; p++) {
            s[p] = p;
            s[2 * (size_t)np - 1 - p] = p;
        }
        seq.alloc(s.size());
        JFG_CUDA(cudaMemcpyAsync(seq.p, s.data(), sizeof(int) * s.size(), cudaMemcpyHostToDevice, st));
    } else if (kind == JFG_SCHWARZ_COLORED) {
        JFG_CHECK(ncolours >= 1 && colour_ptr && colour_patches && colour_ptr[0] == 0, JFG_ERR_BAD_ARG,
                  "coloured Schwarz needs colours");
        std::vector<int> hc;
        DevBuf<int> owner;
        owner.alloc(n);
        JFG_CUDA(cudaMemsetAsync(owner.p, 0xff, sizeof(int) * n, st));
        for (int k = 0; k < ncolours; k++) {
            JFG_CHECK(colour_ptr[k + 1] >= colour_ptr[k], JFG_ERR_BAD_ARG, "bad colour pointer");
            std::vector<int> pl(colour_patches + colour_ptr[k], colour_patches + colour_ptr[k + 1]);
            std::sort(pl.begin(), pl.end());     // IntRBTreeSet iteration order
            for (size_t i = 0; i < pl.size(); i++) {
                JFG_CHECK(pl[i] >= 0 && pl[i] < np, JFG_ERR_BAD_ARG, "colour names an unknown patch");
                JFG_CHECK(i == 0 || pl[i] != pl[i - 1], JFG_ERR_BAD_ARG, "patch repeated in a colour");
            }
            Colour col;
            col.start = (int)hc.size();
            col.count = (int)pl.size();
            hc.insert(hc.end(), pl.begin(), pl.end());
            colours.push_back(col);
        }
        cpat.alloc(std::max<size_t>(hc.size(), 1));
        JFG_CUDA(cudaMemcpyAsync(cpat.p, hc.data(), sizeof(int) * hc.size(), cudaMemcpyHostToDevice, st));
        for (auto& col : colours) {
            if (col.count == 0) continue;
            JFG_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
            const int* pl = cpat.p + col.start;
            k_mark<<<col.count, kSchThreads, 0, st>>>(pl, pptr.p, dofs.p, owner.p, flag.p);
            k_check<<<col.count, kSchThreads, 0, st>>>(csr_of(A), pl, pptr.p, dofs.p, owner.p, flag.p);
            k_unmark<<<col.count, kSchThreads, 0, st>>>(pl, pptr.p, dofs.p, owner.p);
            JFG_CUDA(cudaGetLastError());
            note_launch(3);
            int hf = 0;
            JFG_CUDA(cudaMemcpyAsync(&hf, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            JFG_CUDA(cudaStreamSynchronize(st));
            col.independent = hf == 0;
            if (!col.independent) {
                std::vector<int> pls(hc.begin() + col.start, hc.begin() + col.start + col.count);
                build_scatter(col, hp, hd, pls, h_touched, h_tptr, h_slots);
                need_buffer = true;
            }
        }
        // Independent colours run as batches of up to kMaxBatch patches that
        // share one inverse: on k_schwarz_batch when the colour has many more
        // patches than SMs, else on k_schwarz_colour (about one batch per SM,
        // the inverse in shared memory); JFEM_SCHWARZ_FAST=0 keeps one CTA per
        // patch reading the inverse from global memory.
        const char* ef = getenv("JFEM_SCHWARZ_FAST");
        fast = !(ef && ef[0] == '0');
        // launch shape of k_schwarz_batch: patches per batch (2..4) and threads per CTA (256 or 512)
        const char* eb = getenv("JFEM_SCHWARZ_BATCH");
        if (eb && eb[0] >= '2' && eb[0] <= '4') batch_max = eb[0] - '0';
        const char* et = getenv("JFEM_SCHWARZ_BATCH_THREADS");
        if (et && atoi(et) == 512) batch_threads = 512;
        int dev = 0, nsm = 148;
        JFG_CUDA(cudaGetDevice(&dev));
        JFG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        std::vector<int> h_bpat, h_bptr;
        for (auto& col : colours) {
            for (int q = 0; q < col.count; q++) {
                const int pp = hc[col.start + q];
                col.mcap = std::max<int>(col.mcap, (int)(hp[pp + 1] - hp[pp]));
            }
            if (!fast || !col.independent || col.count == 0) continue;
            int pb = 0;
            if ((col.count + kMaxBatch - 1) / kMaxBatch > nsm && kBatchRows / col.mcap >= 2) {
                col.kern = 1;
                pb = std::min(batch_max, kBatchRows / col.mcap);
            } else {
                pb = std::min(kMaxBatch, (col.count + nsm - 1) / nsm);
                col.rows_cap = pb * col.mcap;
                // the inverse in shared memory when it fits (the FP32 copy is half the
                // size: the FP64 bound decides), else read from global memory
                col.kern = col_smem_inv<double>(col.mcap) + col_smem_rows(col.rows_cap) <= kColSmemMax ? 2 : 3;
                if (col_smem_rows(col.rows_cap) > kColSmemMax) {
                    col.kern = 0;
                    continue;
                }
            }
            std::vector<int> pl(hc.begin() + col.start, hc.begin() + col.start + col.count);
            std::stable_sort(pl.begin(), pl.end(), [&](int a, int b2) { return hoff2[a] < hoff2[b2]; });
            col.b_start = (int)h_bptr.size();
            size_t q = 0;
            while (q < pl.size()) {
                size_t e = q + 1;
                while (e < pl.size() && (int)(e - q) < pb && hoff2[pl[e]] == hoff2[pl[q]]) e++;
                h_bptr.push_back((int)h_bpat.size());
                h_bpat.insert(h_bpat.end(), pl.begin() + q, pl.begin() + e);
                q = e;
            }
            col.b_count = (int)h_bptr.size() - col.b_start;
            h_bptr.push_back((int)h_bpat.size());   // the end of the colour's last batch
            col.grid = col.kern >= 2 ? std::min(col.b_count, nsm) : col.b_count;
        }
        if (!h_bpat.empty()) {
            bpat.alloc(h_bpat.size());
            bptr.alloc(h_bptr.size());
            JFG_CUDA(cudaMemcpyAsync(bpat.p, h_bpat.data(), sizeof(int) * h_bpat.size(), cudaMemcpyHostToDevice, st));
            JFG_CUDA(cudaMemcpyAsync(bptr.p, h_bptr.data(), sizeof(int) * h_bptr.size(), cudaMemcpyHostToDevice, st));
        }
        // ColoredMultiplicativeSubspaceCorrection.solve starts with patch 0 alone
        int zero = 0;
        seq.alloc(1);
        JFG_CUDA(cudaMemcpyAsync(seq.p, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
    } else {
        std::vector<int> pl(np);
        std::iota(pl.begin(), pl.end(), 0);
        all.start = 0;
        all.count = np;
        cpat.alloc(np);
        JFG_CUDA(cudaMemcpyAsync(cpat.p, pl.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
        build_scatter(all, hp, hd, pl, h_touched, h_tptr, h_slots);
        need_buffer = true;
    }
    if (need_buffer) {
        h_tptr.push_back((int64_t)h_slots.size());
        touched.alloc(std::max<size_t>(h_touched.size(), 1));
        tptr.alloc(h_tptr.size());
        slots.alloc(std::max<size_t>(h_slots.size(), 1));
        lsol.alloc(total_m);
        JFG_CUDA(cudaMemcpyAsync(touched.p, h_touched.data(), sizeof(int) * h_touched.size(), cudaMemcpyHostToDevice,
                                 st));
        JFG_CUDA(cudaMemcpyAsync(tptr.p, h_tptr.data(), sizeof(int64_t) * h_tptr.size(), cudaMemcpyHostToDevice, st));
        JFG_CUDA(cudaMemcpyAsync(slots.p, h_slots.data(), sizeof(int64_t) * h_slots.size(), cudaMemcpyHostToDevice,
                                 st));
    }
    JFG_CUDA(cudaStreamSynchronize(st));
}

const float* SchwarzImpl::inverses32()
{
    if (!inv32.p) {
        inv32.alloc(total_inv);
        k_to_f32<<<148 * 8, 256, 0, c->stream>>>(total_inv, inv.p, inv32.p);
        JFG_CUDA(cudaGetLastError());
        note_launch();
    }
    return inv32.p;
}

template <typename T>
static const void* inv_of(SchwarzImpl* s);
template <>
const void* inv_of<double>(SchwarzImpl* s) { return s->inv.p; }
template <>
const void* inv_of<float>(SchwarzImpl* s) { return s->inverses32(); }

template <typename T>
void SchwarzImpl::colour_step(const Colour& col, const T* b, T* x, double om, const int* done, cudaStream_t st)
{
    if (col.count == 0) return;
    using IT = T;
    const IT* iv = static_cast<const IT*>(inv_of<T>(this));
    const bool additive = kind == JFG_SCHWARZ_ADDITIVE;
    if (col.independent && !additive) {
        if (col.kern == 1) {
            if (batch_threads == 256)
                k_schwarz_batch<T, IT, 256><<<col.b_count, 256, 0, st>>>(csr_of(A), bpat.p, bptr.p + col.b_start,
                                                                         pptr.p, dofs.p, inv_off.p, iv, b, x, om,
                                                                         done);
            else
                k_schwarz_batch<T, IT, kBatchThreads><<<col.b_count, kBatchThreads, 0, st>>>(
                    csr_of(A), bpat.p, bptr.p + col.b_start, pptr.p, dofs.p, inv_off.p, iv, b, x, om, done);
        } else if (col.kern == 2) {
            static bool attr = false;      // per instantiation
            if (!attr) {
                JFG_CUDA(cudaFuncSetAttribute(k_schwarz_colour<T, IT, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kColSmemMax));
                attr = true;
            }
            const size_t smem = col_smem_inv<IT>(col.mcap) + col_smem_rows(col.rows_cap);
            k_schwarz_colour<T, IT, true><<<col.grid, kColThreads, smem, st>>>(
                csr_of(A), bpat.p, bptr.p + col.b_start, col.b_count, pptr.p, dofs.p, inv_off.p, iv, col.mcap,
                col.rows_cap, b, x, om, done);
        } else if (col.kern == 3) {
            static bool attr = false;      // per instantiation
            if (!attr) {
                JFG_CUDA(cudaFuncSetAttribute(k_schwarz_colour<T, IT, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kColSmemMax));
                attr = true;
            }
            k_schwarz_colour<T, IT, false><<<col.grid, kColThreads, col_smem_rows(col.rows_cap), st>>>(
                csr_of(A), bpat.p, bptr.p + col.b_start, col.b_count, pptr.p, dofs.p, inv_off.p, iv, col.mcap,
                col.rows_cap, b, x, om, done);
        } else {
            k_schwarz_patches<T, IT><<<col.count, kSchThreads, 0, st>>>(csr_of(A), cpat.p + col.start, pptr.p,
                                                                        dofs.p, inv_off.p, iv, b, x, om, nullptr, 1,
                                                                        done);
        }
        JFG_CUDA(cudaGetLastError());
        note_launch();
        return;
    }
    k_schwarz_patches<T, IT><<<col.count, kSchThreads, 0, st>>>(csr_of(A), cpat.p + col.start, pptr.p, dofs.p,
                                                                inv_off.p, iv, b, x, om, lsol.p, 0, done);
    const int64_t nt = col.t_count;
    const unsigned grid = (unsigned)std::min<int64_t>((nt + 255) / 256, 148 * 16);
    if (nt > 0) {
        if (additive)
            k_schwarz_scatter<T, true><<<grid, 256, 0, st>>>(nt, touched.p + col.t_start, tptr.p + col.t_start,
                                                             slots.p, lsol.p, om, x, done);
        else
            k_schwarz_scatter<T, false><<<grid, 256, 0, st>>>(nt, touched.p + col.t_start, tptr.p + col.t_start,
                                                              slots.p, lsol.p, om, x, done);
    }
    JFG_CUDA(cudaGetLastError());
    note_launch(nt > 0 ? 2 : 1);
}

template <typename T>
void SchwarzImpl::apply(const T* b, T* x, const Scratch&, const int* done, cudaStream_t st)
{
    using IT = T;
    const IT* iv = static_cast<const IT*>(inv_of<T>(this));
    if (kind == JFG_SCHWARZ_MULTIPLICATIVE) {
        // MultiplicativeSubspaceCorrection.apply: patches forward, then backward
        k_schwarz_seq<T, IT><<<1, kSchThreads, 0, st>>>(csr_of(A), seq.p, 2 * np, pptr.p, dofs.p, inv_off.p, iv, b, x,
                                                        done);
        JFG_CUDA(cudaGetLastError());
        note_launch();
    } else if (kind == JFG_SCHWARZ_COLORED) {
        // ColoredMultiplicativeSubspaceCorrection.apply: colours forward, then backward
        for (size_t k = 0; k < colours.size(); k++) colour_step<T>(colours[k], b, x, omega, done, st);
        for (size_t k = colours.size(); k-- > 0;) colour_step<T>(colours[k], b, x, omega, done, st);
    } else {
        // SubspaceCorrection.apply with AdditiveSubspaceCorrection.solve
        colour_step<T>(all, b, x, omega, done, st);
    }
}

template <typename T>
void SchwarzImpl::solve(const T* b, T* out, const Scratch& sc, const int* done, cudaStream_t st)
{
    using IT = T;
    const IT* iv = static_cast<const IT*>(inv_of<T>(this));
    JFG_CUDA(cudaMemsetAsync(out, 0, sizeof(T) * n, st));
    if (kind == JFG_SCHWARZ_MULTIPLICATIVE) {
        // MultiplicativeSubspaceCorrection.solve: patch 0 from b, then 1 .. np-1 on the running residual
        k_schwarz_seq<T, IT><<<1, kSchThreads, 0, st>>>(csr_of(A), seq.p, np, pptr.p, dofs.p, inv_off.p, iv, b, out,
                                                        done);
        JFG_CUDA(cudaGetLastError());
        note_launch();
    } else if (kind == JFG_SCHWARZ_COLORED) {
        k_schwarz_patches<T, IT><<<1, kSchThreads, 0, st>>>(csr_of(A), seq.p, pptr.p, dofs.p, inv_off.p, iv, b, out,
                                                            1.0, nullptr, 1, done);
        JFG_CUDA(cudaGetLastError());
        note_launch();
        for (size_t k = 0; k < colours.size(); k++) colour_step<T>(colours[k], b, out, omega, done, st);
    } else {
        colour_step<T>(all, b, out, omega, done, st);
    }
    (void)sc;
}

template void SchwarzImpl::apply<double>(const double*, double*, const Scratch&, const int*, cudaStream_t);
template void SchwarzImpl::apply<float>(const float*, float*, const Scratch&, const int*, cudaStream_t);
template void SchwarzImpl::solve<double>(const double*, double*, const Scratch&, const int*, cudaStream_t);
template void SchwarzImpl::solve<float>(const float*, float*, const Scratch&, const int*, cudaStream_t);

namespace {
void schwarz_hook(void* self, const double* r, double* z, const Scratch& sc, const int* done, cudaStream_t st)
{
    static_cast<jfg_schwarz*>(self)->s.solve<double>(r, z, sc, done, st);
}
}  // namespace

int schwarz_precond(void* h, Precond<double>& P, int n)
{
    auto* s = static_cast<jfg_schwarz*>(h);
    JFG_CHECK(s && s->s.n == n, JFG_ERR_BAD_ARG, "Schwarz preconditioner does not match the system size");
    P.kind = JFG_PREC_SCHWARZ;
    P.hook = schwarz_hook;
    P.hook_self = s;
    P.hook_uid = s->s.uid;
    P.n = n;
    return s->s.A->nblocks;
}

SchwarzImpl* schwarz_of(jfg_schwarz* s) { return s ? &s->s : nullptr; }

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
int sguard(jfg_ctx* ctx, F&& f)
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

int jfg_schwarz_create(jfg_ctx* ctx, jfg_mat* A, int kind, double omega, int npatches, const int64_t* patch_ptr,
                       const int* patch_dofs, int ncolors, const int* color_ptr, const int* color_patches,
                       jfg_schwarz** out)
{
    if (!ctx || !A || !out || npatches < 1 || !patch_ptr || !patch_dofs) return JFG_ERR_BAD_ARG;
    *out = nullptr;
    return sguard(ctx, [&]() -> int {
        JFG_CHECK(jfg::mat_ctx(A) == ctx, JFG_ERR_BAD_ARG, "matrix from another context");
        auto* s = new jfg_schwarz();
        s->ctx = ctx;
        try {
            s->s.init(jfg::ctx_context(ctx), jfg::mat_of(A), kind, omega, npatches, patch_ptr, patch_dofs, ncolors,
                      color_ptr, color_patches);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
        return JFG_OK;
    });
}

int jfg_schwarz_free(jfg_schwarz* s)
{
    if (!s) return JFG_ERR_BAD_ARG;
    cudaStreamSynchronize(jfg::ctx_stream(s->ctx));
    delete s;
    return JFG_OK;
}

int jfg_schwarz_info(jfg_schwarz* s, int* max_patch, int64_t* inverse_entries, int* independent_colors)
{
    if (!s) return JFG_ERR_BAD_ARG;
    if (max_patch) *max_patch = s->s.max_m;
    if (inverse_entries) *inverse_entries = s->s.total_inv;
    if (independent_colors) {
        int k = 0;
        for (auto& c : s->s.colours) k += c.independent ? 1 : 0;
        *independent_colors = k;
    }
    return JFG_OK;
}

static int schwarz_host_call(jfg_schwarz* s, int op, int runs, const double* h_in, double* h_x)
{
    if (!s || !h_in || !h_x || runs < 0) return JFG_ERR_BAD_ARG;
    return sguard(s->ctx, [&]() -> int {
        jfg::SchwarzImpl& S = s->s;
        cudaStream_t st = jfg::ctx_stream(s->ctx);
        jfg::DevBuf<double> b, x;
        b.alloc(S.n);
        x.alloc(S.n);
        JFG_CUDA(cudaMemcpyAsync(b.p, h_in, sizeof(double) * S.n, cudaMemcpyHostToDevice, st));
        if (op != 1) JFG_CUDA(cudaMemcpyAsync(x.p, h_x, sizeof(double) * S.n, cudaMemcpyHostToDevice, st));
        jfg::Scratch sc{};
        if (op == 0)
            S.apply<double>(b.p, x.p, sc, nullptr, st);
        else if (op == 1)
            S.solve<double>(b.p, x.p, sc, nullptr, st);
        else
            S.smooth<double>(runs, b.p, x.p, sc, nullptr, st);
        JFG_CUDA(cudaMemcpyAsync(h_x, x.p, sizeof(double) * S.n, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        return JFG_OK;
    });
}

int jfg_schwarz_apply(jfg_schwarz* s, const double* h_rhs, double* h_x) { return schwarz_host_call(s, 0, 1, h_rhs, h_x); }

int jfg_schwarz_solve(jfg_schwarz* s, const double* h_rhs, double* h_out)
{
    return schwarz_host_call(s, 1, 1, h_rhs, h_out);
}

int jfg_schwarz_smooth(jfg_schwarz* s, int runs, const double* h_rhs, double* h_x)
{
    return schwarz_host_call(s, 2, runs, h_rhs, h_x);
}

int jfg_schwarz_smooth_dev(jfg_schwarz* s, int runs, const double* d_rhs, double* d_x)
{
    if (!s || !d_rhs || !d_x || runs < 0) return JFG_ERR_BAD_ARG;
    return sguard(s->ctx, [&]() -> int {
        jfg::Scratch sc{};
        s->s.smooth<double>(runs, d_rhs, d_x, sc, nullptr, jfg::ctx_stream(s->ctx));
        JFG_CUDA(cudaStreamSynchronize(jfg::ctx_stream(s->ctx)));
        return JFG_OK;
    });
}

int jfg_schwarz_local_inverse(jfg_schwarz* s, int patch, int* m, int* h_dofs, double* h_inv)
{
    if (!s || patch < 0 || patch >= s->s.np) return JFG_ERR_BAD_ARG;
    return sguard(s->ctx, [&]() -> int {
        jfg::SchwarzImpl& S = s->s;
        cudaStream_t st = jfg::ctx_stream(s->ctx);
        int64_t se[2], off = 0;
        JFG_CUDA(cudaMemcpyAsync(se, S.pptr.p + patch, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaMemcpyAsync(&off, S.inv_off.p + patch, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        int mm = (int)(se[1] - se[0]);
        if (m) *m = mm;
        if (h_dofs) JFG_CUDA(cudaMemcpyAsync(h_dofs, S.dofs.p + se[0], sizeof(int) * mm, cudaMemcpyDeviceToHost, st));
        std::vector<double> t;
        if (h_inv) {
            t.resize((size_t)mm * mm);
            JFG_CUDA(cudaMemcpyAsync(t.data(), S.inv.p + off, sizeof(double) * mm * mm, cudaMemcpyDeviceToHost, st));
        }
        JFG_CUDA(cudaStreamSynchronize(st));
        if (h_inv)   // stored transposed on the device
            for (int i = 0; i < mm; i++)
                for (int j = 0; j < mm; j++) h_inv[(size_t)i * mm + j] = t[(size_t)j * mm + i];
        return JFG_OK;
    });
}

int jfg_schwarz_time(jfg_schwarz* s, int iters, double* ms_apply)
{
    if (!s || iters < 1 || !ms_apply) return JFG_ERR_BAD_ARG;
    return sguard(s->ctx, [&]() -> int {
        jfg::SchwarzImpl& S = s->s;
        cudaStream_t st = jfg::ctx_stream(s->ctx);
        jfg::DevBuf<double> b, x;
        b.alloc(S.n);
        x.alloc(S.n);
        JFG_CUDA(cudaMemsetAsync(b.p, 0, sizeof(double) * S.n, st));
        JFG_CUDA(cudaMemsetAsync(x.p, 0, sizeof(double) * S.n, st));
        jfg::Scratch sc{};
        S.apply<double>(b.p, x.p, sc, nullptr, st);
        cudaEvent_t e0, e1;
        JFG_CUDA(cudaEventCreate(&e0));
        JFG_CUDA(cudaEventCreate(&e1));
        JFG_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < iters; i++) S.apply<double>(b.p, x.p, sc, nullptr, st);
        JFG_CUDA(cudaEventRecord(e1, st));
        JFG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        JFG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_apply = ms / iters;
        return JFG_OK;
    });
}

}  // extern "C"
