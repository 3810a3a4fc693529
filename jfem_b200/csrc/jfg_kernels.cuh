// Device building blocks: deterministic block/grid reductions, the
// row-block CSR SpMV with fused epilogues, and grid-stride vector kernels.
#pragma once
#include "jfg_common.cuh"

namespace jfg {

// ---------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums NR per-thread values over the CTA; the result is valid in thread 0.
// Fixed tree order, so repeated runs give bitwise-identical results.
template <int NR>
__device__ __forceinline__ void block_sum(double (&v)[NR])
{
    __shared__ double sh[NR][kThreads / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < NR; i++) {
        double t = warp_sum(v[i]);
        if (l == 0) sh[i][w] = t;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int i = 0; i < NR; i++) {
            double t = l < kThreads / 32 ? sh[i][l] : 0.0;
            v[i] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Grid reduction with a last-block finaliser.  Every CTA of the launch calls
// reduce() exactly once; the CTA that arrives last sums the per-CTA partials
// in index order and calls fin(totals).  The counter is re-armed to zero.
struct NoFin {
    __device__ void operator()(const double*) const {}
};

template <int NR, class Fin>
struct GridRed {
    double* partials;   // NR * gridDim.x
    unsigned* counter;
    Fin fin;
    __device__ __forceinline__ void reduce(double (&acc)[NR]) const
    {
        __shared__ bool last;
        block_sum<NR>(acc);
        const int G = gridDim.x;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < NR; i++) partials[(size_t)i * G + blockIdx.x] = acc[i];
            __threadfence();
            unsigned t = atomicAdd(counter, 1u);
            last = (t == (unsigned)G - 1);
        }
        __syncthreads();
        if (!last) return;
        __threadfence();
        double s[NR];
#pragma unroll
        for (int i = 0; i < NR; i++) {
            s[i] = 0;
            for (int j = threadIdx.x; j < G; j += kThreads) s[i] += __ldcg(partials + (size_t)i * G + j);
        }
        block_sum<NR>(s);
        if (threadIdx.x == 0) {
            fin(s);
            *counter = 0;
            __threadfence();
        }
    }
};

// ---------------------------------------------------------------------------
// typed 4-wide loads of matrix values
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load4(const double* p, double (&o)[4])
{
    double2 a = __ldg(reinterpret_cast<const double2*>(p));
    double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void load4(const float* p, float (&o)[4])
{
    float4 a = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
__device__ __forceinline__ void load4(const __nv_bfloat16* p, float (&o)[4])
{
    uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
    __nv_bfloat162 lo = *reinterpret_cast<__nv_bfloat162*>(&a.x);
    __nv_bfloat162 hi = *reinterpret_cast<__nv_bfloat162*>(&a.y);
    float2 fl = __bfloat1622float2(lo), fh = __bfloat1622float2(hi);
    o[0] = fl.x; o[1] = fl.y; o[2] = fh.x; o[3] = fh.y;
}
// Matrix-stream loads: every value and column entry is read once per product,
// so it is not allocated in L1 (which then keeps the x entries that
// neighbouring rows gather) and each L2 miss fetches 256 bytes.
__device__ __forceinline__ float ld_stream(const float* p)
{
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_stream(const double* p)
{
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int ld_stream(const int* p)
{
    int v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int ld_stream(const int16_t* p)
{
    short v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.s16 %0, [%1];" : "=h"(v) : "l"(p));
    return (int)v;
}
__device__ __forceinline__ __half ld_stream(const __half* p)
{
    unsigned short v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.b16 %0, [%1];" : "=h"(v) : "l"(p));
    return __ushort_as_half(v);
}
__device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16* p)
{
    unsigned short v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.b16 %0, [%1];" : "=h"(v) : "l"(p));
    return __ushort_as_bfloat16(v);
}

template <typename VT> struct AccOf { using T = VT; };
template <> struct AccOf<__nv_bfloat16> { using T = float; };
template <> struct AccOf<__half> { using T = float; };

__device__ __forceinline__ float to_acc(float v) { return v; }
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ float to_acc(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_acc(__half v) { return __half2float(v); }

// ---------------------------------------------------------------------------
// programmatic dependent launch (PDL) and TMA/mbarrier helpers
// ---------------------------------------------------------------------------
// Every kernel of the solve path waits for its predecessor grid here before it
// reads anything the predecessor wrote (a no-op when launched without PDL).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }


// ---------------------------------------------------------------------------
// SELL-32-sigma SpMV: row sums handed to an epilogue
// ---------------------------------------------------------------------------
// Epilogue concept:  __device__ void operator()(int row, AT sum, double (&acc)[NR]) const
// It writes its outputs for `row` and may add to the NR reduction values.
struct SpmvArgs {
    const int* off;     // nslices + 1
    const int* perm;    // nslices * 32
    const int* col;     // SELL column indices
    int nslots;         // nslices * 32
    int tpr_log2;       // log2 of the threads that share one row (0..3)
    const int16_t* col16;  // SELL 16-bit column offsets (IDX16 kernels) from the slot's row, or from
    const int* cbase;      // the slice's base column cbase[slice] when not null
    float vscale;          // FP16 values: factor of the row sums (2^-k of the value scaling)
};

// 2^tpr_log2 adjacent threads per slot (row) of a 32-row slice; thread `sub`
// of a row takes the row's entries sub, sub + TPR, ...  For a fixed k the
// threads of a warp read consecutive slots of one slice column, so every
// 32-byte sector they touch is used in full.  Partial sums are combined with
// shuffles in a fixed order.  TPR = 1 on large levels (occupancy hides the
// gather latency); TPR = 4..8 on small levels, where the row loop would
// otherwise be a chain of dependent gathers per thread.  No shared memory,
// no barriers.
// Prefetching variant of the row loop (k_spmv with PF): the slot's header
// and its first chunk of matrix entries are loaded before the wait for the
// preceding kernel (programmatic dependent launch), so on small levels that
// dependent chain of loads overlaps the predecessor's tail.  Only for
// matrices that no kernel of the stream writes after set-up (the levels of a
// multigrid hierarchy).  Same entry order and shuffle tree as k_spmv, so the
// same bits.
template <typename VT, typename XT, int NR, int TPR, class Epi, class Fin, bool IDX16>
__device__ __forceinline__ void spmv_prefetched(const SpmvArgs& m, const VT* __restrict__ val,
                                                const XT* __restrict__ x, const Epi& epi,
                                                const GridRed<NR, Fin>& red, const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    constexpr int tpr = TPR;
    constexpr int U = (IDX16 && TPR == 1) ? 8 : 4;
    constexpr int st = 32 * tpr;
    const int gid = blockIdx.x * kThreads + threadIdx.x;
    const int slot = gid / TPR;
    const int sub = gid % TPR;
    int o = 0, len = 0, r = -1, sb = 0;
    if (slot < m.nslots) {
        const int s = slot >> 5;
        const int a = __ldg(m.off + s);
        o = a + (slot & 31);
        len = (__ldg(m.off + s + 1) - a) >> 5;
        r = __ldg(m.perm + slot);
        if (IDX16 && m.cbase) sb = __ldg(m.cbase + s);
    }
    const int base = (IDX16 && m.cbase) ? sb : (r < 0 ? 0 : r);
    int c[U];
    AT v[U];
    auto load_chunk = [&](int k) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = k + u * tpr < len;
            const int idx = o + 32 * k + u * st;
            if constexpr (IDX16)
                c[u] = ok ? base + ld_stream(m.col16 + idx) : base;
            else
                c[u] = ok ? ld_stream(m.col + idx) : 0;
            v[u] = ok ? to_acc(ld_stream(val + idx)) : (AT)0;
        }
    };
    load_chunk(sub);
    pdl_wait();
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    AT sum = 0;
    for (int k = sub; k < len; k += U * tpr) {
        if (k != sub) load_chunk(k);
        AT xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) xv[u] = k + u * tpr < len ? (AT)__ldg(x + c[u]) : (AT)0;
#pragma unroll
        for (int u = 0; u < U; u++)
            if (k + u * tpr < len) sum += v[u] * xv[u];
    }
    for (int q = tpr >> 1; q > 0; q >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, q);
    if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
    if (sub == 0 && r >= 0) epi(r, sum, acc);
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

// PF: use spmv_prefetched (matrices fixed after set-up only).
template <typename VT, typename XT, int NR, int TPR, class Epi, class Fin, bool IDX16 = false, bool PF = false>
__global__ void __launch_bounds__(kThreads)
k_spmv(SpmvArgs m, const VT* __restrict__ val, const XT* __restrict__ x, Epi epi, GridRed<NR, Fin> red,
       const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    if constexpr (PF) {
        spmv_prefetched<VT, XT, NR, TPR, Epi, Fin, IDX16>(m, val, x, epi, red, done);
        return;
    }
    pdl_wait();
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    const int gid = blockIdx.x * kThreads + threadIdx.x;
    constexpr int tpr = TPR;
    const int slot = gid / TPR;
    const int sub = gid % TPR;
    AT sum = 0;
    int r = -1;
    if (slot < m.nslots) {
        const int s = slot >> 5, lane = slot & 31;
        const int o = __ldg(m.off + s);
        const int len = (__ldg(m.off + s + 1) - o) >> 5;
        r = __ldg(m.perm + slot);
        const VT* vp = val + o + lane;
        const int st = 32 * tpr;
        int k = sub;
        if constexpr (IDX16) {
            // columns stored as 16-bit offsets from the row: 2 bytes less per
            // entry.  Chunks of U entries: all column and value loads of a
            // chunk, then all its x gathers, then the sums in entry order
            // (entries past the slice length are predicated off), so a
            // thread has U entries of the matrix stream in flight.
            constexpr int U = TPR == 1 ? 8 : 4;
            const int base = m.cbase ? __ldg(m.cbase + s) : (r < 0 ? 0 : r);
            const int16_t* cp = m.col16 + o + lane;
            for (; k < len; k += U * tpr) {
                int c[U];
                AT v[U], xv[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const bool ok = k + u * tpr < len;
                    c[u] = ok ? base + ld_stream(cp + 32 * k + u * st) : base;
                    v[u] = ok ? to_acc(ld_stream(vp + 32 * k + u * st)) : (AT)0;
                }
#pragma unroll
                for (int u = 0; u < U; u++) xv[u] = k + u * tpr < len ? (AT)__ldg(x + c[u]) : (AT)0;
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (k + u * tpr < len) sum += v[u] * xv[u];
            }
        } else {
            const int* cp = m.col + o + lane;
            for (; k + 3 * tpr < len; k += 4 * tpr) {
                const int c0 = ld_stream(cp + 32 * k), c1 = ld_stream(cp + 32 * k + st);
                const int c2 = ld_stream(cp + 32 * k + 2 * st), c3 = ld_stream(cp + 32 * k + 3 * st);
                const AT v0 = to_acc(ld_stream(vp + 32 * k)), v1 = to_acc(ld_stream(vp + 32 * k + st));
                const AT v2 = to_acc(ld_stream(vp + 32 * k + 2 * st)), v3 = to_acc(ld_stream(vp + 32 * k + 3 * st));
                const AT x0 = (AT)__ldg(x + c0), x1 = (AT)__ldg(x + c1), x2 = (AT)__ldg(x + c2),
                         x3 = (AT)__ldg(x + c3);
                sum += v0 * x0;
                sum += v1 * x1;
                sum += v2 * x2;
                sum += v3 * x3;
            }
            for (; k < len; k += tpr) sum += to_acc(ld_stream(vp + 32 * k)) * (AT)__ldg(x + ld_stream(cp + 32 * k));
        }
    }
    for (int o = tpr >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
    if (sub == 0 && r >= 0) epi(r, sum, acc);
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

// ---------------------------------------------------------------------------
// SELL SpMV with the matrix stream staged through shared memory (large levels)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc)
{
    asm volatile("cp.async.cg.shared.global.L2::256B [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One thread per row, 16-bit columns.  A warp owns one 32-row slice, whose
// entries k..k+U-1 lie contiguously in the SELL arrays.  The warp keeps NS
// such chunks of values and columns in flight into its shared-memory stages
// with asynchronous 16-byte copies (no registers held while they are in
// flight) while its lanes gather x for the current chunk, so the matrix
// stream stays busy during the gather latency instead of alternating with
// it.  Sums in entry order: the same bits as k_spmv.
template <typename VT, typename XT, int NR, int U, int NS, class Epi, class Fin>
__global__ void __launch_bounds__(kThreads)
k_spmv_pipe(SpmvArgs m, const VT* __restrict__ val, const XT* __restrict__ x, Epi epi, GridRed<NR, Fin> red,
            const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    constexpr int W = kThreads / 32;
    constexpr int SV = U * 32;                 // entries of one stage
    static_assert((SV * sizeof(VT)) % 16 == 0 && (SV * 2) % 16 == 0, "stage not a multiple of 16 bytes");
    __shared__ __align__(16) VT s_val[W][NS][SV];
    __shared__ __align__(16) int16_t s_col[W][NS][SV];
    pdl_wait();
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    const int gid = blockIdx.x * kThreads + threadIdx.x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    AT sum = 0;
    int r = -1;
    if (gid < m.nslots) {                      // warp-uniform: nslots is a multiple of 32
        const int s = gid >> 5;
        const int o = __ldg(m.off + s);
        const int len = (__ldg(m.off + s + 1) - o) >> 5;
        r = __ldg(m.perm + gid);
        const int base = m.cbase ? __ldg(m.cbase + s) : (r < 0 ? 0 : r);
        const int nch = (len + U - 1) / U;
        // chunk j = entries [jU, jU + cnt) of the slice: [o + 32 jU, o + 32 (jU + cnt)); o is
        // a multiple of 32, so every copy starts on a 16-byte boundary
        auto issue = [&](int j) {
            const int k = j * U, stg = j % NS;
            const int cnt = min(U, len - k);
            const char* vs = reinterpret_cast<const char*>(val + o + 32 * k);
            char* vd = reinterpret_cast<char*>(&s_val[w][stg][0]);
            const int nv = cnt * 32 * (int)sizeof(VT) / 16;
            for (int i = lane; i < nv; i += 32) cp_async16(vd + 16 * i, vs + 16 * i);
            const char* cs = reinterpret_cast<const char*>(m.col16 + o + 32 * k);
            char* cd = reinterpret_cast<char*>(&s_col[w][stg][0]);
            const int nc = cnt * 64 / 16;
            for (int i = lane; i < nc; i += 32) cp_async16(cd + 16 * i, cs + 16 * i);
        };
#pragma unroll
        for (int j = 0; j < NS - 1; j++) {
            if (j < nch) issue(j);
            cp_async_commit();                 // one group per chunk slot (empty past the end)
        }
        for (int j = 0; j < nch; j++) {
            if (j + NS - 1 < nch) issue(j + NS - 1);
            cp_async_commit();
            cp_async_wait<NS - 1>();           // chunk j has landed
            __syncwarp();
            const int stg = j % NS, cnt = min(U, len - j * U);
            int c[U];
            AT v[U], xv[U];
            if (cnt == U) {                    // full chunk (warp-uniform): no per-entry predicates
#pragma unroll
                for (int u = 0; u < U; u++) {
                    c[u] = base + (int)s_col[w][stg][32 * u + lane];
                    v[u] = to_acc(s_val[w][stg][32 * u + lane]);
                }
#pragma unroll
                for (int u = 0; u < U; u++) xv[u] = (AT)__ldg(x + c[u]);
#pragma unroll
                for (int u = 0; u < U; u++) sum += v[u] * xv[u];
            } else {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const bool ok = u < cnt;
                    c[u] = ok ? base + (int)s_col[w][stg][32 * u + lane] : base;
                    v[u] = ok ? to_acc(s_val[w][stg][32 * u + lane]) : (AT)0;
                }
#pragma unroll
                for (int u = 0; u < U; u++) xv[u] = u < cnt ? (AT)__ldg(x + c[u]) : (AT)0;
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (u < cnt) sum += v[u] * xv[u];
            }
            __syncwarp();                      // the stage is refilled NS - 1 chunks later
        }
    }
    if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
    if (r >= 0) epi(r, sum, acc);
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

// ---------------------------------------------------------------------------
// values-only 9-point stencil SpMV (Matrix::st)
// ---------------------------------------------------------------------------
struct StArgs {
    int S, lo, nreg, ld, nirr, nb_reg;
    const int* irow;
    const int* iptr;
    const int* icol;
    float vscale;          // FP16 values: factor of the row sums
};

// Two consecutive values of one offset stream (the group's start is even and
// the stream stride a multiple of 8 entries: aligned vector loads), read
// once, not allocated in L1.
__device__ __forceinline__ void ldv2(const double* p, double (&o)[2])
{
    asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(o[0]), "=d"(o[1]) : "l"(p));
}
__device__ __forceinline__ void ldv2(const float* p, float (&o)[2])
{
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(o[0]), "=f"(o[1]) : "l"(p));
}
template <typename H>
__device__ __forceinline__ void ldv2_16(const H* p, float (&o)[2])
{
    unsigned a;
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(a) : "l"(p));
    const H* h = reinterpret_cast<const H*>(&a);
    o[0] = to_acc(h[0]);
    o[1] = to_acc(h[1]);
}
__device__ __forceinline__ void ldv2(const __half* p, float (&o)[2]) { ldv2_16(p, o); }
__device__ __forceinline__ void ldv2(const __nv_bfloat16* p, float (&o)[2]) { ldv2_16(p, o); }

// CTAs per SM of the regular part of k_spmv_st (a persistent grid-stride
// loop) for 4- and 2-byte values (64 registers at most); FP64 values take 2
constexpr int kStCtasPerSm = 4;

// Values-only stencil SpMV.  The regular rows are taken in pairs by a
// persistent grid of CTAs striding over the pairs: for a pair, nine aligned
// vector loads of its values (one per offset stream, no column indices) and
// three runs of four consecutive x entries (the grid lines below, at and
// above the rows; the two rows share them).  The values of a thread's next
// pair are loaded before the current pair is summed, so each thread keeps
// two pairs of the matrix stream in flight and no CTA waits on a second
// wave of launches.  The first CTAs of the grid take the irregular rows from
// their CSR copy, one row per thread.  Every row is summed in ascending
// column order from 0 with the same multiply-adds as k_spmv (a stored zero
// adds exactly 0 for finite x): the result equals the SELL kernels' bit for
// bit.  PF: the first pair's values are loaded before the wait for the
// preceding kernel (matrices that are not written after set-up).
template <typename VT, typename XT, int NR, class Epi, class Fin, bool PF = false>
__global__ void __launch_bounds__(kThreads, sizeof(VT) == 8 ? 2 : kStCtasPerSm)
k_spmv_st(StArgs m, const VT* __restrict__ val, const XT* __restrict__ x, Epi epi, GridRed<NR, Fin> red,
          const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    // the irregular rows' CTAs come first: they start in the first wave
    // instead of trailing the persistent regular CTAs
    const int nb_irr = (m.nirr + kThreads - 1) / kThreads;
    const bool regular = (int)blockIdx.x >= nb_irr;
    const int npairs = (m.nreg + 1) >> 1;
    const int stride = m.nb_reg * kThreads;
    int g = (regular ? (int)blockIdx.x - nb_irr : (int)blockIdx.x) * kThreads + threadIdx.x;
    auto full = [&](int gg) { return 2 * gg + 2 <= m.nreg; };
    AT v[9][2];
    bool have = false;
    if (PF && regular && g < npairs && full(g)) {
#pragma unroll
        for (int k = 0; k < 9; k++) ldv2(val + (int64_t)k * m.ld + 2 * g, v[k]);
        have = true;
    }
    pdl_wait();
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int q = 0; q < (NR > 0 ? NR : 1); q++) acc[q] = 0;
    if (regular) {
        for (; g < npairs; g += stride) {
            const int i0 = 2 * g;
            if (full(g)) {
                if (!have) {
#pragma unroll
                    for (int k = 0; k < 9; k++) ldv2(val + (int64_t)k * m.ld + i0, v[k]);
                }
                const int gn = g + stride;      // prefetch the next pair's values
                AT vn[9][2];
                const bool haven = gn < npairs && full(gn);
                if (haven) {
#pragma unroll
                    for (int k = 0; k < 9; k++) ldv2(val + (int64_t)k * m.ld + 2 * gn, vn[k]);
                }
                const int r0 = m.lo + i0;
                AT xs[3][4];
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    const XT* xp = x + (r0 + (j - 1) * m.S - 1);
#pragma unroll
                    for (int e = 0; e < 4; e++) xs[j][e] = (AT)__ldg(xp + e);
                }
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    AT sum = 0;
#pragma unroll
                    for (int k = 0; k < 9; k++) sum += v[k][q] * xs[k / 3][q + k % 3];
                    if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
                    epi(r0 + q, sum, acc);
                }
                if (haven) {
#pragma unroll
                    for (int k = 0; k < 9; k++) {
                        v[k][0] = vn[k][0];
                        v[k][1] = vn[k][1];
                    }
                }
                have = haven;
            } else {                            // the last row of an odd count
                const int i = i0, r = m.lo + i;
                AT sum = 0;
#pragma unroll
                for (int k = 0; k < 9; k++) {
                    const int d = (k / 3 - 1) * m.S + (k % 3 - 1);
                    sum += to_acc(val[(int64_t)k * m.ld + i]) * (AT)__ldg(x + r + d);
                }
                if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
                epi(r, sum, acc);
                have = false;
            }
        }
    } else if (g < m.nirr) {
        const int r = m.irow[g];
        const VT* iv = val + 9 * (int64_t)m.ld;
        AT sum = 0;
        for (int k = m.iptr[g]; k < m.iptr[g + 1]; k++) sum += to_acc(iv[k]) * (AT)__ldg(x + m.icol[k]);
        if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
        epi(r, sum, acc);
    }
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

// ---------------------------------------------------------------------------
// staged point-layout SpMV (Matrix::st, all kinds): the value streams of a
// tile of rows go to shared memory by bulk copies, the x gathers stay loads
// ---------------------------------------------------------------------------
struct PtArgs {
    int S, S2, lo, nreg, ld, nirr, ntiles;
    const int* irow;
    const int* iptr;
    const int* icol;
    float vscale;          // FP16 values: factor of the row sums
    int* err;              // set to 1 when a bulk copy does not complete
};

constexpr int kPtRows = 2 * kThreads;      // rows of one tile (two per thread)
// stages of the value ring: 2-byte values three, FP32 / FP64 values two
template <typename VT>
__host__ __device__ constexpr int pt_stages() { return sizeof(VT) == 2 ? 3 : 2; }
template <typename VT>
constexpr int pt_smem(int K) { return pt_stages<VT>() * K * kPtRows * (int)sizeof(VT); }

__device__ __forceinline__ uint32_t sh_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait on an mbarrier phase (about half a second at most).
__device__ __forceinline__ bool bulk_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (i > 16) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void bulk_arm(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// untiled bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// two consecutive values of one stream from shared memory
__device__ __forceinline__ void sm_ld2(const double* p, double (&o)[2])
{
    const double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x;
    o[1] = v.y;
}
__device__ __forceinline__ void sm_ld2(const float* p, float (&o)[2])
{
    const float2 v = *reinterpret_cast<const float2*>(p);
    o[0] = v.x;
    o[1] = v.y;
}
template <typename H>
__device__ __forceinline__ void sm_ld2(const H* p, float (&o)[2])
{
    o[0] = to_acc(p[0]);
    o[1] = to_acc(p[1]);
}

// The x entries that regular rows i and i + 1 of a point layout read (i
// even; row i + 1 only when it is regular), in slot order: the 9-point kind
// as three runs of four entries (grid lines below, at and above the rows,
// shared by the two rows), the transfer kinds K entries per row.
template <int KIND, typename AT, typename XT, int KX>
__device__ __forceinline__ void pt_gather(const PtArgs& m, const XT* __restrict__ x, int i, AT (&xv)[KX])
{
    if (i >= m.nreg) return;
    const bool two = i + 1 < m.nreg;
    const int r0 = m.lo + i;
    if constexpr (KIND == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const XT* xp = x + (r0 + (a - 1) * m.S - 1);
#pragma unroll
            for (int e = 0; e < 3; e++) xv[4 * a + e] = (AT)__ldg(xp + e);
            xv[4 * a + 3] = two ? (AT)__ldg(xp + 3) : (AT)0;
        }
    } else {
        constexpr int K = KX / 2;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            if (q == 1 && !two) {
#pragma unroll
                for (int k = 0; k < K; k++) xv[K + k] = (AT)0;
                break;
            }
            const int r = r0 + q;
            const int g = r / m.S, h = r - g * m.S;
            if constexpr (KIND == 1) {
                const XT* xp = x + ((g >> 1) * m.S2 + (h >> 1));
                xv[q * K + 0] = (AT)__ldg(xp);
                xv[q * K + 1] = (AT)__ldg(xp + 1);
                xv[q * K + 2] = (AT)__ldg(xp + m.S2);
                xv[q * K + 3] = (AT)__ldg(xp + m.S2 + 1);
            } else {
                const XT* xp = x + (2 * g * m.S2 + 2 * h);
#pragma unroll
                for (int k = 0; k < 9; k++) xv[q * K + k] = (AT)__ldg(xp + ((k / 3 - 1) * m.S2 + (k % 3 - 1)));
            }
        }
    }
}

// Staged point-layout SpMV.  A tile is kPtRows consecutive regular rows; its
// K value streams (one per offset, kPtRows contiguous entries each) arrive in
// shared memory by K bulk copies completing one mbarrier.  Thread 0 of a
// persistent CTA issues the copies ST - 1 tiles ahead of the tile the CTA
// sums, so the matrix stream is in flight without holding registers.  Each
// thread sums two consecutive rows: the 9-point kind shares its three runs of
// four x entries between the two rows, the transfer kinds gather per row.
// Rows are summed in ascending column order from 0 with the same multiply-adds
// as the SELL kernels (a stored zero adds exactly 0 for finite x): the result
// equals theirs bit for bit.  The first CTAs of the grid take the irregular
// rows from their CSR copy, one row per thread.  PF: the first tiles' copies
// are issued before the wait for the preceding kernel (matrices that are not
// written after set-up).  A tile whose copies do not complete within the
// bounded wait sets *err; the CTA then waits (bounded) for the copies it has
// issued and leaves.
template <typename VT, typename XT, int NR, class Epi, class Fin, bool PF, int KIND>
__global__ void __launch_bounds__(kThreads, sizeof(VT) == 8 ? 2 : kStCtasPerSm)
k_spmv_pt(PtArgs m, const VT* __restrict__ val, const XT* __restrict__ x, Epi epi, GridRed<NR, Fin> red,
          const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    constexpr int K = KIND == 1 ? 4 : 9;
    constexpr int ST = pt_stages<VT>();
    constexpr int SE = K * kPtRows;                 // entries of one stage
    extern __shared__ __align__(128) unsigned char pt_raw[];
    VT* vs = reinterpret_cast<VT*>(pt_raw);
    __shared__ __align__(8) uint64_t full[ST];
    const int nb_irr = (m.nirr + kThreads - 1) / kThreads;
    const bool regular = (int)blockIdx.x >= nb_irr;
    const int G = (int)gridDim.x - nb_irr;
    const int b = (int)blockIdx.x - nb_irr;
    const int cnt = regular && b < m.ntiles ? (m.ntiles - 1 - b) / G + 1 : 0;
    int issued = 0;                                 // tiles whose copies thread 0 has issued
    auto issue = [&](int j) {
        constexpr int E = 16 / (int)sizeof(VT);     // copy sizes: multiples of 16 bytes (within ld)
        const int i0 = (b + j * G) * kPtRows;
        const int rows = min(kPtRows, m.nreg - i0);
        const uint32_t bytes = (uint32_t)((rows + E - 1) / E * E * (int)sizeof(VT));
        const int s = j % ST;
        const uint32_t bar = sh_addr(&full[s]);
        bulk_arm(bar, (uint32_t)K * bytes);
#pragma unroll
        for (int k = 0; k < K; k++)
            bulk_copy(sh_addr(vs + s * SE + k * kPtRows), val + (int64_t)k * m.ld + i0, bytes, bar);
    };
    if (cnt > 0) {
        if (threadIdx.x == 0) {
            for (int s = 0; s < ST; s++)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sh_addr(&full[s])) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (PF)
                for (; issued < min(ST, cnt); issued++) issue(issued);
        }
        __syncthreads();
    }
    pdl_wait();
    if (done && *done) {
        if (threadIdx.x == 0)
            for (int j = 0; j < issued; j++) bulk_wait(sh_addr(&full[j]), 0);
        return;
    }
    if (cnt > 0 && threadIdx.x == 0)
        for (; issued < min(ST, cnt); issued++) issue(issued);
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int q = 0; q < (NR > 0 ? NR : 1); q++) acc[q] = 0;
    if (regular) {
        const int l = 2 * (int)threadIdx.x;
        constexpr int KX = KIND == 0 ? 12 : 2 * K;
        AT xv[KX];
        // the x entries of a tile are gathered one tile ahead (their latency
        // overlaps the sums of the tile before)
        if (cnt > 0) pt_gather<KIND>(m, x, b * kPtRows + l, xv);
        for (int j = 0; j < cnt; j++) {
            const int s = j % ST;
            const bool ok = bulk_wait(sh_addr(&full[s]), (uint32_t)((j / ST) & 1));
            // one vote: every thread leaves together, and every thread is past tile j - 1
            if (!__syncthreads_and(ok)) {
                if (threadIdx.x == 0) {
                    atomicOr(m.err, 1);
                    for (int q = j; q < issued; q++) bulk_wait(sh_addr(&full[q % ST]), (uint32_t)((q / ST) & 1));
                }
                return;
            }
            // tile j - 1 + ST into the stage tile j - 1 has left
            if (threadIdx.x == 0 && j >= 1 && issued < cnt) {
                issue(issued);
                issued++;
            }
            const int i = (b + j * G) * kPtRows + l;
            AT xn[KX];
            const bool more = j + 1 < cnt;
            if (more) pt_gather<KIND>(m, x, i + G * kPtRows, xn);
            if (i < m.nreg) {
                const VT* vt = vs + s * SE + l;
                AT v[K][2];
#pragma unroll
                for (int k = 0; k < K; k++) sm_ld2(vt + k * kPtRows, v[k]);
                const bool two = i + 1 < m.nreg;
                const int r0 = m.lo + i;
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    if (q == 1 && !two) break;
                    AT sum = 0;
                    if constexpr (KIND == 0) {
#pragma unroll
                        for (int k = 0; k < 9; k++) sum += v[k][q] * xv[(k / 3) * 4 + q + k % 3];
                    } else {
#pragma unroll
                        for (int k = 0; k < K; k++) sum += v[k][q] * xv[q * K + k];
                    }
                    if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
                    epi(r0 + q, sum, acc);
                }
            }
            if (more) {
#pragma unroll
                for (int e = 0; e < KX; e++) xv[e] = xn[e];
            }
        }
    } else {
        const int g = (int)blockIdx.x * kThreads + (int)threadIdx.x;
        if (g < m.nirr) {
            const int r = m.irow[g];
            const VT* iv = val + (int64_t)K * m.ld;
            AT sum = 0;
            for (int k = m.iptr[g]; k < m.iptr[g + 1]; k++) sum += to_acc(iv[k]) * (AT)__ldg(x + m.icol[k]);
            if constexpr (std::is_same<VT, __half>::value) sum *= m.vscale;
            epi(r, sum, acc);
        }
    }
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

// ---------------------------------------------------------------------------
// grid-stride vector kernels: f(i, acc) per index, optional reduction
// ---------------------------------------------------------------------------
template <int NR, class F, class Fin>
__global__ void __launch_bounds__(kThreads)
k_vec(int n, F f, GridRed<NR, Fin> red, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) f(i, acc);
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

// Single-thread scalar step (device-side control logic between kernels).
template <class F>
__global__ void k_scalar(F f, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    f();
}

}  // namespace jfg
