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
template <typename VT> struct AccOf { using T = VT; };
template <> struct AccOf<__nv_bfloat16> { using T = float; };

__device__ __forceinline__ float to_acc(float v) { return v; }
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ float to_acc(__nv_bfloat16 v) { return __bfloat162float(v); }

// ---------------------------------------------------------------------------
// programmatic dependent launch (PDL) and TMA/mbarrier helpers
// ---------------------------------------------------------------------------
// Every kernel of the solve path waits for its predecessor grid here before it
// reads anything the predecessor wrote (a no-op when launched without PDL).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~2^32 SM cycles (about 2 s) and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1LL << 32)) return false;
    }
    return true;
}
// 1-D bulk copy global -> shared completing on an mbarrier (both addresses
// 16-byte aligned, size a multiple of 16; no multicast).
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Device-side error word (set when a bounded wait gives up); read by the host.
__device__ int g_device_error;

// ---------------------------------------------------------------------------
// row-block CSR SpMV: y-row sums handed to an epilogue
// ---------------------------------------------------------------------------
// Epilogue concept:  __device__ void operator()(int row, AT sum, double (&acc)[NR]) const
// It writes its outputs for `row` and may add to the NR reduction values.
struct SpmvArgs {
    const int* rb;
    const int* rowptr;
    const int* col;
    int nblocks;
};

// Shared-memory layout of the pipelined SpMV: S stages of (columns, values),
// then the product buffer, then S mbarriers.
constexpr int kStageCap = kBlockNnz + 8;
template <typename VT>
__host__ __device__ constexpr int stage_bytes() { return kStageCap * (4 + (int)sizeof(VT)); }
template <typename VT, int S>
__host__ __device__ constexpr int spmv_smem_bytes()
{
    return S * stage_bytes<VT>() + kStageCap * (int)sizeof(typename AccOf<VT>::T) + S * 8 + 16;
}

// Persistent, TMA-pipelined SpMV.  CTA c handles row blocks c, c+G, c+2G, ...
// Thread 0 keeps S blocks in flight: one bulk copy each for the block's
// column indices and values into a shared-memory stage, completing on the
// stage's mbarrier.  For the current block all threads gather x[col] and form
// the products (8 independent gathers per thread), the stage is handed back
// to the producer, and groups of 2^lpr_log2 lanes reduce rows from the
// product buffer and call the epilogue.  Blocks longer than the stage (one
// long row) are read directly from global memory.
template <typename VT, typename XT, int NR, int S, class Epi, class Fin>
__global__ void __launch_bounds__(kThreads)
k_spmv(SpmvArgs m, const VT* __restrict__ val, const XT* __restrict__ x, int lpr_log2, Epi epi,
       GridRed<NR, Fin> red, const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    pdl_wait();
    if (done && *done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    AT* prod = reinterpret_cast<AT*>(smem + S * stage_bytes<VT>());
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S * stage_bytes<VT>() + kStageCap * sizeof(AT));
    __shared__ int ok_sh;
    const int tid = threadIdx.x;
    const int first = blockIdx.x, G = gridDim.x;
    const int nmine = first < m.nblocks ? (m.nblocks - 1 - first) / G + 1 : 0;
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto stage_col = [&](int s) { return reinterpret_cast<int*>(smem + s * stage_bytes<VT>()); };
    auto stage_val = [&](int s) { return reinterpret_cast<VT*>(smem + s * stage_bytes<VT>() + kStageCap * 4); };
    auto issue = [&](int it) {   // thread 0 only
        const int b = first + it * G;
        const int s = it % S;
        const int k0 = m.rowptr[m.rb[b]], k1 = m.rowptr[m.rb[b + 1]];
        const int nk = k1 - k0;
        if (nk > 0 && nk <= kBlockNnz) {
            const int nkp = (nk + 7) & ~7;
            const uint32_t bc = nkp * 4u, bv = nkp * (uint32_t)sizeof(VT);
            mbar_arrive_expect_tx(&bars[s], bc + bv);
            tma_load_1d(stage_col(s), m.col + k0, bc, &bars[s]);
            tma_load_1d(stage_val(s), val + k0, bv, &bars[s]);
        } else {
            mbar_arrive(&bars[s]);
        }
    };
    if (tid == 0)
        for (int it = 0; it < S && it < nmine; it++) issue(it);
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    const int lpr = 1 << lpr_log2;
    const int g = tid >> lpr_log2;
    const int lane = tid & (lpr - 1);
    const int ngroups = kThreads >> lpr_log2;
    int it = 0;
    for (; it < nmine; it++) {
        const int b = first + it * G;
        const int s = it % S;
        const int r0 = m.rb[b], r1 = m.rb[b + 1];
        const int k0 = m.rowptr[r0], k1 = m.rowptr[r1];
        const int nk = k1 - k0;
        if (tid == 0) ok_sh = mbar_wait_bounded(&bars[s], (it / S) & 1) ? 1 : 0;
        __syncthreads();
        if (!ok_sh) {
            if (tid == 0) atomicExch(&g_device_error, 1);
            break;
        }
        if (nk <= kBlockNnz) {
            const int* sc = stage_col(s);
            const VT* sv = stage_val(s);
#pragma unroll
            for (int j = 0; j < kBlockNnz / kThreads; j++) {
                const int k = tid + j * kThreads;
                if (k < nk) prod[k] = to_acc(sv[k]) * (AT)__ldg(x + sc[k]);
            }
            __syncthreads();
            if (tid == 0 && it + S < nmine) issue(it + S);
            for (int base = r0; base < r1; base += ngroups) {
                const int r = base + g;
                AT sum = 0;
                if (r < r1) {
                    const int a = m.rowptr[r] - k0, e = m.rowptr[r + 1] - k0;
                    for (int k = a + lane; k < e; k += lpr) sum += prod[k];
                }
                for (int o = lpr >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
                if (r < r1 && lane == 0) epi(r, sum, acc);
            }
            __syncthreads();
        } else {
            double part[1] = {0};
            for (int k = k0 + tid; k < k1; k += kThreads)
                part[0] += (double)(to_acc(val[k]) * (AT)__ldg(x + m.col[k]));
            block_sum<1>(part);
            if (tid == 0) epi(r0, (AT)part[0], acc);
            if (tid == 0 && it + S < nmine) issue(it + S);
            __syncthreads();
        }
    }
    if (it < nmine && tid == 0) {
        // a wait gave up: let the copies already issued land (bounded) before exit
        for (int j = it + 1; j < nmine && j < it + S; j++) mbar_wait_bounded(&bars[j % S], (j / S) & 1);
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
