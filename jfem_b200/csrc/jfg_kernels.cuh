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
// row-block CSR SpMV: y-row sums handed to an epilogue
// ---------------------------------------------------------------------------
// Epilogue concept:  __device__ void operator()(int row, AT sum, double (&acc)[NR]) const
// It writes its outputs for `row` and may add to the NR reduction values.
struct SpmvArgs {
    const int* rb;
    const int* rowptr;
    const int* col;
};

template <typename VT, typename XT, int NR, class Epi, class Fin>
__global__ void __launch_bounds__(kThreads)
k_spmv(SpmvArgs m, const VT* __restrict__ val, const XT* __restrict__ x, int lpr_log2, Epi epi,
       GridRed<NR, Fin> red, const int* __restrict__ done)
{
    using AT = typename AccOf<VT>::T;
    if (done && *done) return;
    __shared__ __align__(16) AT prod[kBlockNnz + 4];
    const int b = blockIdx.x;
    const int r0 = m.rb[b], r1 = m.rb[b + 1];
    const int k0 = m.rowptr[r0], k1 = m.rowptr[r1];
    const int nk = k1 - k0;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    if (nk <= kBlockNnz) {
        const int nvec = (nk + 3) >> 2;
        const int4* c4p = reinterpret_cast<const int4*>(m.col + k0);
        for (int u = threadIdx.x; u < nvec; u += kThreads) {
            int4 c4 = __ldg(c4p + u);
            AT v[4];
            load4(val + k0 + 4 * u, v);
            prod[4 * u + 0] = v[0] * (AT)__ldg(x + c4.x);
            prod[4 * u + 1] = v[1] * (AT)__ldg(x + c4.y);
            prod[4 * u + 2] = v[2] * (AT)__ldg(x + c4.z);
            prod[4 * u + 3] = v[3] * (AT)__ldg(x + c4.w);
        }
        __syncthreads();
        const int lpr = 1 << lpr_log2;
        const int g = threadIdx.x >> lpr_log2;
        const int lane = threadIdx.x & (lpr - 1);
        const int ngroups = kThreads >> lpr_log2;
        for (int base = r0; base < r1; base += ngroups) {
            const int r = base + g;
            AT s = 0;
            if (r < r1) {
                const int a = m.rowptr[r] - k0, e = m.rowptr[r + 1] - k0;
                for (int k = a + lane; k < e; k += lpr) s += prod[k];
            }
            for (int o = lpr >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (r < r1 && lane == 0) epi(r, s, acc);
        }
    } else {
        // a single row longer than the staging buffer: strided sum + CTA reduction
        double part[1] = {0};
        for (int k = k0 + threadIdx.x; k < k1; k += kThreads)
            part[0] += (double)(to_acc(val[k]) * (AT)__ldg(x + m.col[k]));
        block_sum<1>(part);
        if (threadIdx.x == 0) epi(r0, (AT)part[0], acc);
    }
    if constexpr (NR > 0) red.reduce(acc);
}

// ---------------------------------------------------------------------------
// grid-stride vector kernels: f(i, acc) per index, optional reduction
// ---------------------------------------------------------------------------
template <int NR, class F, class Fin>
__global__ void __launch_bounds__(kThreads)
k_vec(int n, F f, GridRed<NR, Fin> red, const int* __restrict__ done)
{
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) f(i, acc);
    if constexpr (NR > 0) red.reduce(acc);
}

// Single-thread scalar step (device-side control logic between kernels).
template <class F>
__global__ void k_scalar(F f, const int* __restrict__ done)
{
    if (done && *done) return;
    f();
}

}  // namespace jfg
