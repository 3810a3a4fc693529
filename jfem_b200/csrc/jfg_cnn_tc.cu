// 32 -> 32 3x3 convolutions of the learned smoother on the fifth-generation
// tensor cores (tcgen05.mma, accumulators in TMEM), fed by TMA: the forward
// layers and, with flipped channel-transposed weights and FP32 epilogues, the
// input gradients of the backward pass.
//
// Implicit GEMM per tile of 16 x 8 = 128 output pixels (the MMA's M):
//   D[p][co] = sum_{tap, ci} X[p + tap][ci] * W[co][tap * 32 + ci]
// with K = 9 taps x 32 channels = 288 = 18 MMAs of K = 16, N = 32.
//
// Shared-memory layout (canonical K-major, no swizzle: core matrices of 8
// rows x 16 bytes):
//  - the input halo (18 x 10 pixels) arrives by four TMA box loads of 8
//    channels each (box 8 x 10 x 18, zero fill outside the image), plane q of
//    a stage at q * 2944, pixel (hy, hx) at (hy * 10 + hx) * 16 inside it.
//    Because a tile is 8 pixels wide, the 8 rows of every core matrix of the A
//    operand of any tap are 8 consecutive halo pixels of one halo row, the
//    next core matrix (next tile row) is 160 bytes further and the next 8
//    channels one plane further: every tap's A operand is a descriptor view of
//    the halo (start, LBO = plane, SBO = halo row), nothing is copied;
//  - the weights W[co][k] at (co / 8) * 4608 + (k / 8) * 128 + (co % 8) * 16
//    + (k % 8) * 2 (LBO = 128, SBO = 4608).
// Two stages, software-pipelined: the TMA loads of a CTA's tiles run two
// tiles ahead and the MMAs of tile i + 1 run while tile i's epilogue reads
// its own TMEM accumulator (2 x 32 columns).  One thread issues the TMA loads
// and the 18 MMAs (committed to an mbarrier); after the bounded wait each warp reads its
// 32 TMEM lanes (one pixel per thread, 32 FP32 channels), adds the skip
// input, applies ReLU and stores BF16.  Persistent CTAs of 128 threads stride
// over the tiles (~42 KB of shared memory and 64 TMEM columns each).
#include <cudaTypedefs.h>

#include "jfg_ops.cuh"

namespace jfg {
namespace {

typedef __nv_bfloat16 bf16;

constexpr int kTH = 16, kTW = 8;                 // tile rows x columns (128 pixels)
constexpr int kHH = kTH + 2, kHW = kTW + 2;      // halo 18 x 10
constexpr int kPlaneData = kHH * kHW * 16;       // bytes one TMA box writes (2880)
constexpr int kPlane = 2944;                     // plane stride: 2880 rounded up to 128
constexpr int kHaloBytes = 4 * kPlane;           // 11,776 per stage
constexpr int kStages = 2;
constexpr int kWRowGroup = 36 * 128;             // bytes per 8 output channels (4608)
constexpr int kWBytes = 4 * kWRowGroup;          // 18,432
constexpr int kTcThreads = 128;
constexpr int kTcCtasPerSm = 5;
// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, N = 32, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;      // descriptor version of sm_100; base offset 0, no swizzle
    return d;
}

// Bounded wait on an mbarrier phase (about a second at most).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (i > 32) __nanosleep(128);
    }
    return false;
}

__device__ __forceinline__ void tma_plane(uint32_t dst, const CUtensorMap* map, int c, int x, int y, int b,
                                          uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c), "r"(x), "r"(y), "r"(b)
        : "memory");
}

// Epilogue modes (acc = the convolution, FP32 from TMEM; one pixel per thread):
//   kFwd:     out(bf16) = relu(acc)                          forward, no skip
//   kFwdSkip: out(bf16) = relu(acc + skip(bf16))             forward with the residual input
//   kBwdMask: out(f32) = acc * (mask(bf16) > 0), out16 = the same in BF16
//             (an input gradient through the next layer's ReLU, and its BF16
//             copy: the TMA input of the following input-gradient convolution)
//   kBwdSkip: out(f32) = acc + skip(f32)                     input gradient plus the skip path's
constexpr int kFwd = 0, kFwdSkip = 1, kBwdMask = 2, kBwdSkip = 3;
//   kFwdProj: the last 32 -> 32 layer (with skip) fused with the projection of
//   the 32 -> 1 output layer: h = relu(acc + skip) rounded to BF16 (the values
//   the output layer would read back), then u[t][p] = sum_c w6[c][t] h[c] for
//   the nine taps t, written as nine FP32 planes; y = sum_t u[t][p + off_t]
//   follows in a small kernel.  Warp-specialised kernel only.
constexpr int kFwdProj = 4;

// The epilogue of one output pixel: its 32 FP32 channel sums r (from TMEM)
// combined and stored as MODE says; base = the pixel's first channel.
template <int MODE>
__device__ __forceinline__ void conv_store(const uint32_t (&r)[32], size_t base, const void* __restrict__ aux,
                                           void* __restrict__ out, bf16* __restrict__ out16)
{
    if constexpr (MODE == kFwd || MODE == kFwdSkip) {
        __align__(16) bf16 o[32];
        __align__(16) bf16 sv[32];
        if (MODE == kFwdSkip) {
            const bf16* skip = static_cast<const bf16*>(aux);
#pragma unroll
            for (int q = 0; q < 4; q++)
                *reinterpret_cast<uint4*>(sv + 8 * q) =
                    __ldg(reinterpret_cast<const uint4*>(skip + base + 8 * q));
        }
#pragma unroll
        for (int c = 0; c < 32; c++) {
            float v = __uint_as_float(r[c]);
            if (MODE == kFwdSkip) v += __bfloat162float(sv[c]);
            o[c] = __float2bfloat16_rn(fmaxf(v, 0.f));
        }
        bf16* ob = static_cast<bf16*>(out);
#pragma unroll
        for (int q = 0; q < 4; q++)
            *reinterpret_cast<uint4*>(ob + base + 8 * q) = *reinterpret_cast<const uint4*>(o + 8 * q);
    } else if constexpr (MODE == kBwdMask) {
        const bf16* mask = static_cast<const bf16*>(aux);
        __align__(16) bf16 mv[32];
#pragma unroll
        for (int q = 0; q < 4; q++)
            *reinterpret_cast<uint4*>(mv + 8 * q) = __ldg(reinterpret_cast<const uint4*>(mask + base + 8 * q));
        __align__(16) float f[32];
        __align__(16) bf16 o[32];
#pragma unroll
        for (int c = 0; c < 32; c++) {
            const float v = __bfloat162float(mv[c]) > 0.f ? __uint_as_float(r[c]) : 0.f;
            f[c] = v;
            o[c] = __float2bfloat16_rn(v);
        }
        float* of = static_cast<float*>(out);
#pragma unroll
        for (int q = 0; q < 8; q++)
            *reinterpret_cast<float4*>(of + base + 4 * q) = *reinterpret_cast<const float4*>(f + 4 * q);
#pragma unroll
        for (int q = 0; q < 4; q++)
            *reinterpret_cast<uint4*>(out16 + base + 8 * q) = *reinterpret_cast<const uint4*>(o + 8 * q);
    } else {
        const float* skip = static_cast<const float*>(aux);
        float* of = static_cast<float*>(out);
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const float4 sk = __ldg(reinterpret_cast<const float4*>(skip + base + 4 * q));
            float4 v;
            v.x = __uint_as_float(r[4 * q]) + sk.x;
            v.y = __uint_as_float(r[4 * q + 1]) + sk.y;
            v.z = __uint_as_float(r[4 * q + 2]) + sk.z;
            v.w = __uint_as_float(r[4 * q + 3]) + sk.w;
            *reinterpret_cast<float4*>(of + base + 4 * q) = v;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(kTcThreads)
k_conv_mid_tc(const __grid_constant__ CUtensorMap tin, int B, int H, int W, const bf16* __restrict__ wk,
              const void* __restrict__ aux, void* __restrict__ out, bf16* __restrict__ out16, int* __restrict__ err)
{
    __shared__ __align__(128) unsigned char wsm[kWBytes];
    __shared__ __align__(128) unsigned char halo[kStages][kHaloBytes];
    __shared__ __align__(8) uint64_t full[kStages], mdone[kStages];
    __shared__ uint32_t tmem_sh;
    __shared__ int s_stop;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 32 * 36; i += kTcThreads) {
        const int co = i / 36, j = i % 36;
        const uint4 v = *reinterpret_cast<const uint4*>(wk + co * 288 + j * 8);
        *reinterpret_cast<uint4*>(wsm + (co >> 3) * kWRowGroup + j * 128 + (co & 7) * 16) = v;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(&tmem_sh))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        s_stop = 0;
        for (int s = 0; s < kStages; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mdone[s])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the weights written by threads are read by the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    const uint32_t wbase = smem_u32(wsm);
    const int tilesx = (W + kTW - 1) / kTW, tilesy = (H + kTH - 1) / kTH;
    const int per_img = tilesx * tilesy;
    const int ntiles = per_img * B;

    auto issue_load = [&](int t, int s) {       // thread 0 only
        const int b = t / per_img, rem = t - b * per_img;
        const int y0 = (rem / tilesx) * kTH, x0 = (rem % tilesx) * kTW;
        const uint32_t bar = smem_u32(&full[s]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(4 * kPlaneData)
                     : "memory");
        const uint32_t dst = smem_u32(halo[s]);
#pragma unroll
        for (int q = 0; q < 4; q++) tma_plane(dst + q * kPlane, &tin, 8 * q, x0 - 1, y0 - 1, b, bar);
    };

    // tiles of this CTA: t_i = blockIdx.x + i * gridDim.x, i < cnt
    const int cnt = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile_of = [&](int i) { return (int)blockIdx.x + i * (int)gridDim.x; };
    auto issue_mma = [&](int i) -> bool {     // thread 0: wait for tile i's halo, MMAs into TMEM stage i & 1
        const int s = i & 1;
        if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((i >> 1) & 1))) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t hb = smem_u32(halo[s]);
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            const int dy = tap / 3, dx = tap % 3;
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const uint64_t da = umma_desc(hb + 2 * k * kPlane + (dy * kHW + dx) * 16, kPlane, kHW * 16);
                const uint64_t db = umma_desc(wbase + (4 * tap + 2 * k) * 128, 128, kWRowGroup);
                const uint32_t accum = (tap | k) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem + (uint32_t)(s * 32)), "l"(da), "l"(db), "r"(kIdesc), "r"(accum)
                    : "memory");
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mdone[s]))
                     : "memory");
        return true;
    };

    // Pipeline: loads run two tiles ahead, the MMAs of tile i + 1 run during
    // the epilogue of tile i.  Outstanding async work is tracked by thread 0
    // for the error path.
    int loads_issued = 0, loads_done = 0, mmas_issued = 0;
    if (tid == 0) {
        for (int i = 0; i < 2 && i < cnt; i++) {
            issue_load(tile_of(i), i);
            loads_issued++;
        }
        if (cnt > 0) {
            if (issue_mma(0)) {
                loads_done = 1;
                mmas_issued = 1;
            } else {
                s_stop = 1;
            }
        }
    }
    __syncthreads();
    int i = 0;
    for (; i < cnt && !s_stop; i++) {
        const int s = i & 1;
        const bool ok = mbar_wait(smem_u32(&mdone[s]), (uint32_t)((i >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) s_stop = 1;
            break;
        }
        if (tid == 0) {
            if (i + 2 < cnt) {                   // its buffer held tile i, whose MMAs are complete
                issue_load(tile_of(i + 2), s);
                loads_issued++;
            }
            if (i + 1 < cnt) {
                if (issue_mma(i + 1)) {
                    loads_done++;
                    mmas_issued++;
                } else {
                    s_stop = 1;
                }
            }
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t r[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(s * 32))
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int t = tile_of(i);
        const int b = t / per_img, rem = t - b * per_img;
        const int y0 = (rem / tilesx) * kTH, x0 = (rem % tilesx) * kTW;
        const int m = warp * 32 + lane;
        const int gy = y0 + (m >> 3), gx = x0 + (m & 7);
        if (gy < H && gx < W) {
            const size_t base = (((size_t)b * H + gy) * W + gx) * 32;
            conv_store<MODE>(r, base, aux, out, out16);
        }
        // every thread's TMEM reads are done before the MMAs two tiles on overwrite this stage
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (s_stop && tid == 0) {
        // error path: report, then let the copies and MMAs still in flight finish (bounded) before TMEM is freed
        atomicOr(err, 1);
        for (int k = loads_done; k < loads_issued; k++) mbar_wait(smem_u32(&full[k & 1]), (uint32_t)((k >> 1) & 1));
        for (int k = i; k < mmas_issued; k++) mbar_wait(smem_u32(&mdone[k & 1]), (uint32_t)((k >> 1) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Warp-specialised pipeline (the default).  Per CTA of 256 threads:
//   warp 0 (one lane): TMA producer -- tile i's whole halo (18 x 10 pixels x
//     32 channels) as ONE box with a 64-byte inner extent into staging buffer
//     i % ST, once the transposers released it (mbarrier `sempty`); one
//     64-byte row per pixel instead of four 16-byte ones;
//   warps 6-7: transposers -- wait for the box (`sfull`, transaction bytes)
//     and for a free plane buffer (`pempty`), copy the pixels' four 16-byte
//     channel chunks into the four 8-channel planes the MMA descriptors view,
//     make those writes visible to the tensor core (fence.proxy.async) and
//     release the staging buffer (`sempty`) and publish the planes (`pfull`);
//   warp 1 (one lane): MMA issuer -- waits for the planes (`pfull`) and a free
//     TMEM accumulator (`tempty`), issues the 18 MMAs and commits them to
//     `pempty` (planes free) and `tfull` (accumulator ready);
//   warps 2-5: epilogue -- each reads its 32 TMEM lanes (warp w owns lanes
//     32 (w % 4) ...) of the ready accumulator, releases it (`tempty`, one
//     arrival per warp), then combines and stores its 32 pixels.
// No CTA-wide barrier inside the tile loop.  Every wait is bounded
// (mbar_wait); a timeout sets *err, every role stops, and the copies and MMAs
// still in flight are waited for (bounded) before TMEM is released.
constexpr int kWsAcc = 2;
constexpr int kWsThreads = 256;
constexpr int kStageBytes = kHH * kHW * 64;      // 11,520: the halo as 64-byte pixels
// shared memory of a CTA with ST stages (+ alignment slack); CTAs per SM as
// many as fit 228 KB, at most 8 (64 TMEM columns each)
template <int ST> constexpr int ws_smem() { return kWBytes + ST * (kStageBytes + kHaloBytes) + 128; }
template <int ST> constexpr int ws_ctas_per_sm() { return 228 * 1024 / (ws_smem<ST>() + 1024) < 8 ? 228 * 1024 / (ws_smem<ST>() + 1024) : 8; }

// kFwdProj epilogue of one pixel (see kFwdProj); w6s is [tap][channel] FP32
__device__ __forceinline__ void proj_store(const uint32_t (&r)[32], size_t pix, size_t npx,
                                           const bf16* __restrict__ skip, const float* w6s, float* __restrict__ u)
{
    __align__(16) bf16 sv[32];
#pragma unroll
    for (int q = 0; q < 4; q++)
        *reinterpret_cast<uint4*>(sv + 8 * q) = __ldg(reinterpret_cast<const uint4*>(skip + pix * 32 + 8 * q));
    float h[32];
#pragma unroll
    for (int c = 0; c < 32; c++)
        h[c] = __bfloat162float(__float2bfloat16_rn(fmaxf(__uint_as_float(r[c]) + __bfloat162float(sv[c]), 0.f)));
#pragma unroll
    for (int t = 0; t < 9; t++) {
        const float4* w4 = reinterpret_cast<const float4*>(w6s + t * 32);
        float acc = 0.f;
#pragma unroll
        for (int c4 = 0; c4 < 8; c4++) {
            const float4 w = w4[c4];
            acc += w.x * h[4 * c4];
            acc += w.y * h[4 * c4 + 1];
            acc += w.z * h[4 * c4 + 2];
            acc += w.w * h[4 * c4 + 3];
        }
        u[(size_t)t * npx + pix] = acc;
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

template <int MODE, int ST>
__global__ void __launch_bounds__(kWsThreads)
k_conv_ws(const __grid_constant__ CUtensorMap tin, int B, int H, int W, const bf16* __restrict__ wk,
          const void* __restrict__ aux, void* __restrict__ out, bf16* __restrict__ out16, int* __restrict__ err,
          const float* __restrict__ proj)
{
    extern __shared__ unsigned char dsm_raw[];
    unsigned char* dsm = reinterpret_cast<unsigned char*>(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
    unsigned char* wsm = dsm;                                 // weights, kWBytes
    unsigned char* stage = dsm + kWBytes;                     // ST x kStageBytes (TMA boxes)
    unsigned char* planes = stage + ST * kStageBytes;         // ST x kHaloBytes (MMA operands)
    __shared__ __align__(8) uint64_t sfull[ST], sempty[ST], pfull[ST], pempty[ST], tfull[kWsAcc], tempty[kWsAcc];
    __shared__ uint32_t tmem_sh;
    __shared__ volatile int s_stop;
    __shared__ int s_loads, s_trans, s_mmas;                  // progress counts, for the error path
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 32 * 36; i += kWsThreads) {
        const int co = i / 36, j = i % 36;
        const uint4 v = *reinterpret_cast<const uint4*>(wk + co * 288 + j * 8);
        *reinterpret_cast<uint4*>(wsm + (co >> 3) * kWRowGroup + j * 128 + (co & 7) * 16) = v;
    }
    __shared__ __align__(16) float w6s[MODE == kFwdProj ? 9 * 32 : 4];    // output-layer weights [tap][channel]
    if constexpr (MODE == kFwdProj)
        for (int i = tid; i < 9 * 32; i += kWsThreads) w6s[(i % 9) * 32 + i / 9] = proj[i];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(&tmem_sh))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        s_stop = 0;
        s_loads = 0;
        s_trans = 0;
        s_mmas = 0;
        for (int q = 0; q < ST; q++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sfull[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(smem_u32(&sempty[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(smem_u32(&pfull[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&pempty[q])) : "memory");
        }
        for (int q = 0; q < kWsAcc; q++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&tfull[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&tempty[q])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // weights: generic writes, async-proxy reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    const uint32_t wbase = smem_u32(wsm);
    const int tilesx = (W + kTW - 1) / kTW, tilesy = (H + kTH - 1) / kTH;
    const int per_img = tilesx * tilesy;
    const int ntiles = per_img * B;
    const int cnt = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile_of = [&](int i) { return (int)blockIdx.x + i * (int)gridDim.x; };

    if (warp == 0) {
        if (lane == 0) {                               // TMA producer
            for (int i = 0; i < cnt && !s_stop; i++) {
                const int q = i % ST;
                if (i >= ST && !mbar_wait(smem_u32(&sempty[q]), (uint32_t)((i / ST - 1) & 1))) {
                    s_stop = 1;
                    break;
                }
                const int t = tile_of(i);
                const int b = t / per_img, rem = t - b * per_img;
                const int y0 = (rem / tilesx) * kTH, x0 = (rem % tilesx) * kTW;
                const uint32_t bar = smem_u32(&sfull[q]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kStageBytes)
                             : "memory");
                tma_plane(smem_u32(stage + q * kStageBytes), &tin, 0, x0 - 1, y0 - 1, b, bar);
                s_loads = i + 1;
            }
        }
    } else if (warp >= 6) {                            // transposers
        const int tt = tid - 192;
        for (int i = 0; i < cnt; i++) {
            const int q = i % ST;
            bool ok = !s_stop && mbar_wait(smem_u32(&sfull[q]), (uint32_t)((i / ST) & 1));
            if (ok && i >= ST) ok = mbar_wait(smem_u32(&pempty[q]), (uint32_t)((i / ST - 1) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) s_stop = 1;
                break;
            }
            const unsigned char* src = stage + q * kStageBytes;
            unsigned char* dst = planes + q * kHaloBytes;
            for (int m = tt; m < kHH * kHW * 4; m += 64) {
                const int pix = m >> 2, part = m & 3;
                *reinterpret_cast<uint4*>(dst + part * kPlane + pix * 16) =
                    *reinterpret_cast<const uint4*>(src + pix * 64 + part * 16);
            }
            // the planes are read by the tensor core (async proxy)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(smem_u32(&sempty[q]));
                mbar_arrive(smem_u32(&pfull[q]));
                if (warp == 6) s_trans = i + 1;
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {                               // MMA issuer
            for (int i = 0; i < cnt && !s_stop; i++) {
                const int q = i % ST, a = i % kWsAcc;
                if (!mbar_wait(smem_u32(&pfull[q]), (uint32_t)((i / ST) & 1))) {
                    s_stop = 1;
                    break;
                }
                if (i >= kWsAcc && !mbar_wait(smem_u32(&tempty[a]), (uint32_t)((i / kWsAcc - 1) & 1))) {
                    s_stop = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t hb = smem_u32(planes + q * kHaloBytes);
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap % 3;
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                        const uint64_t da = umma_desc(hb + 2 * k * kPlane + (dy * kHW + dx) * 16, kPlane, kHW * 16);
                        const uint64_t db = umma_desc(wbase + (4 * tap + 2 * k) * 128, 128, kWRowGroup);
                        const uint32_t accum = (tap | k) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                            ::"r"(tmem + (uint32_t)(a * 32)), "l"(da), "l"(db), "r"(kIdesc), "r"(accum)
                            : "memory");
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&pempty[q]))
                             : "memory");
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&tfull[a]))
                             : "memory");
                s_mmas = i + 1;
            }
        }
    } else {                                           // epilogue warps 2..5
        const int lg = warp & 3;                       // TMEM lane group this warp may access
        const int m = lg * 32 + lane;                  // pixel of the 16 x 8 tile
        for (int i = 0; i < cnt; i++) {
            const int a = i % kWsAcc;
            const bool ok = !s_stop && mbar_wait(smem_u32(&tfull[a]), (uint32_t)((i / kWsAcc) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) s_stop = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)(a * 32))
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&tempty[a]));
            const int t = tile_of(i);
            const int b = t / per_img, rem = t - b * per_img;
            const int gy = (rem / tilesx) * kTH + (m >> 3), gx = (rem % tilesx) * kTW + (m & 7);
            if (gy < H && gx < W) {
                const size_t pix = ((size_t)b * H + gy) * W + gx;
                if constexpr (MODE == kFwdProj)
                    proj_store(r, pix, (size_t)B * H * W, static_cast<const bf16*>(aux), w6s,
                               static_cast<float*>(out));
                else
                    conv_store<MODE>(r, pix * 32, aux, out, out16);
            }
        }
    }
    __syncthreads();
    if (s_stop && tid == 32) {
        // report, then let the copies and MMAs still in flight finish (bounded) before TMEM is freed
        atomicOr(err, 1);
        const int nl = s_loads, nt = s_trans, nm = s_mmas;
        for (int k = nt; k < nl; k++) mbar_wait(smem_u32(&sfull[k % ST]), (uint32_t)((k / ST) & 1));
        if (nm > 0) mbar_wait(smem_u32(&tfull[(nm - 1) % kWsAcc]), (uint32_t)(((nm - 1) / kWsAcc) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Strip convolution: the activations are the MMA's A operand in TMEM.
//
// A work item is a strip of 128 consecutive output pixels of a row (the
// MMA's M: TMEM lane = x position) over a segment of rows.  Each input row
// (130 pixels with the x halo) arrives in shared memory by four TMA boxes of
// 8 channels (the canonical K-major planes of the tiled kernels), and one
// thread copies it into TMEM three times, shifted by -1, 0, +1 pixels
// (tcgen05.cp 128x256b: 128 lanes x 16 channels per copy), so that the tap
// (dy, dx) of output row y reads input row y + dy - 1 at its dx copy.  The 18
// MMAs of an output row (9 taps x K = 16 twice, N = 32) then read only the
// weights from shared memory: 1 KB per MMA instead of 4 KB of A plus 1 KB of
// B.  Rows live in a ring of four TMEM slots (48 columns each: 3 shifts x
// 16); two 32-column accumulators let the epilogue of row j overlap the MMAs
// of row j + 1; 256 TMEM columns per CTA, two CTAs per SM.  The MMAs of every output pixel run in the tiled kernels'
// order (taps in order, two K halves), so the results are theirs bit for
// bit.  Roles: warp 0 TMA producer, warp 1 copy + MMA issuer, warps 2-5
// epilogue (conv_store / proj_store of the tiled kernels).  Every wait is
// bounded; a timeout sets *err and the CTA drains what it issued.
// ---------------------------------------------------------------------------
constexpr int kSW = 128;                         // output pixels of a strip row (M)
constexpr int kSPx = kSW + 2;                    // input pixels of a row, x halo included
constexpr int kSPlane = 2176;                    // plane stride: 130 x 16 B rounded up to 128
constexpr int kSRowBytes = 4 * kSPlane;          // one input row in four 8-channel planes
constexpr int kSRows = 6;                        // input rows in shared memory
constexpr int kSSlots = 4;                       // input rows in TMEM
constexpr int kSSlotCols = 48;                   // TMEM columns of a row: 3 shifts x 16
constexpr int kSDcol = kSSlots * kSSlotCols;     // TMEM column of the two accumulators (192)
constexpr int kSTmemCols = 256;
constexpr int kSCtasPerSm = 2;
constexpr int kSThreads = 192;
// two CTAs per SM (256 TMEM columns each): the request is padded past a third
// of the SM's shared memory, so that no third CTA (which would wait for TMEM)
// is placed
constexpr int kStripSmemUsed = kWBytes + kSRows * kSRowBytes + 128;
constexpr int kStripSmem = kStripSmemUsed > 80 * 1024 ? kStripSmemUsed : 80 * 1024;

struct StripGeo {
    int B, H, W, nstrips, nsegs, rs;            // rs: output rows per segment
};

__device__ __forceinline__ void strip_item(const StripGeo& g, int t, int& b, int& sx, int& y0, int& y1)
{
    const int per_img = g.nstrips * g.nsegs;
    b = t / per_img;
    const int rem = t - b * per_img;
    sx = rem / g.nsegs;
    y0 = (rem - sx * g.nsegs) * g.rs;
    y1 = min(g.H, y0 + g.rs);
}

template <int MODE>
__global__ void __launch_bounds__(kSThreads, kSCtasPerSm)
k_conv_strip(const __grid_constant__ CUtensorMap trow, StripGeo g, const bf16* __restrict__ wk,
             const void* __restrict__ aux, void* __restrict__ out, bf16* __restrict__ out16, int* __restrict__ err,
             const float* __restrict__ proj)
{
    extern __shared__ unsigned char dsm_raw[];
    unsigned char* dsm = reinterpret_cast<unsigned char*>(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
    unsigned char* wsm = dsm;                                  // weights, kWBytes
    unsigned char* rows = dsm + kWBytes;                       // kSRows input rows
    __shared__ __align__(8) uint64_t rfull[kSRows], rcp[kSRows], dfull[2], dempty[2];
    __shared__ uint32_t tmem_sh;
    __shared__ volatile int s_stop;
    __shared__ int s_loads, s_copies, s_mmas;                  // progress counts, for the error path
    __shared__ __align__(16) float w6s[MODE == kFwdProj ? 9 * 32 : 4];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 32 * 36; i += kSThreads) {
        const int co = i / 36, j = i % 36;
        const uint4 v = *reinterpret_cast<const uint4*>(wk + co * 288 + j * 8);
        *reinterpret_cast<uint4*>(wsm + (co >> 3) * kWRowGroup + j * 128 + (co & 7) * 16) = v;
    }
    if constexpr (MODE == kFwdProj)
        for (int i = tid; i < 9 * 32; i += kSThreads) w6s[(i % 9) * 32 + i / 9] = proj[i];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "n"(kSTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        s_stop = 0;
        s_loads = 0;
        s_copies = 0;
        s_mmas = 0;
        for (int q = 0; q < kSRows; q++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&rfull[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&rcp[q])) : "memory");
        }
        for (int q = 0; q < 2; q++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&dfull[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&dempty[q])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // weights: generic writes, async-proxy reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    const uint32_t wbase = smem_u32(wsm);
    const uint32_t rbase = smem_u32(rows);
    const int items = g.B * g.nstrips * g.nsegs;
    const int cnt = (int)blockIdx.x < items ? (items - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 0) {
        if (lane == 0) {                               // TMA producer: the input rows of every item in order
            int q = 0;
            for (int i = 0; i < cnt && !s_stop; i++) {
                int b, sx, y0, y1;
                strip_item(g, (int)blockIdx.x + i * (int)gridDim.x, b, sx, y0, y1);
                for (int yin = y0 - 1; yin <= y1 && !s_stop; yin++, q++) {
                    const int sl = q % kSRows;
                    if (q >= kSRows && !mbar_wait(smem_u32(&rcp[sl]), (uint32_t)((q / kSRows - 1) & 1))) {
                        s_stop = 1;
                        break;
                    }
                    const uint32_t bar = smem_u32(&rfull[sl]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                                 "r"(4 * kSPx * 16)
                                 : "memory");
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        tma_plane(rbase + sl * kSRowBytes + c * kSPlane, &trow, 8 * c, sx * kSW - 1, yin, b, bar);
                    s_loads = q + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int q = 0;                                 // input rows copied into TMEM (CTA-wide sequence)
            int j = 0;                                 // output rows issued
            // input row qq: wait for its TMA boxes, copy it three times shifted
            // into TMEM slot qq % kSSlots, commit the copies to rcp
            auto copy_row = [&](int qq) -> bool {
                const int sl = qq % kSRows;
                if (!mbar_wait(smem_u32(&rfull[sl]), (uint32_t)((qq / kSRows) & 1))) return false;
                const uint32_t src = rbase + sl * kSRowBytes;
                const uint32_t dst = tmem + (uint32_t)((qq % kSSlots) * kSSlotCols);
#pragma unroll
                for (int dx = 0; dx < 3; dx++)
#pragma unroll
                    for (int kh = 0; kh < 2; kh++) {
                        const uint64_t sd = umma_desc(src + 2 * kh * kSPlane + dx * 16, kSPlane, 128);
                        asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(dst + (uint32_t)(dx * 16 + kh * 8)),
                                     "l"(sd)
                                     : "memory");
                    }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&rcp[sl]))
                             : "memory");
                s_copies = qq + 1;
                return true;
            };
            auto copied = [&](int qq) {
                return mbar_wait(smem_u32(&rcp[qq % kSRows]), (uint32_t)((qq / kSRows) & 1));
            };
            for (int i = 0; i < cnt && !s_stop; i++) {
                int b, sx, y0, y1;
                strip_item(g, (int)blockIdx.x + i * (int)gridDim.x, b, sx, y0, y1);
                (void)b;
                (void)sx;
                const int q0 = q;                      // sequence number of input row y0 - 1
                // the previous item's MMAs are complete before its TMEM rows are overwritten
                if (j > 0 && !mbar_wait(smem_u32(&dfull[(j - 1) & 1]), (uint32_t)(((j - 1) >> 1) & 1))) {
                    s_stop = 1;
                    break;
                }
                bool ok = copy_row(q0) && copy_row(q0 + 1) && copy_row(q0 + 2);
                q = q0 + 3;
                for (int y = y0; ok && y < y1; y++, j++) {
                    const int a = j & 1, r = y - y0;
                    // the epilogue has read accumulator a (output row j - 2)
                    if (j >= 2 && !mbar_wait(smem_u32(&dempty[a]), (uint32_t)(((j >> 1) - 1) & 1))) {
                        ok = false;
                        break;
                    }
                    if (!(copied(q0 + r) && copied(q0 + r + 1) && copied(q0 + r + 2))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                    for (int tap = 0; tap < 9; tap++) {
                        const int dy = tap / 3, dx = tap % 3;
                        const uint32_t arow = tmem + (uint32_t)(((q0 + r + dy) % kSSlots) * kSSlotCols + dx * 16);
#pragma unroll
                        for (int kh = 0; kh < 2; kh++) {
                            const uint64_t db = umma_desc(wbase + (4 * tap + 2 * kh) * 128, 128, kWRowGroup);
                            const uint32_t accum = (tap | kh) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
                                ::"r"(tmem + (uint32_t)(kSDcol + a * 32)), "r"(arow + (uint32_t)(kh * 8)), "l"(db),
                                  "r"(kIdesc), "r"(accum)
                                : "memory");
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&dfull[a]))
                                 : "memory");
                    s_mmas = j + 1;
                    // input row y + 2 goes into the slot of input row y - 2, which
                    // output row j - 1 reads last: wait for that row's MMAs (row j's
                    // are queued behind them), then copy
                    if (y + 2 <= y1) {
                        if (j >= 1 && !mbar_wait(smem_u32(&dfull[(j - 1) & 1]), (uint32_t)(((j - 1) >> 1) & 1))) {
                            ok = false;
                            break;
                        }
                        if (!copy_row(q0 + r + 3)) {
                            ok = false;
                            break;
                        }
                        q = q0 + r + 4;
                    }
                }
                if (!ok) {
                    s_stop = 1;
                    break;
                }
            }
        }
    } else {
        const int lg = warp & 3;                       // TMEM lane group of this warp
        int j = 0;
        bool ok = true;
        for (int i = 0; ok && i < cnt; i++) {
            int b, sx, y0, y1;
            strip_item(g, (int)blockIdx.x + i * (int)gridDim.x, b, sx, y0, y1);
            for (int y = y0; y < y1; y++, j++) {
                const int a = j & 1;
                ok = !s_stop && mbar_wait(smem_u32(&dfull[a]), (uint32_t)((j >> 1) & 1));
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) s_stop = 1;
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                uint32_t r[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)(kSDcol + a * 32))
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&dempty[a]));
                const int x = sx * kSW + lg * 32 + lane;
                if (x < g.W) {
                    const size_t pix = ((size_t)b * g.H + y) * g.W + x;
                    if constexpr (MODE == kFwdProj)
                        proj_store(r, pix, (size_t)g.B * g.H * g.W, static_cast<const bf16*>(aux), w6s,
                                   static_cast<float*>(out));
                    else
                        conv_store<MODE>(r, pix * 32, aux, out, out16);
                }
            }
        }
    }
    __syncthreads();
    if (s_stop && tid == 32) {
        // report, then let the loads, copies and MMAs still in flight finish (bounded) before TMEM is freed
        atomicOr(err, 1);
        const int nl = s_loads, nc = s_copies, nm = s_mmas;
        for (int k = nc; k < nl; k++) mbar_wait(smem_u32(&rfull[k % kSRows]), (uint32_t)((k / kSRows) & 1));
        if (nc > 0) mbar_wait(smem_u32(&rcp[(nc - 1) % kSRows]), (uint32_t)(((nc - 1) / kSRows) & 1));
        if (nm > 0) mbar_wait(smem_u32(&dfull[(nm - 1) & 1]), (uint32_t)(((nm - 1) >> 1) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(kSTmemCols) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Weight gradient of a 32 -> 32 layer on the tensor cores:
//   dW[co][tap][ci] = sum_p G[p][co] X[p + tap][ci]
// One MMA per tap and 16 pixels: D_tap (M = 128 rows, the first 32 = co;
// N = 32 = ci) += A (G^T: rows co, K = 16 pixels) x B_tap (rows ci, K = the
// same 16 pixels of X shifted by the tap).  Both operands are K-major
// (channel-planar tiles in shared memory: core matrices of 8 channels x 8
// pixels), so the pixels are the contraction: a tile of 8 x 32 output pixels
// is 16 K-steps, its X halo (10 rows) is kept in three copies shifted by
// dx - 1 pixels so that every tap's B is a descriptor view (the dy shift is
// whole 32-pixel rows).  A's rows 32..127 are a zero region.  The nine
// 32-column accumulators stay in TMEM over all tiles of the CTA; the epilogue
// writes the CTA's partial dW (FP32, [co][tap * 32 + ci]) for the ordered
// reduction of k_wgrad_mid_reduce.  Staging is done by all threads from the
// BF16 images, one tile at a time (training-path kernel).
// ---------------------------------------------------------------------------
// Core matrices are 128 bytes apart along K plus 16 bytes of padding (LBO =
// 144) and the 8-channel row groups 32 bytes past a multiple of 128 (SBO), so
// that the staging stores of a warp (4 channel groups x 2 chunks x 4 pixel
// pairs, one channel row each) fall into 32 distinct banks.
constexpr int kGTH = 8, kGTW = 16;               // output tile rows x columns (128 pixels)
constexpr int kGLbo = 144;
constexpr int kGChunks = kGTH * kGTW / 8;        // 16 chunks of 8 pixels
constexpr int kGSbo = kGChunks * kGLbo + 32;     // A: bytes per 8-channel row group (2,336)
constexpr int kGABytes = 16 * kGSbo;             // 128 rows (32 real + 96 zero): 37,376
constexpr int kXRows = kGTH + 2;                 // halo rows
constexpr int kXChunks = kXRows * kGTW / 8;      // 20
constexpr int kXSbo = kXChunks * kGLbo + 96;     // 2,976
constexpr int kXCopyBytes = 4 * kXSbo;           // 11,904
constexpr int kGStage = kGABytes + 3 * kXCopyBytes;   // 73,088: one tile's operands
constexpr int kWgSmem = 2 * kGStage + 128;       // two stages: staging overlaps the MMAs

__device__ __forceinline__ uint4 ld_px(const bf16* __restrict__ img, int b, int H, int W, int y, int x)
{
    if (y < 0 || y >= H || x < 0 || x >= W) return make_uint4(0, 0, 0, 0);
    return __ldg(reinterpret_cast<const uint4*>(img + (((size_t)b * H + y) * W + x) * 32));
}

// two pixels' 8 channels (a = pixel k, c = pixel k + 1, k even) into the
// K-major core matrix rows: 8 words of (pixel k, pixel k + 1) per channel
__device__ __forceinline__ void put_pair(unsigned char* dst, const uint4& a, const uint4& c)
{
    const uint32_t av[4] = {a.x, a.y, a.z, a.w}, cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
        // channel 2j in the low halves, 2j + 1 in the high halves
        *reinterpret_cast<uint32_t*>(dst + (2 * j) * 16) = (av[j] & 0xFFFFu) | (cv[j] << 16);
        *reinterpret_cast<uint32_t*>(dst + (2 * j + 1) * 16) = (av[j] >> 16) | (cv[j] & 0xFFFF0000u);
    }
}

__global__ void __launch_bounds__(256, 1)
k_wgrad_tc(int B, int H, int W, const bf16* __restrict__ G, const bf16* __restrict__ X, float* __restrict__ part,
           int* __restrict__ err)
{
    extern __shared__ unsigned char dsm_raw[];
    unsigned char* dsm = reinterpret_cast<unsigned char*>(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
    // stage s: A (G^T, 128 rows) at s * kGStage, then the three shifted X copies
    __shared__ __align__(8) uint64_t mdone[2];
    __shared__ uint32_t tmem_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 2 * kGStage / 16; i += 256) reinterpret_cast<uint4*>(dsm)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tmem_sh))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mdone[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mdone[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    const uint32_t sbase = smem_u32(dsm);
    const int tx = (W + kGTW - 1) / kGTW, ty = (H + kGTH - 1) / kGTH;
    const int ntiles = tx * ty * B;
    bool ok = true;
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
        const int b = t / (tx * ty), rem = t - b * (tx * ty);
        const int y0 = (rem / tx) * kGTH, x0 = (rem % tx) * kGTW;
        const int sg = it & 1;
        unsigned char* asm_ = dsm + sg * kGStage;
        unsigned char* xsm = asm_ + kGABytes;
        if (it >= 2) {                               // tile it - 2's MMAs have read this stage
            const bool w = tid == 0 ? mbar_wait(smem_u32(&mdone[sg]), (uint32_t)(((it >> 1) - 1) & 1)) : true;
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
        }
        // G tile -> A rows 0..31: 128 pixel pairs x 4 channel groups
        for (int i = tid; i < (kGTH * kGTW / 2) * 4; i += 256) {      // one item per thread
            const int pp = i >> 2, g = i & 3, k = 2 * pp;
            const int r = k / kGTW, c = k % kGTW;
            // the 8 channels of group g are the g-th 16 bytes of the pixel's 64
            const uint4 a8 = ld_px(G + 8 * g, b, H, W, y0 + r, x0 + c);
            const uint4 c8 = ld_px(G + 8 * g, b, H, W, y0 + r, x0 + c + 1);
            put_pair(asm_ + g * kGSbo + (k / 8) * kGLbo + (k % 8) * 2, a8, c8);
        }
        // X halo -> three copies shifted by dx - 1: 10 rows x 16 pairs x 4 groups each
        for (int i = tid; i < 3 * (kXRows * kGTW / 2) * 4; i += 256) {
            const int g = i & 3, rest = i >> 2;
            const int dx = rest / (kXRows * kGTW / 2), pp = rest % (kXRows * kGTW / 2), k = 2 * pp;
            const int hr = k / kGTW, c = k % kGTW;
            const uint4 a8 = ld_px(X + 8 * g, b, H, W, y0 + hr - 1, x0 + c + dx - 1);
            const uint4 c8 = ld_px(X + 8 * g, b, H, W, y0 + hr - 1, x0 + c + dx);
            put_pair(xsm + dx * kXCopyBytes + g * kXSbo + (k / 8) * kGLbo + (k % 8) * 2, a8, c8);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            const uint32_t abase = sbase + sg * kGStage, xbase = abase + kGABytes;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int sk = 0; sk < kGTH * kGTW / 16; sk++) {         // one K-step per 16-pixel tile row
                const int r = sk, h = 0;
                const uint64_t da = umma_desc(abase + sk * 2 * kGLbo, kGLbo, kGSbo);
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap % 3;
                    const uint64_t db =
                        umma_desc(xbase + dx * kXCopyBytes + ((r + dy) * (kGTW / 8) + 2 * h) * kGLbo, kGLbo, kXSbo);
                    const uint32_t accum = (it > 0 || sk > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(tmem + (uint32_t)(tap * 32)), "l"(da), "l"(db), "r"(kIdesc), "r"(accum)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mdone[sg]))
                         : "memory");
        }
    }
    // all MMAs complete, then each CTA writes its partial dW from TMEM rows 0..31 (warp 0)
    // commits complete in order: the last tile's covers every MMA
    const bool w = (tid == 0 && ok && it > 0) ? mbar_wait(smem_u32(&mdone[(it - 1) & 1]), (uint32_t)(((it - 1) >> 1) & 1))
                                              : true;
    ok = __syncthreads_and(ok && w);
    if (!ok && tid == 0) atomicOr(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) {
        float* dst = part + (size_t)blockIdx.x * (32 * 288) + (size_t)lane * 288;
#pragma unroll 1
        for (int tap = 0; tap < 9; tap++) {
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(tmem + (uint32_t)(tap * 32))
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int ci = 0; ci < 32; ci++)
                dst[tap * 32 + ci] = (it > 0 && ok) ? __uint_as_float(r[ci]) : 0.f;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
}

}  // namespace

// The driver's tensor-map encoder, fetched once through the runtime (no link
// against libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        JFG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        JFG_CHECK(q == cudaDriverEntryPointSuccess && p, JFG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// box_c: channels per box (32: the whole 64-byte pixel; 8: one plane)
static CUtensorMap conv_input_map(int B, int H, int W, const __nv_bfloat16* in, int box_c)
{
    CUtensorMap map;
    const cuuint64_t dims[4] = {32, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {64, (cuuint64_t)W * 64, (cuuint64_t)W * H * 64};
    const cuuint32_t box[4] = {(cuuint32_t)box_c, (cuuint32_t)kHW, (cuuint32_t)kHH, 1};
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    CUresult r = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(in), dims,
                                      strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    JFG_CHECK(r == CUDA_SUCCESS, JFG_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return map;
}

// One input row of a strip: box of 8 channels x 130 pixels x 1 row (zero fill
// outside the image: the x halo at the image edges and rows -1 and H).
static CUtensorMap conv_row_map(int B, int H, int W, const __nv_bfloat16* in)
{
    CUtensorMap map;
    const cuuint64_t dims[4] = {32, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {64, (cuuint64_t)W * 64, (cuuint64_t)W * H * 64};
    const cuuint32_t box[4] = {8, (cuuint32_t)kSPx, 1, 1};
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    CUresult r = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(in), dims,
                                      strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    JFG_CHECK(r == CUDA_SUCCESS, JFG_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return map;
}

// JFEM_CNN_STRIP=1 selects the strip kernel (k_conv_strip, activations in
// TMEM) for the 32 -> 32 layers
static bool use_strip()
{
    const char* e = getenv("JFEM_CNN_STRIP");
    return e && e[0] == '1';
}

// Strip geometry: strips of 128 pixels, segments of rows sized so that the
// items fill the SMs (one CTA per SM) in whole rounds: at most two items per
// CTA when the image allows.
static StripGeo strip_geo(int B, int H, int W)
{
    StripGeo g;
    g.B = B;
    g.H = H;
    g.W = W;
    g.nstrips = (W + kSW - 1) / kSW;
    const int slots = 2 * sm_count();
    int nsegs = std::max(1, slots / std::max(1, B * g.nstrips));
    nsegs = std::min(nsegs, H);
    g.rs = (H + nsegs - 1) / nsegs;
    g.nsegs = (H + g.rs - 1) / g.rs;
    return g;
}

template <int MODE>
static void launch_strip(cudaStream_t st, int B, int H, int W, const bf16* in, const bf16* w, const void* aux,
                         void* out, bf16* out16, int* err, const float* proj = nullptr)
{
    JFG_CHECK(((uintptr_t)in & 15) == 0, JFG_ERR_BAD_ARG, "convolution input not 16-byte aligned");
    const StripGeo g = strip_geo(B, H, W);
    const long long items = (long long)B * g.nstrips * g.nsegs;
    JFG_CHECK(items < (1LL << 31), JFG_ERR_UNSUPPORTED, "image too large for the strip convolution");
    const int grid = (int)std::min<long long>(items, (long long)kSCtasPerSm * sm_count());
    if (grid <= 0) return;
    static bool attr = false;
    if (!attr) {
        JFG_CUDA(cudaFuncSetAttribute(k_conv_strip<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStripSmem));
        attr = true;
    }
    const CUtensorMap map = conv_row_map(B, H, W, in);
    k_conv_strip<MODE><<<grid, kSThreads, kStripSmem, st>>>(map, g, w, aux, out, out16, err, proj);
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

// JFEM_CNN_WS=0 selects the single-role kernel (k_conv_mid_tc) instead of the
// warp-specialised pipeline (k_conv_ws); JFEM_CNN_WS_STAGES = 2, 3 or 4 sets
// its stages (default kWsDefaultStages)
constexpr int kWsDefaultStages = 2;
static bool use_ws()
{
    const char* e = getenv("JFEM_CNN_WS");
    return !(e && e[0] == '0');
}
static int ws_stages()
{
    const char* e = getenv("JFEM_CNN_WS_STAGES");
    const int v = e ? atoi(e) : kWsDefaultStages;
    return (v == 2 || v == 3 || v == 4) ? v : kWsDefaultStages;
}
static int ws_ctas(int st) { return st == 2 ? ws_ctas_per_sm<2>() : (st == 3 ? ws_ctas_per_sm<3>() : ws_ctas_per_sm<4>()); }

static int conv_grid(int B, int H, int W, const void* in)
{
    const long long ntiles = (long long)((W + kTW - 1) / kTW) * ((H + kTH - 1) / kTH) * B;
    JFG_CHECK(ntiles < (1LL << 31), JFG_ERR_UNSUPPORTED, "image too large for the tensor-core convolution");
    JFG_CHECK(((uintptr_t)in & 15) == 0, JFG_ERR_BAD_ARG, "convolution input not 16-byte aligned");
    const int per_sm = use_ws() ? ws_ctas(ws_stages()) : kTcCtasPerSm;
    return (int)std::min<long long>(ntiles, (long long)sm_count() * per_sm);
}

template <int MODE, int ST>
static void launch_ws(cudaStream_t st, int grid, const CUtensorMap& map, int B, int H, int W, const bf16* w,
                      const void* aux, void* out, bf16* out16, int* err, const float* proj = nullptr)
{
    static bool attr = false;
    if (!attr) {
        JFG_CUDA(cudaFuncSetAttribute(k_conv_ws<MODE, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, ws_smem<ST>()));
        attr = true;
    }
    k_conv_ws<MODE, ST><<<grid, kWsThreads, ws_smem<ST>(), st>>>(map, B, H, W, w, aux, out, out16, err, proj);
}

template <int MODE>
static void launch_conv(cudaStream_t st, int grid, const CUtensorMap& map, int B, int H, int W, const bf16* w,
                        const void* aux, void* out, bf16* out16, int* err)
{
    if (use_ws()) {
        switch (ws_stages()) {
        case 2: launch_ws<MODE, 2>(st, grid, map, B, H, W, w, aux, out, out16, err); break;
        case 3: launch_ws<MODE, 3>(st, grid, map, B, H, W, w, aux, out, out16, err); break;
        default: launch_ws<MODE, 4>(st, grid, map, B, H, W, w, aux, out, out16, err); break;
        }
    } else {
        k_conv_mid_tc<MODE><<<grid, kTcThreads, 0, st>>>(map, B, H, W, w, aux, out, out16, err);
    }
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

// out = relu(conv3x3(in, wk) [+ skip]) for BF16 (B, H, W, 32) images; wk is
// BF16 [32 outputs][9 taps x 32 inputs].  err is set to 1 if a TMA or MMA
// wait timed out (the output is then incomplete).
void conv_mid_tc(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* in, const __nv_bfloat16* wk,
                 const __nv_bfloat16* skip, __nv_bfloat16* out, int* err)
{
    if (use_strip()) {
        if (skip)
            launch_strip<kFwdSkip>(st, B, H, W, in, wk, skip, out, nullptr, err);
        else
            launch_strip<kFwd>(st, B, H, W, in, wk, nullptr, out, nullptr, err);
        return;
    }
    const int grid = conv_grid(B, H, W, in);
    if (grid <= 0) return;
    const CUtensorMap map = conv_input_map(B, H, W, in, use_ws() ? 32 : 8);
    if (skip)
        launch_conv<kFwdSkip>(st, grid, map, B, H, W, wk, skip, out, nullptr, err);
    else
        launch_conv<kFwd>(st, grid, map, B, H, W, wk, nullptr, out, nullptr, err);
}

// The last 32 -> 32 layer with its skip input fused with the projection of
// the 32 -> 1 output layer (kFwdProj): u receives nine FP32 planes of B*H*W
// entries, u[t][p] = sum_c w6[c][t] relu(conv + skip)[p][c] (BF16-rounded
// activations); w6 is FP32 [32 channels][9 taps].  Warp-specialised kernel
// only (the caller checks conv_proj_available()).
bool conv_proj_available() { return use_strip() || use_ws(); }

void conv_mid_tc_proj(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* in, const __nv_bfloat16* wk,
                      const __nv_bfloat16* skip, const float* w6, float* u, int* err)
{
    if (use_strip()) {
        launch_strip<kFwdProj>(st, B, H, W, in, wk, skip, u, nullptr, err, w6);
        return;
    }
    const int grid = conv_grid(B, H, W, in);
    if (grid <= 0) return;
    JFG_CHECK(use_ws(), JFG_ERR_UNSUPPORTED, "the fused output projection needs the warp-specialised convolution");
    const CUtensorMap map = conv_input_map(B, H, W, in, 32);
    switch (ws_stages()) {
    case 2: launch_ws<kFwdProj, 2>(st, grid, map, B, H, W, wk, skip, u, nullptr, err, w6); break;
    case 3: launch_ws<kFwdProj, 3>(st, grid, map, B, H, W, wk, skip, u, nullptr, err, w6); break;
    default: launch_ws<kFwdProj, 4>(st, grid, map, B, H, W, wk, skip, u, nullptr, err, w6); break;
    }
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

// Input gradient of a 32 -> 32 layer on the tensor cores: conv3x3 of the
// BF16 gradient image gin with the flipped, channel-transposed weights wt
// (the layout of wk), FP32 accumulation.  mask != nullptr: out = acc *
// (mask > 0) and out16 = its BF16 copy; else out = acc + skip (FP32).
void conv_mid_tc_bwd(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* gin, const __nv_bfloat16* wt,
                     const __nv_bfloat16* mask, const float* skip, float* out, __nv_bfloat16* out16, int* err)
{
    if (use_strip()) {
        if (mask)
            launch_strip<kBwdMask>(st, B, H, W, gin, wt, mask, out, out16, err);
        else
            launch_strip<kBwdSkip>(st, B, H, W, gin, wt, skip, out, nullptr, err);
        return;
    }
    const int grid = conv_grid(B, H, W, gin);
    if (grid <= 0) return;
    const CUtensorMap map = conv_input_map(B, H, W, gin, use_ws() ? 32 : 8);
    if (mask)
        launch_conv<kBwdMask>(st, grid, map, B, H, W, wt, mask, out, out16, err);
    else
        launch_conv<kBwdSkip>(st, grid, map, B, H, W, wt, skip, out, nullptr, err);
}

// Per-CTA partial weight gradients of a 32 -> 32 layer on the tensor cores
// (k_wgrad_tc) from the BF16 gradient image G16 and the BF16 layer input X:
// part[cta][co * 288 + tap * 32 + ci]; returns the number of CTAs (at most
// max_parts).  err is set to 1 if the MMA wait timed out.
int wgrad_mid_tc(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* G16, const __nv_bfloat16* X,
                 float* part, int max_parts, int* err)
{
    const long long ntiles = (long long)((W + kGTW - 1) / kGTW) * ((H + kGTH - 1) / kGTH) * B;
    JFG_CHECK(ntiles < (1LL << 31), JFG_ERR_UNSUPPORTED, "image too large for the tensor-core weight gradient");
    const int ctas = (int)std::min<long long>(std::min<long long>(ntiles, sm_count()), max_parts);
    if (ctas <= 0) return 0;
    static bool attr = false;
    if (!attr) {
        JFG_CUDA(cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem));
        attr = true;
    }
    k_wgrad_tc<<<ctas, 256, kWgSmem, st>>>(B, H, W, G16, X, part, err);
    JFG_CUDA(cudaGetLastError());
    note_launch();
    return ctas;
}

}  // namespace jfg
