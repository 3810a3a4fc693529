// 32 -> 32 3x3 convolution of the learned smoother's forward pass on the
// fifth-generation tensor cores (tcgen05.mma, accumulator in TMEM).
//
// Implicit GEMM per tile of 16 x 8 = 128 output pixels (the MMA's M):
//   D[p][co] = sum_{tap, ci} X[p + tap][ci] * W[co][tap * 32 + ci]
// with K = 9 taps x 32 channels = 288 = 18 MMAs of K = 16, N = 32.
//
// Shared-memory layout (canonical K-major, no swizzle: core matrices of 8
// rows x 16 bytes):
//  - the input halo (18 x 10 pixels) is stored as four planes of 8 channels,
//    pixel (hy, hx) of plane q at q * 2880 + (hy * 10 + hx) * 16.  Because a
//    tile is 8 pixels wide, the 8 rows of every core matrix of the A operand
//    of any tap are 8 consecutive halo pixels of one halo row, the next core
//    matrix (next tile row) is 160 bytes further, and the next 8 channels are
//    one plane further: every tap's A operand is a descriptor view of the
//    halo (start, LBO = plane, SBO = halo row), nothing is copied;
//  - the weights W[co][k] at (co / 8) * 4608 + (k / 8) * 128 + (co % 8) * 16
//    + (k % 8) * 2 (LBO = 128, SBO = 4608).
// One thread issues the 18 MMAs and commits them to an mbarrier; after the
// (bounded) wait each warp reads its 32 TMEM lanes (one pixel per thread, 32
// FP32 channels), adds the skip input, applies ReLU and stores BF16.
// Persistent CTAs of 128 threads stride over the tiles; ~30 KB of shared
// memory and 32 TMEM columns each (at most 16 CTAs per SM fit in 512 columns).
#include "jfg_ops.cuh"

namespace jfg {
namespace {

typedef __nv_bfloat16 bf16;

constexpr int kTH = 16, kTW = 8;                 // tile rows x columns (128 pixels)
constexpr int kHH = kTH + 2, kHW = kTW + 2;      // halo 18 x 10
constexpr int kPlane = kHH * kHW * 16;           // bytes of one 8-channel plane
constexpr int kHaloBytes = 4 * kPlane;           // 11,520
constexpr int kWRowGroup = 36 * 128;             // bytes per 8 output channels (4608)
constexpr int kWBytes = 4 * kWRowGroup;          // 18,432
constexpr int kTcThreads = 128;
constexpr int kTcCtasPerSm = 7;
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

template <int SK>
__global__ void __launch_bounds__(kTcThreads)
k_conv_mid_tc(int B, int H, int W, const bf16* __restrict__ in, const bf16* __restrict__ wk,
              const bf16* __restrict__ skip, bf16* __restrict__ out, int* __restrict__ err)
{
    __shared__ __align__(128) unsigned char wsm[kWBytes];
    __shared__ __align__(128) unsigned char halo[kHaloBytes];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 32 * 36; i += kTcThreads) {
        const int co = i / 36, j = i % 36;
        const uint4 v = *reinterpret_cast<const uint4*>(wk + co * 288 + j * 8);
        *reinterpret_cast<uint4*>(wsm + (co >> 3) * kWRowGroup + j * 128 + (co & 7) * 16) = v;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&tmem_sh))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    const uint32_t bar = smem_u32(&mbar);
    const uint32_t hbase = smem_u32(halo), wbase = smem_u32(wsm);
    const int tilesx = (W + kTW - 1) / kTW, tilesy = (H + kTH - 1) / kTH;
    const int ntiles = tilesx * tilesy * B;
    uint32_t parity = 0;
    bool healthy = true;
    for (int t = blockIdx.x; t < ntiles && healthy; t += gridDim.x) {
        const int b = t / (tilesx * tilesy), rem = t - b * (tilesx * tilesy);
        const int y0 = (rem / tilesx) * kTH, x0 = (rem % tilesx) * kTW;
        for (int i = tid; i < kHH * kHW * 4; i += kTcThreads) {
            const int q = i & 3, pix = i >> 2;
            const int hy = pix / kHW, hx = pix - hy * kHW;
            const int gy = y0 + hy - 1, gx = x0 + hx - 1;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gy >= 0 && gy < H && gx >= 0 && gx < W)
                v = *reinterpret_cast<const uint4*>(in + (((size_t)b * H + gy) * W + gx) * 32 + q * 8);
            *reinterpret_cast<uint4*>(halo + q * kPlane + (hy * kHW + hx) * 16) = v;
        }
        // generic-proxy writes -> visible to the tensor core's async proxy; the
        // previous tile's TMEM reads finish before the MMAs overwrite D
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                const int dy = tap / 3, dx = tap % 3;
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    const uint64_t da = umma_desc(hbase + 2 * s * kPlane + (dy * kHW + dx) * 16, kPlane, kHW * 16);
                    const uint64_t db = umma_desc(wbase + (4 * tap + 2 * s) * 128, 128, kWRowGroup);
                    const uint32_t accum = (tap | s) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(accum)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        const bool ok = mbar_wait(bar, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(err, 1);
            healthy = false;
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
            : "r"(tmem + ((uint32_t)(warp * 32) << 16))
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int m = warp * 32 + lane;
        const int gy = y0 + (m >> 3), gx = x0 + (m & 7);
        if (gy < H && gx < W) {
            const size_t base = (((size_t)b * H + gy) * W + gx) * 32;
            __align__(16) bf16 o[32];
            __align__(16) bf16 sv[32];
            if (SK) {
#pragma unroll
                for (int q = 0; q < 4; q++)
                    *reinterpret_cast<uint4*>(sv + 8 * q) = *reinterpret_cast<const uint4*>(skip + base + 8 * q);
            }
#pragma unroll
            for (int c = 0; c < 32; c++) {
                float v = __uint_as_float(r[c]);
                if (SK) v += __bfloat162float(sv[c]);
                o[c] = __float2bfloat16_rn(fmaxf(v, 0.f));
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                *reinterpret_cast<uint4*>(out + base + 8 * q) = *reinterpret_cast<const uint4*>(o + 8 * q);
        }
    }
    if (!healthy) mbar_wait(bar, parity ^ 1u);   // MMAs in flight finish before their TMEM is released
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
    }
}

}  // namespace

// out = relu(conv3x3(in, wk) [+ skip]) for BF16 (B, H, W, 32) images; wk is
// BF16 [32 outputs][9 taps x 32 inputs].  err is set to 1 if an MMA wait
// timed out (the output is then incomplete).
void conv_mid_tc(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* in, const __nv_bfloat16* wk,
                 const __nv_bfloat16* skip, __nv_bfloat16* out, int* err)
{
    const long long ntiles = (long long)((W + kTW - 1) / kTW) * ((H + kTH - 1) / kTH) * B;
    JFG_CHECK(ntiles < (1LL << 31), JFG_ERR_UNSUPPORTED, "image too large for the tensor-core convolution");
    const int grid = (int)std::min<long long>(ntiles, (long long)sm_count() * kTcCtasPerSm);
    if (grid <= 0) return;
    if (skip)
        k_conv_mid_tc<1><<<grid, kTcThreads, 0, st>>>(B, H, W, in, wk, skip, out, err);
    else
        k_conv_mid_tc<0><<<grid, kTcThreads, 0, st>>>(B, H, W, in, wk, nullptr, out, err);
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

}  // namespace jfg
