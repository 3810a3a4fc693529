// The learned smoother: a 6-layer 3x3 convolutional residual network on the
// node grid (C = 32 channels, no biases), trained and applied on the GPU.
//
//   h1 = relu(conv1(x))          1 -> 32   (FP32 CUDA cores, BF16 out)
//   a2 = relu(conv2(h1))         32 -> 32  (BF16 tensor cores, FP32 accumulate)
//   h3 = relu(h1 + conv3(a2))    32 -> 32
//   a4 = relu(conv4(h3))         32 -> 32
//   h5 = relu(h3 + conv5(a4))    32 -> 32
//   y  = conv6(h5)               32 -> 1   (FP32 CUDA cores)
//
// The forward 32 -> 32 convolutions run on tcgen05 with TMEM accumulators
// (jfg_cnn_tc.cu).  The kernels below are the mma.sync versions: the input
// gradients of the backward pass, and the forward when JFEM_CNN_TC=0.  They
// are implicit GEMMs (M = pixels, N = 32,
// K = 9 taps x 32 channels) on mma.sync m16n8k16 BF16 with FP32 accumulators:
// a CTA stages an 18x18 halo of NHWC activations and the 32x288 weights in
// shared memory (padded rows, conflict-free ldmatrix) and each warp computes
// two 16-pixel rows x 32 outputs.  The same kernel computes the input
// gradient with flipped, channel-transposed weights.  The weight gradient is
// a second implicit GEMM (M = 32 outputs, N = 288, K = pixels) with
// ldmatrix.trans fragments, one warp per tap, and a deterministic reduction
// of per-CTA partials.  Master weights and Adam moments are FP32.
#include <cmath>
#include <cstring>

#include "jfg_krylov.cuh"

namespace jfg {

constexpr int kC = 32;                         // channels
constexpr int kTile = 16;                      // output tile edge (pixels)
constexpr int kHalo = kTile + 2;
constexpr int kPixStride = 40;                 // bf16 per staged pixel (32 + 8 pad)
constexpr int kWStride = 9 * kC + 8;           // bf16 per staged weight row (288 + 8 pad)
constexpr int kMidParams = kC * kC * 9;        // 9216
constexpr int kNumParams = kC * 9 + 4 * kMidParams + kC * 9;   // 37440
constexpr int kLayerOff[7] = {0, 288, 288 + 9216, 288 + 2 * 9216, 288 + 3 * 9216, 288 + 4 * 9216, kNumParams};

namespace {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float ld_as_f(const bf16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float ld_as_f(const float* p) { return *p; }

// Stages 8 channels of one pixel (InT) as bf16 into shared memory,
// multiplied by (mask > 0) when a mask is given; zeros outside the image.
template <typename InT>
__device__ __forceinline__ void stage8(bf16* dst, const InT* src, const bf16* mask, bool inside)
{
    __align__(16) bf16 v[8];
    if (inside) {
#pragma unroll
        for (int c = 0; c < 8; c++) {
            float f = ld_as_f(src + c);
            if (mask && !(__bfloat162float(mask[c]) > 0.f)) f = 0.f;
            v[c] = __float2bfloat16_rn(f);
        }
    } else {
#pragma unroll
        for (int c = 0; c < 8; c++) v[c] = __float2bfloat16_rn(0.f);
    }
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
}

// 32 -> 32 convolution, implicit GEMM on tensor cores.
//   out = [relu]( conv(in [* (imask > 0)], Wk) [+ skip] ) [* (omask > 0)]
// Wk: bf16 [32 outputs][9 taps x 32 inputs].  SK: 0 no skip, 1 bf16, 2 float.
template <typename InT, typename OutT, int SK, bool RELU, bool OMASK>
__global__ void __launch_bounds__(256)
k_conv_mid(int B, int H, int W, const InT* __restrict__ in, const bf16* __restrict__ imask,
           const bf16* __restrict__ wk, const void* __restrict__ skip, const bf16* __restrict__ omask,
           OutT* __restrict__ out)
{
    __shared__ __align__(16) bf16 halo[kHalo * kHalo * kPixStride];
    __shared__ __align__(16) bf16 wsm[kC * kWStride];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile, b = blockIdx.z;
    // weights: 32 rows x 36 chunks of 8
    for (int i = tid; i < kC * 36; i += 256) {
        int row = i / 36, ch = i % 36;
        *reinterpret_cast<uint4*>(wsm + row * kWStride + ch * 8) =
            *reinterpret_cast<const uint4*>(wk + row * 288 + ch * 8);
    }
    // halo: 324 pixels x 4 chunks of 8 channels
    for (int i = tid; i < kHalo * kHalo * 4; i += 256) {
        int pix = i >> 2, part = i & 3;
        int hy = pix / kHalo, hx = pix % kHalo;
        int gy = y0 + hy - 1, gx = x0 + hx - 1;
        bool inside = gy >= 0 && gy < H && gx >= 0 && gx < W;
        size_t g = inside ? (((size_t)b * H + gy) * W + gx) * kC + part * 8 : 0;
        stage8<InT>(halo + pix * kPixStride + part * 8, in + g, imask ? imask + g : nullptr, inside);
    }
    __syncthreads();
    float acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[mi][j][q] = 0.f;
    const int mm = lane >> 3, rr = lane & 7;
#pragma unroll 1
    for (int tap = 0; tap < 9; tap++) {
        const int dy = tap / 3, dx = tap % 3;
#pragma unroll
        for (int c = 0; c < 2; c++) {
            uint32_t a[2][4];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) {
                const int ry = 2 * warp + mi;
                const int px = rr + 8 * (mm & 1);
                ldsm_x4(a[mi], halo + ((ry + dy) * kHalo + (px + dx)) * kPixStride + 16 * c + 8 * (mm >> 1));
            }
            uint32_t bq[2][4];
#pragma unroll
            for (int jp = 0; jp < 2; jp++) {
                const int n = 8 * (2 * jp + (mm >> 1)) + rr;
                ldsm_x4(bq[jp], wsm + n * kWStride + tap * 32 + 16 * c + 8 * (mm & 1));
            }
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_bf16(acc[mi][j], a[mi], bq[j >> 1][2 * (j & 1)], bq[j >> 1][2 * (j & 1) + 1]);
        }
    }
    // epilogue
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 2; mi++) {
        const int gy = y0 + 2 * warp + mi;
        if (gy >= H) continue;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int gx = x0 + g + 8 * half;
            if (gx >= W) continue;
            const size_t base = (((size_t)b * H + gy) * W + gx) * kC;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int co = 8 * j + 2 * t;
                float v0 = acc[mi][j][2 * half], v1 = acc[mi][j][2 * half + 1];
                if (SK == 1) {
                    const bf16* s = static_cast<const bf16*>(skip) + base + co;
                    v0 += __bfloat162float(s[0]);
                    v1 += __bfloat162float(s[1]);
                } else if (SK == 2) {
                    const float* s = static_cast<const float*>(skip) + base + co;
                    v0 += s[0];
                    v1 += s[1];
                }
                if (RELU) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                if (OMASK) {
                    if (!(__bfloat162float(omask[base + co]) > 0.f)) v0 = 0.f;
                    if (!(__bfloat162float(omask[base + co + 1]) > 0.f)) v1 = 0.f;
                }
                if constexpr (sizeof(OutT) == 2) {
                    __nv_bfloat162 p;
                    p.x = __float2bfloat16_rn(v0);
                    p.y = __float2bfloat16_rn(v1);
                    *reinterpret_cast<__nv_bfloat162*>(out + base + co) = p;
                } else {
                    *reinterpret_cast<float2*>(out + base + co) = make_float2(v0, v1);
                }
            }
        }
    }
}

// Weight gradient of a 32 -> 32 layer: dW[co][ci][tap] = sum_p G[p][co] X[p + tap][ci].
// 9 warps (one per tap); CTAs stride over 16x16 pixel tiles; per-CTA partials
// part[cta][co][tap*32 + ci] (FP32).
__global__ void __launch_bounds__(288)
k_wgrad_mid(int B, int H, int W, const float* __restrict__ G, const bf16* __restrict__ X, float* __restrict__ part)
{
    __shared__ __align__(16) bf16 gsm[kTile * kTile * kPixStride];
    __shared__ __align__(16) bf16 xh[kHalo * kHalo * kPixStride];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tx = (W + kTile - 1) / kTile, ty = (H + kTile - 1) / kTile;
    const int ntiles = tx * ty * B;
    float acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[mi][j][q] = 0.f;
    const int dy = warp / 3, dx = warp % 3;
    const int mm = lane >> 3, rr = lane & 7;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int b = tile / (tx * ty);
        const int rem = tile % (tx * ty);
        const int y0 = (rem / tx) * kTile, x0 = (rem % tx) * kTile;
        __syncthreads();
        for (int i = tid; i < kTile * kTile * 4; i += 288) {
            int pix = i >> 2, part8 = i & 3;
            int gy = y0 + pix / kTile, gx = x0 + pix % kTile;
            bool inside = gy < H && gx < W;
            size_t g = inside ? (((size_t)b * H + gy) * W + gx) * kC + part8 * 8 : 0;
            stage8<float>(gsm + pix * kPixStride + part8 * 8, G + g, nullptr, inside);
        }
        for (int i = tid; i < kHalo * kHalo * 4; i += 288) {
            int pix = i >> 2, part8 = i & 3;
            int hy = pix / kHalo, hx = pix % kHalo;
            int gy = y0 + hy - 1, gx = x0 + hx - 1;
            bool inside = gy >= 0 && gy < H && gx >= 0 && gx < W;
            size_t g = inside ? (((size_t)b * H + gy) * W + gx) * kC + part8 * 8 : 0;
            stage8<bf16>(xh + pix * kPixStride + part8 * 8, X + g, nullptr, inside);
        }
        __syncthreads();
#pragma unroll 1
        for (int ry = 0; ry < kTile; ry++) {
            // A = G^T (m = co, k = 16 pixels of row ry) via ldmatrix.trans
            uint32_t a[2][4];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) {
                const int px = rr + 8 * (mm >> 1);
                const int co = 16 * mi + 8 * (mm & 1);
                ldsm_x4_t(a[mi], gsm + (ry * kTile + px) * kPixStride + co);
            }
            // B = X shifted by the tap (k = pixels, n = ci) via ldmatrix.trans
            uint32_t bq[2][4];
#pragma unroll
            for (int jp = 0; jp < 2; jp++) {
                const int px = rr + 8 * (mm & 1);
                const int ci = 8 * (2 * jp + (mm >> 1));
                bq[jp][0] = 0;
                ldsm_x4_t(bq[jp], xh + ((ry + dy) * kHalo + (px + dx)) * kPixStride + ci);
            }
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    mma_bf16(acc[mi][j], a[mi], bq[j >> 1][2 * (j & 1)], bq[j >> 1][2 * (j & 1) + 1]);
        }
    }
    // acc[mi][j]: rows m = co = 16 mi + g (+8), cols n = ci = 8 j + 2 t (+1)
    const int g = lane >> 2, t = lane & 3;
    float* dst = part + (size_t)blockIdx.x * kMidParams;
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int co = 16 * mi + g + 8 * (q >> 1);
                const int ci = 8 * j + 2 * t + (q & 1);
                dst[co * 288 + warp * 32 + ci] = acc[mi][j][q];
            }
}

// sum of per-CTA partials in CTA order -> dW in (co, ci, dy, dx) layout
__global__ void k_wgrad_mid_reduce(int nparts, const float* __restrict__ part, float* __restrict__ dw)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;   // index in [co][tap*32 + ci]
    if (i >= kMidParams) return;
    float s = 0.f;
    for (int p = 0; p < nparts; p++) s += part[(size_t)p * kMidParams + i];
    int co = i / 288, k = i % 288, tap = k / 32, ci = k % 32;
    dw[(co * kC + ci) * 9 + tap] = s;
}

// first layer 1 -> 32 with ReLU: h1 = relu(sum_tap w1[co][tap] x[p + tap])
// First and last layers on CUDA cores.  A CTA row of the grid is one image
// row (blockIdx.y = b * H + y); four lanes per pixel, lane q owning channels
// 8q .. 8q + 7 (one 16-byte chunk of the pixel's 64-byte activation row), so
// a warp's activation loads and stores cover eight whole consecutive pixel
// rows.  No division per pixel, the nine taps unrolled with predicated
// loads; weights in shared memory as [tap][channel], read as float4 vectors
// at uniform addresses.
constexpr int kLanesPerPx = 4;
constexpr int kEdgePx = 256 / kLanesPerPx;        // pixels of one CTA (64 along x)

// first layer 1 -> 32 with ReLU: h1[p][co] = relu(sum_tap w1[co][tap] x[p + tap]),
// each output's taps summed in order.  A thread keeps the 72 weights of its
// eight channels in registers and walks kInRows rows down one column with a
// sliding 3 x 3 input window (three new inputs per row), so the weights are
// read from shared memory once per kInRows pixels.
constexpr int kInRows = 8;

__global__ void __launch_bounds__(256)
k_conv_in(int B, int H, int W, const float* __restrict__ x, const float* __restrict__ w1, bf16* __restrict__ h1)
{
    __shared__ __align__(16) float ws[9 * kC];
    for (int i = threadIdx.x; i < kC * 9; i += blockDim.x) ws[(i % 9) * kC + i / 9] = w1[i];
    __syncthreads();
    const int xx = blockIdx.x * kEdgePx + (int)threadIdx.x / kLanesPerPx, q = threadIdx.x % kLanesPerPx;
    const int ry = (H + kInRows - 1) / kInRows;
    const int bb = blockIdx.y / ry, y0 = (blockIdx.y - bb * ry) * kInRows;
    if (xx >= W) return;
    float w[9][8];
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
        const float4* w4 = reinterpret_cast<const float4*>(ws + tap * kC + 8 * q);
        const float4 wa = w4[0], wb = w4[1];
        w[tap][0] = wa.x;
        w[tap][1] = wa.y;
        w[tap][2] = wa.z;
        w[tap][3] = wa.w;
        w[tap][4] = wb.x;
        w[tap][5] = wb.y;
        w[tap][6] = wb.z;
        w[tap][7] = wb.w;
    }
    const float* xb = x + (size_t)bb * H * W;
    auto row3 = [&](int yy, float (&v)[3]) {
        const bool okr = yy >= 0 && yy < H;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++)
            v[dx + 1] = okr && xx + dx >= 0 && xx + dx < W ? __ldg(xb + (size_t)yy * W + xx + dx) : 0.f;
    };
    float win[3][3];
    row3(y0 - 1, win[0]);
    row3(y0, win[1]);
    const int y1 = min(H, y0 + kInRows);
    for (int yy = y0; yy < y1; yy++) {
        row3(yy + 1, win[2]);
        float s[8];
#pragma unroll
        for (int c = 0; c < 8; c++) s[c] = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            const float in = win[tap / 3][tap % 3];
#pragma unroll
            for (int c = 0; c < 8; c++) s[c] += w[tap][c] * in;
        }
        __align__(16) bf16 o[8];
#pragma unroll
        for (int c = 0; c < 8; c++) o[c] = __float2bfloat16_rn(fmaxf(s[c], 0.f));
        *reinterpret_cast<uint4*>(h1 + (((size_t)bb * H + yy) * W + xx) * kC + 8 * q) =
            *reinterpret_cast<const uint4*>(o);
#pragma unroll
        for (int e = 0; e < 3; e++) {
            win[0][e] = win[1][e];
            win[1][e] = win[2][e];
        }
    }
}

// last layer 32 -> 1: y = sum_tap sum_ci w6[ci][tap] h5[p + tap][ci]; lane q
// sums its eight channels over the taps, the four lanes' sums are added by
// two shuffles (lanes (0+1) + (2+3))
__global__ void __launch_bounds__(256)
k_conv_out(int B, int H, int W, const bf16* __restrict__ h5, const float* __restrict__ w6, float* __restrict__ y)
{
    __shared__ __align__(16) float ws[9 * kC];
    for (int i = threadIdx.x; i < kC * 9; i += blockDim.x) ws[(i % 9) * kC + i / 9] = w6[i];
    __syncthreads();
    const int row = blockIdx.y, yy = row % H;
    const int xx = blockIdx.x * kEdgePx + (int)threadIdx.x / kLanesPerPx, q = threadIdx.x % kLanesPerPx;
    const bool valid = xx < W;                      // every lane reaches the shuffles
    const bf16* hr = h5 + ((size_t)row * W + xx) * kC + 8 * q;
    float s = 0.f;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
        const bool okr = valid && yy + dy >= 0 && yy + dy < H;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            if (!(okr && xx + dx >= 0 && xx + dx < W)) continue;
            const int tap = (dy + 1) * 3 + dx + 1;
            const uint4 u = __ldg(reinterpret_cast<const uint4*>(hr + ((ptrdiff_t)dy * W + dx) * kC));
            const float4* w4 = reinterpret_cast<const float4*>(ws + tap * kC + 8 * q);
            const float4 wa = w4[0], wb = w4[1];
            const float wq[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
            const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float2 f = __bfloat1622float2(h2[e]);
                s += wq[2 * e] * f.x + wq[2 * e + 1] * f.y;
            }
        }
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (valid && q == 0) y[(size_t)row * W + xx] = s;
}

// y[p] = sum_t u[t][p + off_t] over the taps whose pixel lies in the image:
// the output layer after the fused projection (kFwdProj) of the last 32 -> 32
// layer.  One thread per pixel, one CTA row per image row.
__global__ void __launch_bounds__(256)
k_conv_taps(int B, int H, int W, const float* __restrict__ u, float* __restrict__ y)
{
    const int row = blockIdx.y, yy = row % H;
    const int xx = blockIdx.x * 256 + (int)threadIdx.x;
    if (xx >= W) return;
    const size_t npx = (size_t)B * H * W;
    const size_t p = (size_t)row * W + xx;
    float s = 0.f;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
        const bool okr = yy + dy >= 0 && yy + dy < H;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            if (!(okr && xx + dx >= 0 && xx + dx < W)) continue;
            const int t = (dy + 1) * 3 + dx + 1;
            s += __ldg(u + (size_t)t * npx + p + (ptrdiff_t)dy * W + dx);
        }
    }
    y[p] = s;
}

// JFEM_CNN_PROJ=0 keeps the separate output layer in inference forwards
bool cnn_proj_enabled()
{
    const char* e = getenv("JFEM_CNN_PROJ");
    return !(e && e[0] == '0');
}

// loss = mean (y - t)^2 (FP64 sum), dy = 2 (y - t) / N
struct VLoss {
    const float* y;
    const float* t;
    float* dy;
    float inv2n;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        float d = y[i] - t[i];
        dy[i] = d * inv2n;
        acc[0] += (double)d * d;
    }
};
struct FinLoss {
    double* out;
    double invn;
    __device__ void operator()(const double* s) const { *out = s[0] * invn; }
};

// dh5[p][ci] = sum_tap w6[ci][tap] dy[p - (tap - 4 offset)]  (input gradient of conv6)
__global__ void k_conv_out_bwd(int B, int H, int W, const float* __restrict__ dy, const float* __restrict__ w6,
                               float* __restrict__ dh5)
{
    __shared__ float ws[kC * 9];
    for (int i = threadIdx.x; i < kC * 9; i += blockDim.x) ws[i] = w6[i];
    __syncthreads();
    const size_t npx = (size_t)B * H * W;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(p % W), yy = (int)((p / W) % H);
        const size_t bb = p / ((size_t)H * W);
        float g9[9];
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            // dx[q] += w[tap] g[q - (dy-1, dx-1)]
            int gy = yy - (tap / 3 - 1), gx = xx - (tap % 3 - 1);
            g9[tap] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? dy[(bb * H + gy) * W + gx] : 0.f;
        }
        float* o = dh5 + p * kC;
#pragma unroll 4
        for (int ci = 0; ci < kC; ci++) {
            float s = 0.f;
#pragma unroll
            for (int tap = 0; tap < 9; tap++) s += ws[ci * 9 + tap] * g9[tap];
            o[ci] = s;
        }
    }
}

// weight gradients of the scalar-channel layers, per-CTA partials (32 x 9):
// MODE 0: dW1[co][tap] = sum_p g1[p][co] x[p + tap]
// MODE 1: dW6[ci][tap] = sum_p dy[p] h5[p + tap][ci]
template <int MODE>
__global__ void k_wgrad_edge(int B, int H, int W, const float* __restrict__ gc, const float* __restrict__ xs,
                             const bf16* __restrict__ hc, float* __restrict__ part)
{
    float acc[kC * 9];
#pragma unroll
    for (int i = 0; i < kC * 9; i++) acc[i] = 0.f;
    const size_t npx = (size_t)B * H * W;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(p % W), yy = (int)((p / W) % H);
        const size_t bb = p / ((size_t)H * W);
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            int gy = yy + tap / 3 - 1, gx = xx + tap % 3 - 1;
            if (gy < 0 || gy >= H || gx < 0 || gx >= W) continue;
            size_t q = (bb * H + gy) * W + gx;
            if (MODE == 0) {
                float xv = xs[q];
#pragma unroll
                for (int c = 0; c < kC; c++) acc[c * 9 + tap] += gc[p * kC + c] * xv;
            } else {
                float gv = xs[p];
#pragma unroll
                for (int c = 0; c < kC; c++) acc[c * 9 + tap] += gv * __bfloat162float(hc[q * kC + c]);
            }
        }
    }
    // block reduction (fixed order) of the 288 accumulators
    __shared__ float sh[kC * 9];
    for (int i = threadIdx.x; i < kC * 9; i += blockDim.x) sh[i] = 0.f;
    __syncthreads();
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        if ((int)(threadIdx.x >> 5) == w) {
#pragma unroll
            for (int i = 0; i < kC * 9; i++) {
                float v = warp_sum(acc[i]);
                if ((threadIdx.x & 31) == 0) sh[i] += v;
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kC * 9; i += blockDim.x) part[(size_t)blockIdx.x * kC * 9 + i] = sh[i];
}

__global__ void k_wgrad_edge_reduce(int nparts, const float* __restrict__ part, float* __restrict__ dw)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kC * 9) return;
    float s = 0.f;
    for (int p = 0; p < nparts; p++) s += part[(size_t)p * kC * 9 + i];
    dw[i] = s;
}

// g = d * (a > 0), and g16 = the same in BF16 when given (the TMA input of
// the tensor-core input-gradient convolution)
__global__ void k_relu_mask(size_t n, const float* __restrict__ d, const bf16* __restrict__ a, float* __restrict__ g,
                            bf16* __restrict__ g16)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = __bfloat162float(a[i]) > 0.f ? d[i] : 0.f;
        g[i] = v;
        if (g16) g16[i] = __float2bfloat16_rn(v);
    }
}

// BF16 weight layouts from the FP32 master (co, ci, dy, dx):
//   fwd: wk[l][co][tap*32 + ci]       bwd: wt[l][ci][tap'*32 + co] = w[co][ci][8 - tap']
__global__ void k_pack_weights(const float* __restrict__ w32, bf16* __restrict__ wk, bf16* __restrict__ wt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 4 * kMidParams) return;
    int l = i / kMidParams, r = i % kMidParams;
    const float* w = w32 + kLayerOff[1] + (size_t)l * kMidParams;
    int co = r / 288, k = r % 288, tap = k / 32, ci = k % 32;
    wk[i] = __float2bfloat16_rn(w[(co * kC + ci) * 9 + tap]);
    // transposed / flipped: row = ci', k' = tap'*32 + co'
    int ci2 = co, co2 = ci;   // reuse indices: r enumerates [ci][tap'*32 + co]
    wt[i] = __float2bfloat16_rn(w[(co2 * kC + ci2) * 9 + (8 - tap)]);
}

// Adam (FP32 master weights)
__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

void conv_mid_tc(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* in, const __nv_bfloat16* wk,
                 const __nv_bfloat16* skip, __nv_bfloat16* out, int* err);
void conv_mid_tc_bwd(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* gin, const __nv_bfloat16* wt,
                     const __nv_bfloat16* mask, const float* skip, float* out, __nv_bfloat16* out16, int* err);
bool conv_proj_available();
void conv_mid_tc_proj(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* in, const __nv_bfloat16* wk,
                      const __nv_bfloat16* skip, const float* w6, float* u, int* err);
int wgrad_mid_tc(cudaStream_t st, int B, int H, int W, const __nv_bfloat16* G16, const __nv_bfloat16* X,
                 float* part, int max_parts, int* err);
}  // namespace jfg

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct jfg_ctx;
namespace jfg {
cudaStream_t ctx_stream(jfg_ctx* ctx);
int ctx_device(jfg_ctx* ctx);
void ctx_set_error(jfg_ctx* ctx, const std::string& msg);
}  // namespace jfg

struct jfg_cnn {
    jfg_ctx* ctx = nullptr;
    jfg::DevBuf<float> w32, g32, m, v, part;
    jfg::DevBuf<__nv_bfloat16> wk, wt, h1, a2, h3, a4, h5;
    jfg::DevBuf<float> y, dy, gA, gB, gC;
    jfg::DevBuf<float> u9;                   // nine tap planes of the fused output projection (inference)
    jfg::DevBuf<__nv_bfloat16> gB16, gC16;   // BF16 copies of gB / gC: inputs of the tensor-core input gradients
    jfg::DevBuf<double> loss;
    jfg::DevBuf<double> partials;
    jfg::DevBuf<unsigned> counter;
    jfg::DevBuf<int> tc_err;        // set by the tensor-core convolution when an MMA wait timed out
    size_t cap = 0;
    int adam_t = 0;
    bool packed = false;
};

namespace jfg {
namespace {

constexpr int kEdgeCtas = 296;
constexpr int kMidWgradCtas = 296;

void cnn_reserve(jfg_cnn* n, size_t npx)
{
    if (npx <= n->cap) return;
    n->h1.alloc(npx * kC);
    n->a2.alloc(npx * kC);
    n->h3.alloc(npx * kC);
    n->a4.alloc(npx * kC);
    n->h5.alloc(npx * kC);
    n->y.alloc(npx);
    n->dy.alloc(npx);
    n->gA.alloc(npx * kC);
    n->gB.alloc(npx * kC);
    n->gC.alloc(npx * kC);
    n->gB16.alloc(npx * kC);
    n->gC16.alloc(npx * kC);
    n->u9.alloc(npx * 9);
    n->cap = npx;
}

void cnn_pack(jfg_cnn* n, cudaStream_t st)
{
    if (n->packed) return;
    k_pack_weights<<<(4 * kMidParams + 255) / 256, 256, 0, st>>>(n->w32.p, n->wk.p, n->wt.p);
    JFG_CUDA(cudaGetLastError());
    n->packed = true;
}

// synchronises the stream; a timed-out tensor-core wait becomes an error
void cnn_check_tc(jfg_cnn* n, cudaStream_t st)
{
    int h = 0;
    JFG_CUDA(cudaMemcpyAsync(&h, n->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    JFG_CHECK(h == 0, JFG_ERR_CUDA, "tensor-core convolution: an MMA wait timed out");
}

inline unsigned grid1d(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

template <typename InT, typename OutT, int SK, bool RELU, bool OMASK>
void conv_mid(cudaStream_t st, int B, int H, int W, const InT* in, const bf16* wk, const void* skip,
              const bf16* omask, OutT* out)
{
    dim3 grid((W + kTile - 1) / kTile, (H + kTile - 1) / kTile, B);
    k_conv_mid<InT, OutT, SK, RELU, OMASK><<<grid, 256, 0, st>>>(B, H, W, in, nullptr, wk, skip, omask, out);
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

bool use_tc();

// JFEM_CNN_WGRAD_TC=0 keeps the weight gradients on the mma.sync kernel
// when the tensor-core path is on
bool wgrad_tc_enabled()
{
    const char* e = getenv("JFEM_CNN_WGRAD_TC");
    return !(e && e[0] == '0');
}

// G16: the BF16 copy of G (the tensor-core path reads it; the mma.sync kernel
// rounds G to BF16 itself, so both contract the same values)
void wgrad_mid(jfg_cnn* n, cudaStream_t st, int B, int H, int W, const float* G, const bf16* G16, const bf16* X,
               float* dw)
{
    int ctas;
    if (G16 && use_tc() && wgrad_tc_enabled()) {
        ctas = wgrad_mid_tc(st, B, H, W, G16, X, n->part.p, kMidWgradCtas, n->tc_err.p);
    } else {
        int ntiles = ((W + kTile - 1) / kTile) * ((H + kTile - 1) / kTile) * B;
        ctas = std::min(ntiles, kMidWgradCtas);
        k_wgrad_mid<<<ctas, 288, 0, st>>>(B, H, W, G, X, n->part.p);
    }
    k_wgrad_mid_reduce<<<(kMidParams + 255) / 256, 256, 0, st>>>(ctas, n->part.p, dw);
    JFG_CUDA(cudaGetLastError());
    note_launch(2);
}

// The forward 32 -> 32 layers run on tcgen05 (jfg_cnn_tc.cu) unless
// JFEM_CNN_TC=0 selects the mma.sync kernels.
bool use_tc()
{
    const char* e = getenv("JFEM_CNN_TC");
    return !(e && e[0] == '0');
}

// keep_acts: training forwards keep every activation (h5 included) for the
// backward pass; inference forwards (keep_acts = false) fuse the output layer
// into the last tensor-core layer's epilogue (kFwdProj) when available.
void cnn_forward(jfg_cnn* n, cudaStream_t st, int B, int H, int W, const float* x, float* y, bool keep_acts = true)
{
    cnn_pack(n, st);
    const bf16* wk = n->wk.p;
    JFG_CHECK((size_t)B * H < 65536, JFG_ERR_UNSUPPORTED, "image batch too large (B * H >= 65536 rows)");
    const dim3 edge_grid((unsigned)((W + kEdgePx - 1) / kEdgePx), (unsigned)(B * H));
    const dim3 in_grid((unsigned)((W + kEdgePx - 1) / kEdgePx), (unsigned)(B * ((H + kInRows - 1) / kInRows)));
    k_conv_in<<<in_grid, 256, 0, st>>>(B, H, W, x, n->w32.p + kLayerOff[0], n->h1.p);
    JFG_CUDA(cudaGetLastError());
    if (use_tc()) {
        int* err = n->tc_err.p;
        conv_mid_tc(st, B, H, W, n->h1.p, wk + 0 * kMidParams, nullptr, n->a2.p, err);
        conv_mid_tc(st, B, H, W, n->a2.p, wk + 1 * kMidParams, n->h1.p, n->h3.p, err);
        conv_mid_tc(st, B, H, W, n->h3.p, wk + 2 * kMidParams, nullptr, n->a4.p, err);
        if (!keep_acts && cnn_proj_enabled() && conv_proj_available()) {
            conv_mid_tc_proj(st, B, H, W, n->a4.p, wk + 3 * kMidParams, n->h3.p, n->w32.p + kLayerOff[5], n->u9.p,
                             err);
            k_conv_taps<<<dim3((unsigned)((W + 255) / 256), (unsigned)(B * H)), 256, 0, st>>>(B, H, W, n->u9.p, y);
            JFG_CUDA(cudaGetLastError());
            note_launch(2);
            return;
        }
        conv_mid_tc(st, B, H, W, n->a4.p, wk + 3 * kMidParams, n->h3.p, n->h5.p, err);
    } else {
        conv_mid<bf16, bf16, 0, true, false>(st, B, H, W, n->h1.p, wk + 0 * kMidParams, nullptr, nullptr, n->a2.p);
        conv_mid<bf16, bf16, 1, true, false>(st, B, H, W, n->a2.p, wk + 1 * kMidParams, n->h1.p, nullptr,
                                             n->h3.p);
        conv_mid<bf16, bf16, 0, true, false>(st, B, H, W, n->h3.p, wk + 2 * kMidParams, nullptr, nullptr, n->a4.p);
        conv_mid<bf16, bf16, 1, true, false>(st, B, H, W, n->a4.p, wk + 3 * kMidParams, n->h3.p, nullptr,
                                             n->h5.p);
    }
    k_conv_out<<<edge_grid, 256, 0, st>>>(B, H, W, n->h5.p, n->w32.p + kLayerOff[5], y);
    JFG_CUDA(cudaGetLastError());
    note_launch(2);
}

// gradients of mean((y - t)^2) into n->g32 (forward activations must be current)
void cnn_backward(jfg_cnn* n, cudaStream_t st, int B, int H, int W, const float* x, const float* t)
{
    size_t npx = (size_t)B * H * W;
    JFG_CHECK(npx < (size_t)INT32_MAX, JFG_ERR_UNSUPPORTED, "too many pixels for one training batch");
    const bf16* wt = n->wt.p;
    float* g = n->g32.p;
    Scratch sc{n->partials.p, n->counter.p};
    vec_launch<1>(st, (int)npx, VLoss{n->y.p, t, n->dy.p, (float)(2.0 / npx)}, sc, nullptr,
                  FinLoss{n->loss.p, 1.0 / npx});
    k_wgrad_edge<1><<<kEdgeCtas, 256, 0, st>>>(B, H, W, nullptr, n->dy.p, n->h5.p, n->part.p);
    k_wgrad_edge_reduce<<<2, 256, 0, st>>>(kEdgeCtas, n->part.p, g + kLayerOff[5]);
    k_conv_out_bwd<<<grid1d(npx), 256, 0, st>>>(B, H, W, n->dy.p, n->w32.p + kLayerOff[5], n->gA.p);
    // input gradients on the tensor cores (BF16 copies of the gradient images
    // as their TMA inputs) unless JFEM_CNN_TC=0 selects the mma.sync kernels;
    // both round the gradient images to BF16 for the products
    const bool tc = use_tc();
    bf16* gB16 = tc ? n->gB16.p : nullptr;
    int* err = n->tc_err.p;
    k_relu_mask<<<grid1d(npx * kC), 256, 0, st>>>(npx * kC, n->gA.p, n->h5.p, n->gB.p, gB16);      // g5
    JFG_CUDA(cudaGetLastError());
    wgrad_mid(n, st, B, H, W, n->gB.p, gB16, n->a4.p, g + kLayerOff[4]);                            // dW5
    if (tc)
        conv_mid_tc_bwd(st, B, H, W, gB16, wt + 3 * kMidParams, n->a4.p, nullptr, n->gC.p, n->gC16.p, err);
    else
        conv_mid<float, float, 0, false, true>(st, B, H, W, n->gB.p, wt + 3 * kMidParams, nullptr, n->a4.p,
                                               n->gC.p);                                            // g4
    wgrad_mid(n, st, B, H, W, n->gC.p, tc ? n->gC16.p : nullptr, n->h3.p, g + kLayerOff[3]);     // dW4
    if (tc)
        conv_mid_tc_bwd(st, B, H, W, n->gC16.p, wt + 2 * kMidParams, nullptr, n->gB.p, n->gA.p, nullptr, err);
    else
        conv_mid<float, float, 2, false, false>(st, B, H, W, n->gC.p, wt + 2 * kMidParams, n->gB.p, nullptr,
                                                n->gA.p);                                           // dh3
    k_relu_mask<<<grid1d(npx * kC), 256, 0, st>>>(npx * kC, n->gA.p, n->h3.p, n->gB.p, gB16);      // g3
    wgrad_mid(n, st, B, H, W, n->gB.p, gB16, n->a2.p, g + kLayerOff[2]);                            // dW3
    if (tc)
        conv_mid_tc_bwd(st, B, H, W, gB16, wt + 1 * kMidParams, n->a2.p, nullptr, n->gC.p, n->gC16.p, err);
    else
        conv_mid<float, float, 0, false, true>(st, B, H, W, n->gB.p, wt + 1 * kMidParams, nullptr, n->a2.p,
                                               n->gC.p);                                            // g2
    wgrad_mid(n, st, B, H, W, n->gC.p, tc ? n->gC16.p : nullptr, n->h1.p, g + kLayerOff[1]);     // dW2
    if (tc)
        conv_mid_tc_bwd(st, B, H, W, n->gC16.p, wt + 0 * kMidParams, nullptr, n->gB.p, n->gA.p, nullptr, err);
    else
        conv_mid<float, float, 2, false, false>(st, B, H, W, n->gC.p, wt + 0 * kMidParams, n->gB.p, nullptr,
                                                n->gA.p);                                           // dh1
    k_relu_mask<<<grid1d(npx * kC), 256, 0, st>>>(npx * kC, n->gA.p, n->h1.p, n->gB.p, nullptr);   // g1
    k_wgrad_edge<0><<<kEdgeCtas, 256, 0, st>>>(B, H, W, n->gB.p, x, nullptr, n->part.p);
    k_wgrad_edge_reduce<<<2, 256, 0, st>>>(kEdgeCtas, n->part.p, g + kLayerOff[0]);
    JFG_CUDA(cudaGetLastError());
    note_launch(9);
}

}  // namespace
}  // namespace jfg

using jfg::DevBuf;

extern "C" {

int jfg_cnn_num_params(int* count)
{
    if (!count) return JFG_ERR_BAD_ARG;
    *count = jfg::kNumParams;
    return JFG_OK;
}

int jfg_cnn_create(jfg_ctx* ctx, jfg_cnn** out)
{
    if (!ctx || !out) return JFG_ERR_BAD_ARG;
    *out = nullptr;
    auto* n = new jfg_cnn();
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(ctx)));
        n->ctx = ctx;
        n->w32.alloc(jfg::kNumParams);
        n->g32.alloc(jfg::kNumParams);
        n->m.alloc(jfg::kNumParams);
        n->v.alloc(jfg::kNumParams);
        n->wk.alloc(4 * jfg::kMidParams);
        n->wt.alloc(4 * jfg::kMidParams);
        n->part.alloc((size_t)std::max(jfg::kMidWgradCtas * jfg::kMidParams, jfg::kEdgeCtas * jfg::kC * 9));
        n->loss.alloc(1);
        n->partials.alloc(4 * jfg::kVecGrid);
        n->counter.alloc(4);
        n->tc_err.alloc(1);
        cudaStream_t st = jfg::ctx_stream(ctx);
        JFG_CUDA(cudaMemsetAsync(n->tc_err.p, 0, sizeof(int), st));
        JFG_CUDA(cudaMemsetAsync(n->w32.p, 0, sizeof(float) * jfg::kNumParams, st));
        JFG_CUDA(cudaMemsetAsync(n->m.p, 0, sizeof(float) * jfg::kNumParams, st));
        JFG_CUDA(cudaMemsetAsync(n->v.p, 0, sizeof(float) * jfg::kNumParams, st));
        JFG_CUDA(cudaMemsetAsync(n->counter.p, 0, sizeof(unsigned) * 4, st));
        JFG_CUDA(cudaStreamSynchronize(st));
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(ctx, e.msg);
        delete n;
        return e.status;
    }
    *out = n;
    return JFG_OK;
}

int jfg_cnn_free(jfg_cnn* n)
{
    if (!n) return JFG_ERR_BAD_ARG;
    cudaStreamSynchronize(jfg::ctx_stream(n->ctx));
    delete n;
    return JFG_OK;
}

int jfg_cnn_set_weights(jfg_cnn* n, const float* h_w)
{
    if (!n || !h_w) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(n->ctx)));
        cudaStream_t st = jfg::ctx_stream(n->ctx);
        JFG_CUDA(cudaMemcpyAsync(n->w32.p, h_w, sizeof(float) * jfg::kNumParams, cudaMemcpyHostToDevice, st));
        JFG_CUDA(cudaMemsetAsync(n->m.p, 0, sizeof(float) * jfg::kNumParams, st));
        JFG_CUDA(cudaMemsetAsync(n->v.p, 0, sizeof(float) * jfg::kNumParams, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        n->adam_t = 0;
        n->packed = false;
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(n->ctx, e.msg);
        return e.status;
    }
}

int jfg_cnn_get_weights(jfg_cnn* n, float* h_w)
{
    if (!n || !h_w) return JFG_ERR_BAD_ARG;
    try {
        cudaStream_t st = jfg::ctx_stream(n->ctx);
        JFG_CUDA(cudaMemcpyAsync(h_w, n->w32.p, sizeof(float) * jfg::kNumParams, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(n->ctx, e.msg);
        return e.status;
    }
}

int jfg_cnn_forward_dev(jfg_cnn* n, int B, int H, int W, const float* d_x, float* d_y)
{
    if (!n || B < 1 || H < 1 || W < 1 || !d_x || !d_y) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(n->ctx)));
        cudaStream_t st = jfg::ctx_stream(n->ctx);
        jfg::cnn_reserve(n, (size_t)B * H * W);
        jfg::cnn_forward(n, st, B, H, W, d_x, d_y, false);
        jfg::cnn_check_tc(n, st);
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(n->ctx, e.msg);
        return e.status;
    }
}

int jfg_cnn_loss_grad_dev(jfg_cnn* n, int B, int H, int W, const float* d_x, const float* d_t, double* loss,
                          float* h_grad)
{
    if (!n || B < 1 || H < 1 || W < 1 || !d_x || !d_t) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(n->ctx)));
        cudaStream_t st = jfg::ctx_stream(n->ctx);
        jfg::cnn_reserve(n, (size_t)B * H * W);
        jfg::cnn_forward(n, st, B, H, W, d_x, n->y.p);
        jfg::cnn_backward(n, st, B, H, W, d_x, d_t);
        if (loss) JFG_CUDA(cudaMemcpyAsync(loss, n->loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        if (h_grad)
            JFG_CUDA(cudaMemcpyAsync(h_grad, n->g32.p, sizeof(float) * jfg::kNumParams, cudaMemcpyDeviceToHost, st));
        jfg::cnn_check_tc(n, st);
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(n->ctx, e.msg);
        return e.status;
    }
}

int jfg_cnn_adam_step(jfg_cnn* n, double lr, double beta1, double beta2, double eps)
{
    if (!n || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0))
        return JFG_ERR_BAD_ARG;
    try {
        cudaStream_t st = jfg::ctx_stream(n->ctx);
        n->adam_t++;
        float c1 = (float)(1.0 - std::pow(beta1, n->adam_t)), c2 = (float)(1.0 - std::pow(beta2, n->adam_t));
        jfg::k_adam<<<(jfg::kNumParams + 255) / 256, 256, 0, st>>>(jfg::kNumParams, n->w32.p, n->g32.p, n->m.p,
                                                                    n->v.p, (float)lr, (float)beta1, (float)beta2,
                                                                    (float)eps, c1, c2);
        JFG_CUDA(cudaGetLastError());
        jfg::note_launch();
        n->packed = false;
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(n->ctx, e.msg);
        return e.status;
    }
}

int jfg_cnn_time_forward(jfg_cnn* n, int B, int H, int W, int iters, double* ms_total, double* ms_mid)
{
    if (!n || B < 1 || H < 1 || W < 1 || iters < 1 || !ms_total) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(n->ctx)));
        cudaStream_t st = jfg::ctx_stream(n->ctx);
        size_t npx = (size_t)B * H * W;
        jfg::cnn_reserve(n, npx);
        DevBuf<float> x;
        x.alloc(npx);
        JFG_CUDA(cudaMemsetAsync(x.p, 0, sizeof(float) * npx, st));
        cudaEvent_t e0, e1, e2;
        JFG_CUDA(cudaEventCreate(&e0));
        JFG_CUDA(cudaEventCreate(&e1));
        JFG_CUDA(cudaEventCreate(&e2));
        jfg::cnn_forward(n, st, B, H, W, x.p, n->y.p, false);
        JFG_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < iters; i++) jfg::cnn_forward(n, st, B, H, W, x.p, n->y.p, false);
        JFG_CUDA(cudaEventRecord(e1, st));
        const bool tc = jfg::use_tc();
        for (int i = 0; i < iters; i++) {
            if (tc)
                jfg::conv_mid_tc(st, B, H, W, n->h1.p, n->wk.p, nullptr, n->a2.p, n->tc_err.p);
            else
                jfg::conv_mid<__nv_bfloat16, __nv_bfloat16, 0, true, false>(st, B, H, W, n->h1.p, n->wk.p, nullptr,
                                                                             nullptr, n->a2.p);
        }
        JFG_CUDA(cudaEventRecord(e2, st));
        JFG_CUDA(cudaEventSynchronize(e2));
        jfg::cnn_check_tc(n, st);
        float t1 = 0, t2 = 0;
        JFG_CUDA(cudaEventElapsedTime(&t1, e0, e1));
        JFG_CUDA(cudaEventElapsedTime(&t2, e1, e2));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        *ms_total = t1 / iters;
        if (ms_mid) *ms_mid = t2 / iters;
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(n->ctx, e.msg);
        return e.status;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// FP32 V-cycle followed by the learned smoother (a preconditioner for FGMRES)
// ---------------------------------------------------------------------------
struct jfg_mat;
namespace jfg {
Matrix* mat_of(jfg_mat* m);
jfg_ctx* mat_ctx(jfg_mat* m);
}  // namespace jfg

struct jfg_mgcnn {
    jfg_ctx* ctx = nullptr;
    jfg_mg* mg = nullptr;
    jfg_cnn* net = nullptr;
    jfg::Matrix* A = nullptr;
    int H = 0, W = 0, n = 0, use_net = 1;
    double out_scale = 1.0;
    uint64_t uid = jfg::next_uid();
    jfg::DevBuf<int> dof;
    jfg::DevBuf<unsigned char> bd;
    jfg::DevBuf<float> r32, z32, img_in, img_out;
    jfg::DevBuf<double> rp, scale;
    jfg::DevBuf<double> partials;     // scratch of jfg_mgcnn_apply_dev
    jfg::DevBuf<unsigned> counter;
};

namespace jfg {
namespace {

struct FinRms {   // scale = rms of the vector (1 when it is zero)
    double* scale;
    double invn;
    __device__ void operator()(const double* s) const
    {
        double r = sqrt(s[0] * invn);
        *scale = r > 0 ? r : 1.0;
    }
};

struct EpiResidJac {   // y = b - A x, acc += (y / diag)^2 (zero diagonals count as 1)
    const double* b;
    const double* diag;
    double* y;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&acc)[K]) const
    {
        double v = b[r] - (double)s;
        y[r] = v;
        double d = diag[r];
        double q = v / (d != 0.0 ? d : 1.0);
        acc[0] += q * q;
    }
};

__global__ void k_gather_img(int npix, const int* __restrict__ dof, const double* __restrict__ r,
                             const double* __restrict__ diag, const double* __restrict__ scale,
                             float* __restrict__ img)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    int d = dof[i];
    double dg = diag[d];
    img[i] = (float)(r[d] / (dg != 0.0 ? dg : 1.0) / *scale);
}

__global__ void k_scatter_img(int npix, const int* __restrict__ dof, const unsigned char* __restrict__ bd,
                              const float* __restrict__ img, const double* __restrict__ scale, double out_scale,
                              double* __restrict__ z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    int d = dof[i];
    if (bd[d]) return;
    z[d] += (double)img[i] * (*scale) * out_scale;
}

void mgcnn_apply(void* self, const double* v, double* z, const Scratch& sc, const int* done, cudaStream_t st)
{
    auto* p = static_cast<jfg_mgcnn*>(self);
    const int n = p->n;
    vec_launch<0>(st, n, VCast<double, float>{v, p->r32.p}, sc, done);
    p->mg->fp32()->apply(p->r32.p, p->z32.p, sc, done, st);
    vec_launch<0>(st, n, VCast<float, double>{p->z32.p, z}, sc, done);
    if (!p->use_net) return;
    spmv_launch<double, double, 1>(st, p->A, p->A->val.p, z, EpiResidJac{v, p->A->diag.p, p->rp.p}, sc, done,
                                   FinRms{p->scale.p, 1.0 / n});
    const int npix = p->H * p->W;
    k_gather_img<<<(npix + 255) / 256, 256, 0, st>>>(npix, p->dof.p, p->rp.p, p->A->diag.p, p->scale.p,
                                                      p->img_in.p);
    // repack the BF16 weights every application: a replayed graph then always
    // sees the current master weights
    k_pack_weights<<<(4 * kMidParams + 255) / 256, 256, 0, st>>>(p->net->w32.p, p->net->wk.p, p->net->wt.p);
    p->net->packed = true;
    JFG_CUDA(cudaGetLastError());
    note_launch(2);
    cnn_forward(p->net, st, 1, p->H, p->W, p->img_in.p, p->img_out.p, false);
    k_scatter_img<<<(npix + 255) / 256, 256, 0, st>>>(npix, p->dof.p, p->bd.p, p->img_out.p, p->scale.p,
                                                       p->out_scale, z);
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

}  // namespace

// Fills a Precond<double> with the mgcnn hook; returns the largest SpMV grid.
int mgcnn_precond(void* h, Precond<double>& P, int n)
{
    auto* p = static_cast<jfg_mgcnn*>(h);
    JFG_CHECK(p && p->n == n, JFG_ERR_BAD_ARG, "multigrid + network preconditioner does not match the system size");
    P.kind = JFG_PREC_MG_CNN;
    P.hook = mgcnn_apply;
    P.hook_self = p;
    P.hook_uid = p->uid;
    P.mg = nullptr;
    P.n = n;
    return std::max(p->mg->fp32()->max_blocks(), p->A->nblocks);
}

}  // namespace jfg

extern "C" {

int jfg_mgcnn_create(jfg_ctx* ctx, jfg_mg* mg, jfg_cnn* net, jfg_mat* A, int H, int W, const int* h_dof_of_pixel,
                     const int* h_bdry, int n_bdry, double out_scale, int use_net, jfg_mgcnn** out)
{
    if (!ctx || !mg || !net || !A || !out || H < 1 || W < 1 || !h_dof_of_pixel || n_bdry < 0 ||
        (n_bdry > 0 && !h_bdry))
        return JFG_ERR_BAD_ARG;
    *out = nullptr;
    auto* p = new jfg_mgcnn();
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(ctx)));
        cudaStream_t st = jfg::ctx_stream(ctx);
        jfg::Matrix* M = jfg::mat_of(A);
        JFG_CHECK(jfg::mat_ctx(A) == ctx, JFG_ERR_BAD_ARG, "matrix from another context");
        JFG_CHECK(M->rows == M->cols, JFG_ERR_BAD_ARG, "matrix is not square");
        int n = M->rows;
        JFG_CHECK((int64_t)H * W == n, JFG_ERR_BAD_ARG, "H * W must equal the number of unknowns");
        JFG_CHECK(mg->d64 && mg->d64->n[mg->levels - 1] == n, JFG_ERR_BAD_ARG,
                  "multigrid hierarchy does not match the matrix");
        for (int i = 0; i < n; i++)
            JFG_CHECK(h_dof_of_pixel[i] >= 0 && h_dof_of_pixel[i] < n, JFG_ERR_BAD_ARG, "pixel map out of range");
        for (int i = 0; i < n_bdry; i++)
            JFG_CHECK(h_bdry[i] >= 0 && h_bdry[i] < n, JFG_ERR_BAD_ARG, "boundary node out of range");
        p->ctx = ctx;
        p->mg = mg;
        p->net = net;
        p->A = M;
        p->H = H;
        p->W = W;
        p->n = n;
        p->use_net = use_net ? 1 : 0;
        p->out_scale = out_scale;
        mg->fp32();
        p->dof.alloc(n);
        p->bd.alloc(n);
        p->r32.alloc(n);
        p->z32.alloc(n);
        p->img_in.alloc(n);
        p->img_out.alloc(n);
        p->rp.alloc(n);
        p->scale.alloc(1);
        std::vector<unsigned char> hb(n, 0);
        for (int i = 0; i < n_bdry; i++) hb[h_bdry[i]] = 1;
        JFG_CUDA(cudaMemcpyAsync(p->dof.p, h_dof_of_pixel, sizeof(int) * n, cudaMemcpyHostToDevice, st));
        JFG_CUDA(cudaMemcpyAsync(p->bd.p, hb.data(), n, cudaMemcpyHostToDevice, st));
        jfg::cnn_reserve(net, (size_t)n);
        int mb = std::max(std::max(mg->fp32()->max_blocks(), M->nblocks), jfg::kVecGrid);
        p->partials.alloc((size_t)4 * mb);
        p->counter.alloc(4);
        JFG_CUDA(cudaMemsetAsync(p->counter.p, 0, 4 * sizeof(unsigned), st));
        JFG_CUDA(cudaStreamSynchronize(st));
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(ctx, e.msg);
        delete p;
        return e.status;
    }
    *out = p;
    return JFG_OK;
}

int jfg_mgcnn_set(jfg_mgcnn* p, double out_scale, int use_net)
{
    if (!p || !std::isfinite(out_scale)) return JFG_ERR_BAD_ARG;
    p->out_scale = out_scale;
    p->use_net = use_net ? 1 : 0;
    p->uid = jfg::next_uid();     // graphs captured with the old settings are not reused
    return JFG_OK;
}

int jfg_mgcnn_apply_dev(jfg_mgcnn* p, const double* d_v, double* d_z)
{
    if (!p || !d_v || !d_z) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(p->ctx)));
        cudaStream_t st = jfg::ctx_stream(p->ctx);
        jfg::Scratch sc{p->partials.p, p->counter.p};
        jfg::mgcnn_apply(p, d_v, d_z, sc, nullptr, st);
        JFG_CUDA(cudaStreamSynchronize(st));
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(p->ctx, e.msg);
        return e.status;
    }
}

int jfg_mgcnn_free(jfg_mgcnn* p)
{
    if (!p) return JFG_ERR_BAD_ARG;
    cudaStreamSynchronize(jfg::ctx_stream(p->ctx));
    delete p;
    return JFG_OK;
}

}  // extern "C"
