// Block-diagonal preconditioner of a saddle-point system on the device:
//   z[0, nv)      = V(r[0, nv))          a velocity multigrid application (FP64, or FP32 V-cycle)
//   z[nv, nv+np)  = pinv * r[nv, nv+np)  a diagonal pressure block (lumped pressure-mass inverse)
// The velocity unknowns come first, so both blocks are contiguous slices of
// the Krylov vectors and need no gather.
#include "jfg_krylov.cuh"

struct jfg_blockdiag {
    jfg_ctx* ctx = nullptr;
    jfg_mg* mg = nullptr;
    int nv = 0, np = 0, fp32 = 0;
    uint64_t uid = jfg::next_uid();
    jfg::DevBuf<double> pinv;
    jfg::DevBuf<float> r32, z32;
    jfg::DevBuf<double> partials;
    jfg::DevBuf<unsigned> counter;
};

namespace jfg {
cudaStream_t ctx_stream(jfg_ctx* ctx);
int ctx_device(jfg_ctx* ctx);
void ctx_set_error(jfg_ctx* ctx, const std::string& msg);

namespace {

__global__ void k_diag_scale(int n, const double* __restrict__ d, const double* __restrict__ r, double* __restrict__ z,
                             const int* done)
{
    if (done && *done) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = d[i] * r[i];
}

void blockdiag_apply(void* self, const double* r, double* z, const Scratch& sc, const int* done, cudaStream_t st)
{
    auto* b = static_cast<jfg_blockdiag*>(self);
    if (b->fp32) {
        vec_launch<0>(st, b->nv, VCast<double, float>{r, b->r32.p}, sc, done);
        b->mg->fp32()->apply(b->r32.p, b->z32.p, sc, done, st);
        vec_launch<0>(st, b->nv, VCast<float, double>{b->z32.p, z}, sc, done);
    } else {
        b->mg->d64->apply(r, z, sc, done, st);
    }
    if (b->np > 0) {
        const int grid = std::min((b->np + 255) / 256, 148 * 8);
        k_diag_scale<<<grid, 256, 0, st>>>(b->np, b->pinv.p, r + b->nv, z + b->nv, done);
        JFG_CUDA(cudaGetLastError());
        note_launch();
    }
}

}  // namespace

int blockdiag_precond(void* h, Precond<double>& P, int n)
{
    auto* b = static_cast<jfg_blockdiag*>(h);
    JFG_CHECK(b && b->nv + b->np == n, JFG_ERR_BAD_ARG, "block preconditioner does not match the system size");
    P.kind = JFG_PREC_BLOCKDIAG;
    P.hook = blockdiag_apply;
    P.hook_self = b;
    P.hook_uid = b->uid;
    P.n = n;
    return b->fp32 ? b->mg->fp32()->max_blocks() : b->mg->d64->max_blocks();
}

}  // namespace jfg

extern "C" {

int jfg_blockdiag_create(jfg_ctx* ctx, jfg_mg* mg, int nv, int np, const double* h_pinv, int fp32_vcycle,
                         jfg_blockdiag** out)
{
    if (!ctx || !mg || !out || nv < 1 || np < 0 || (np > 0 && !h_pinv)) return JFG_ERR_BAD_ARG;
    *out = nullptr;
    auto* b = new jfg_blockdiag();
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(ctx)));
        cudaStream_t st = jfg::ctx_stream(ctx);
        JFG_CHECK(mg->d64 && mg->d64->n[mg->levels - 1] == nv, JFG_ERR_BAD_ARG,
                  "velocity multigrid does not match the velocity block size");
        b->ctx = ctx;
        b->mg = mg;
        b->nv = nv;
        b->np = np;
        b->fp32 = fp32_vcycle ? 1 : 0;
        b->pinv.alloc(std::max(np, 1));
        if (np > 0) JFG_CUDA(cudaMemcpyAsync(b->pinv.p, h_pinv, sizeof(double) * np, cudaMemcpyHostToDevice, st));
        if (b->fp32) {
            mg->fp32();
            b->r32.alloc(nv);
            b->z32.alloc(nv);
        }
        int mb = std::max(b->fp32 ? mg->fp32()->max_blocks() : mg->d64->max_blocks(), jfg::kVecGrid);
        b->partials.alloc((size_t)4 * mb);
        b->counter.alloc(4);
        JFG_CUDA(cudaMemsetAsync(b->counter.p, 0, 4 * sizeof(unsigned), st));
        JFG_CUDA(cudaStreamSynchronize(st));
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(ctx, e.msg);
        delete b;
        return e.status;
    }
    *out = b;
    return JFG_OK;
}

int jfg_blockdiag_apply(jfg_blockdiag* b, const double* h_v, double* h_out)
{
    if (!b || !h_v || !h_out) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(b->ctx)));
        cudaStream_t st = jfg::ctx_stream(b->ctx);
        const int n = b->nv + b->np;
        jfg::DevBuf<double> v, z;
        v.alloc(n);
        z.alloc(n);
        JFG_CUDA(cudaMemcpyAsync(v.p, h_v, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        jfg::Scratch sc{b->partials.p, b->counter.p};
        jfg::blockdiag_apply(b, v.p, z.p, sc, nullptr, st);
        JFG_CUDA(cudaMemcpyAsync(h_out, z.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        return JFG_OK;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(b->ctx, e.msg);
        return e.status;
    }
}

int jfg_blockdiag_free(jfg_blockdiag* b)
{
    if (!b) return JFG_ERR_BAD_ARG;
    cudaStreamSynchronize(jfg::ctx_stream(b->ctx));
    delete b;
    return JFG_OK;
}

}  // extern "C"
