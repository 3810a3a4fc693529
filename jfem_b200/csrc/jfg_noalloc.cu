// CG on caller-owned device CSR arrays without any device allocation.
//
// Some callers cannot allocate device memory at the moment they solve: a host
// framework that owns the device heap (a memory pool or budget that the
// library must not grow or fragment), or a real-time loop that cannot afford
// the latency and implicit synchronisation of cudaMalloc/cudaFree.  For them
// this file offers jfg_cg_noalloc: the same CG iteration as
// jfg_solve_dev(JFG_CG, ...) (IterativeSolver.solveCG semantics: start iterate
// taken from x, absolute tolerance, iteration cap), but every work vector,
// the reduction partials and the control block live in one file-scope
// __device__ array of fixed size.  The caller passes the matrix (CSR), the
// right-hand side and the iterate as device pointers.
//
// The call runs eagerly on the context's stream and synchronises the host
// with it: every 8 iterations it reads the device convergence flag back.
//
// The array is a single process-wide resource per GPU: every call shares it
// and it keeps the contents of the last call.  Calls that overlap on the GPU
// (two streams, two host threads) race on it.  The first call on a device
// looks up the array's device address (cudaGetSymbolAddress) with that
// device current and caches it for the rest of the process; the cache
// assumes the runtime's primary context of that device stays the same for
// the process lifetime (no cudaDeviceReset in between).
#include <cmath>
#include <cstring>
#include <mutex>

#include "jfg_ops.cuh"

namespace {

using namespace jfg;

constexpr int kNoAllocMaxRows = 1 << 18;   // 262,144 unknowns
constexpr size_t kCtlBytes = 256;
constexpr size_t kCounterBytes = 256;
constexpr size_t kPartialBytes = sizeof(double) * 2 * kVecGrid;
constexpr size_t kVecBytes = sizeof(double) * kNoAllocMaxRows;
constexpr size_t kScratchBytes = kCtlBytes + kCounterBytes + ((kPartialBytes + 255) / 256) * 256 + 3 * kVecBytes;
static_assert(sizeof(Ctl) <= kCtlBytes, "control block does not fit its slot");

// ~6.3 MB per GPU that loads the library, held until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct ScratchLayout {
    Ctl* ctl;
    unsigned* counter;
    double* partials;
    double* r;
    double* p;
    double* Ap;
};

std::mutex g_setup_mutex;
void* g_scratch_addr[128] = {nullptr};

// Device address of the scratch array on the current device (looked up once).
ScratchLayout scratch_for_device(int device)
{
    JFG_CHECK(device >= 0 && device < 128, JFG_ERR_BAD_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            throw Error{JFG_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e)};
        g_scratch_addr[device] = ptr;
    }
    unsigned char* base = static_cast<unsigned char*>(g_scratch_addr[device]);
    ScratchLayout L;
    L.ctl = reinterpret_cast<Ctl*>(base);
    L.counter = reinterpret_cast<unsigned*>(base + kCtlBytes);
    L.partials = reinterpret_cast<double*>(base + kCtlBytes + kCounterBytes);
    unsigned char* vec = base + kCtlBytes + kCounterBytes + ((kPartialBytes + 255) / 256) * 256;
    L.r = reinterpret_cast<double*>(vec);
    L.p = reinterpret_cast<double*>(vec + kVecBytes);
    L.Ap = reinterpret_cast<double*>(vec + 2 * kVecBytes);
    return L;
}

// One thread per CSR row (row sums in column order).
template <int NR, class Epi, class Fin>
__global__ void __launch_bounds__(kThreads)
k_csr_spmv(int n, const int* __restrict__ ptr, const int* __restrict__ col, const double* __restrict__ val,
           const double* __restrict__ x, Epi epi, GridRed<NR, Fin> red, const int* __restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int i = 0; i < (NR > 0 ? NR : 1); i++) acc[i] = 0;
    for (int r = blockIdx.x * kThreads + threadIdx.x; r < n; r += gridDim.x * kThreads) {
        double s = 0;
        for (int k = __ldg(ptr + r); k < __ldg(ptr + r + 1); k++) s += __ldg(val + k) * __ldg(x + __ldg(col + k));
        epi(r, s, acc);
    }
    pdl_launch_dependents();
    if constexpr (NR > 0) red.reduce(acc);
}

__device__ void nc_check(Ctl* c, double rn)
{
    c->res_norm = rn;
    if (!isfinite(rn)) {
        c->done = 1;
        c->status = JFG_NONFINITE;
    } else if (!(rn > c->tol)) {
        c->done = 1;
        c->status = JFG_OK;
    } else if (c->iter >= c->maxit) {
        c->done = 1;
        c->status = JFG_NOT_CONVERGED;
    }
}
struct NcInit {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->rr = t[0];
        nc_check(c, sqrt(t[0]));
    }
};
struct NcAlpha {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->alpha = c->rr / t[0];
        if (!(t[0] > 0)) c->not_pd = 1;
    }
};
struct NcUpdate {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->iter++;
        c->beta = t[0] / c->rr;
        c->rr = t[0];
        nc_check(c, sqrt(t[0]));
    }
};
struct VNcUpdate {   // x += p*alpha; r = r - Ap*alpha; acc += r^2
    double* x;
    const double* p;
    double* r;
    const double* Ap;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        double a = c->alpha;
        x[i] = x[i] + p[i] * a;
        double rn = r[i] - Ap[i] * a;
        r[i] = rn;
        acc[0] += rn * rn;
    }
};
struct NcReset {     // the array keeps the previous call's contents: a fresh control block
    Ctl* c;
    double tol;
    int maxit, n;
    __device__ void operator()() const
    {
        Ctl h{};
        h.tol = tol;
        h.maxit = maxit;
        h.n = n;
        h.status = JFG_NOT_CONVERGED;
        *c = h;
    }
};
struct VNcDir {      // p = r + p*beta
    const double* r;
    double* p;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { p[i] = r[i] + p[i] * c->beta; }
};

template <int NR, class Epi, class Fin>
void csr_launch(cudaStream_t st, int n, const int* ptr, const int* col, const double* val, const double* x, Epi epi,
                const Scratch& sc, const int* done, Fin fin)
{
    GridRed<NR, Fin> red{sc.partials, sc.counter, fin};
    launch_ex(k_csr_spmv<NR, Epi, Fin>, dim3(vec_grid(n)), dim3(kThreads), 0, st, n, ptr, col, val, x, epi, red,
              done);
}

}  // namespace

struct jfg_ctx;
namespace jfg {
// implemented in jfg_api.cu: the context's stream/device and error channel
cudaStream_t ctx_stream(jfg_ctx* ctx);
int ctx_device(jfg_ctx* ctx);
void ctx_set_error(jfg_ctx* ctx, const std::string& msg);
}  // namespace jfg

extern "C" int jfg_cg_noalloc(jfg_ctx* ctx, int n, const int* d_rowptr, const int* d_col, const double* d_val,
                              const double* d_b, double* d_x, double tol, int maxit, int* iterations,
                              double* final_norm)
{
    if (!ctx) return JFG_ERR_BAD_ARG;
    try {
        JFG_CUDA(cudaSetDevice(jfg::ctx_device(ctx)));
        JFG_CHECK(n >= 0, JFG_ERR_BAD_ARG, "negative system size");
        JFG_CHECK(n <= kNoAllocMaxRows, JFG_ERR_BAD_ARG,
                  "jfg_cg_noalloc: system size " + std::to_string(n) + " exceeds the fixed scratch limit of " +
                      std::to_string(kNoAllocMaxRows) + " unknowns");
        JFG_CHECK(n == 0 || (d_rowptr && d_col && d_val && d_b && d_x), JFG_ERR_BAD_ARG, "null device pointer");
        JFG_CHECK(tol >= 0 && std::isfinite(tol), JFG_ERR_BAD_ARG, "bad tolerance");
        cudaStream_t st = jfg::ctx_stream(ctx);
        ScratchLayout L = scratch_for_device(jfg::ctx_device(ctx));
        if (maxit <= 0) maxit = n;
        // the array keeps the previous call's contents: reset the reduction
        // counter and the control block on the device
        JFG_CUDA(cudaMemsetAsync(L.counter, 0, kCounterBytes, st));
        scalar_launch(st, NcReset{L.ctl, tol, maxit, n}, nullptr);
        int it = 0;
        double rn = 0;
        if (n > 0) {
            Scratch sc{L.partials, L.counter};
            const int* done = &L.ctl->done;
            csr_launch<1>(st, n, d_rowptr, d_col, d_val, d_x, EpiResid<double>{d_b, L.r}, sc, nullptr, NcInit{L.ctl});
            vec_launch<0>(st, n, VCopy<double>{L.r, L.p}, sc, done);
            int h_done = 0;
            while (!h_done) {
                for (int k = 0; k < 8; k++) {
                    csr_launch<1>(st, n, d_rowptr, d_col, d_val, L.p, EpiStoreDot<double>{L.Ap, L.p}, sc, done,
                                  NcAlpha{L.ctl});
                    vec_launch<1>(st, n, VNcUpdate{d_x, L.p, L.r, L.Ap, L.ctl}, sc, done, NcUpdate{L.ctl});
                    vec_launch<0>(st, n, VNcDir{L.r, L.p, L.ctl}, sc, done);
                }
                JFG_CUDA(cudaMemcpyAsync(&h_done, done, sizeof(int), cudaMemcpyDeviceToHost, st));
                JFG_CUDA(cudaStreamSynchronize(st));
            }
        }
        Ctl out;
        JFG_CUDA(cudaMemcpyAsync(&out, L.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        it = out.iter;
        rn = out.res_norm;
        if (iterations) *iterations = it;
        if (final_norm) *final_norm = rn;
        if (n > 0 && out.not_pd)   // the same condition jfg_solve_dev reports in jfg_solve_info.not_pd
            jfg::ctx_set_error(ctx, "jfg_cg_noalloc: p.Ap <= 0 met (matrix not positive definite)");
        return n == 0 ? JFG_OK : out.status;
    } catch (const jfg::Error& e) {
        jfg::ctx_set_error(ctx, e.msg);
        return e.status;
    } catch (...) {
        jfg::ctx_set_error(ctx, "unknown error");
        return JFG_ERR_CUDA;
    }
}
