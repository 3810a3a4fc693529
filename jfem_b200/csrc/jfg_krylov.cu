// Krylov iterations on the device: CG / PCG (IterativeSolver.java:48-162),
// BiCGStab / PBiCGStab (:256-402), restarted GMRES with Givens rotations
// (GMRES.java:40-251), and the FP64 defect-correction outer loop around FP32
// inner solves.  Every scalar lives in the device control block (Ctl); every
// reduction is a deterministic last-block grid reduction whose finaliser
// updates the control block, so one iteration is a fixed kernel sequence.
#include <cmath>

#include "jfg_krylov.cuh"

namespace jfg {

namespace {

// ---------------------------------------------------------------------------
// control-block helpers (single thread)
// ---------------------------------------------------------------------------
__device__ void publish(Ctl* c, double rn)
{
    c->res_norm = rn;
    if (c->hist && c->iter >= 1 && c->iter <= c->hist_cap) c->hist[c->iter - 1] = rn;
}
// the loop test `iter < maxit && ||r|| > tol` (IterativeSolver.java:78, 139, 290, 366)
__device__ void check(Ctl* c, double rn)
{
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

struct FinInit {     // r = b - A x done: rr
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->rr = t[0];
        c->rz = t[0];
        check(c, sqrt(t[0]));
        c->res_norm = sqrt(t[0]);
    }
};
struct FinRZ {       // rz = r . z
    Ctl* c;
    __device__ void operator()(const double* t) const { c->rz = t[0]; }
};
struct FinAlpha {    // alpha = rz / p.Ap
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->pAp = t[0];
        c->alpha = c->rz / t[0];
        if (!(t[0] > 0)) c->not_pd = 1;
    }
};
struct FinCGRes {    // after x += alpha p, r -= alpha Ap: t = ||r||^2
    Ctl* c;
    int pcg;
    __device__ void operator()(const double* t) const
    {
        c->iter++;
        if (!pcg) {
            c->beta = t[0] / c->rr;
            c->rz = t[0];
        }
        c->rr = t[0];
        publish(c, sqrt(t[0]));
        check(c, sqrt(t[0]));
    }
};
struct FinBeta {     // beta = r'.z' / r.z
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->beta = t[0] / c->rz;
        c->rz = t[0];
    }
};

// ---------------------------------------------------------------------------
// vector functors of the iterations
// ---------------------------------------------------------------------------
template <typename T>
struct VCGUpdate {   // x += p*alpha; r = r - Ap*alpha; acc += r^2
    T* x;
    const T* p;
    T* r;
    const T* Ap;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        T a = (T)c->alpha;
        x[i] = x[i] + p[i] * a;
        T rn = r[i] - Ap[i] * a;
        r[i] = rn;
        acc[0] += (double)rn * (double)rn;
    }
};
template <typename T>
struct VXpby {       // p = z + p*beta
    const T* z;
    T* p;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { p[i] = z[i] + p[i] * (T)c->beta; }
};
// FP64 PCG with an FP32 multigrid preconditioner: the r -> FP32 copy is
// written by the update kernel and z is consumed in FP32 (widened exactly
// inside the dot and the direction update), which gives bit-identical
// iterates without two cast kernels and the FP64 z vector per iteration.
struct VCGUpdate32 {  // VCGUpdate<double> and r32 = (float) r
    double* x;
    const double* p;
    double* r;
    const double* Ap;
    float* r32;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        double a = c->alpha;
        x[i] = x[i] + p[i] * a;
        double rn = r[i] - Ap[i] * a;
        r[i] = rn;
        r32[i] = (float)rn;
        acc[0] += rn * rn;
    }
};
struct VDotMixed {    // acc += r . (double) z32
    const double* r;
    const float* z;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const { acc[0] += r[i] * (double)z[i]; }
};
struct VXpby32 {      // p = (double) z32 + p * beta
    const float* z;
    double* p;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { p[i] = (double)z[i] + p[i] * c->beta; }
};

template <typename T>
struct VJacobiPre {  // z = dinv * r
    const T* d;
    const T* r;
    T* z;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { z[i] = d[i] * r[i]; }
};

template <typename T>
struct VCopyNorm {   // b = a, acc += a^2
    const T* a;
    T* b;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        T v = a[i];
        b[i] = v;
        acc[0] += (double)v * (double)v;
    }
};
template <typename T>
struct VNorm2 {
    const T* a;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const { acc[0] += (double)a[i] * (double)a[i]; }
};

// BiCGStab pieces (IterativeSolver.java:290-318)
struct FinRho {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->rho = t[0];
        if (fabs(c->rho_last) < c->tol) {
            c->done = 1;
            c->status = JFG_BREAKDOWN;
            return;
        }
        c->beta = c->alpha / c->omega * c->rho / c->rho_last;
    }
};
template <typename T>
struct VBicgP {      // p = (r + p*beta) - v*(omega*beta)
    const T* r;
    T* p;
    const T* v;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&)[K]) const
    {
        T b = (T)c->beta, ob = (T)(c->omega * c->beta);
        p[i] = (r[i] + p[i] * b) - v[i] * ob;
    }
};
struct FinAlphaB {   // alpha = rho / v.r0
    Ctl* c;
    __device__ void operator()(const double* t) const { c->alpha = c->rho / t[0]; }
};
template <typename T>
struct VBicgS {      // s = r - v*alpha; acc += s^2
    const T* r;
    const T* v;
    T* s;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        T sv = r[i] - v[i] * (T)c->alpha;
        s[i] = sv;
        acc[0] += (double)sv * (double)sv;
    }
};
struct FinS {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        c->s_norm = sqrt(t[0]);
        c->sdone = c->s_norm < c->tol ? 1 : 0;
        c->skip = c->sdone;
    }
};
template <typename T>
struct EpiStoreDot2 {  // t = A s; acc0 += t.s, acc1 += t.t
    T* y;
    const T* s;
    template <typename AT, int K>
    __device__ void operator()(int r, AT v, double (&acc)[K]) const
    {
        y[r] = (T)v;
        acc[0] += (double)v * (double)s[r];
        acc[1] += (double)v * (double)v;
    }
};
template <typename T>
struct VDot2 {       // acc0 += a.b, acc1 += a.a
    const T* a;
    const T* b;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        acc[0] += (double)a[i] * (double)b[i];
        acc[1] += (double)a[i] * (double)a[i];
    }
};
struct FinOmega {
    Ctl* c;
    __device__ void operator()(const double* t) const { c->omega = t[0] / t[1]; }
};
template <typename T>
struct VBicgEnd {    // sdone: x += y*alpha  else: x = (x + y*alpha) + z*omega; r = s - t*omega
    T* x;
    const T* y;
    const T* z;
    const T* s;
    const T* t;
    T* r;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const
    {
        T a = (T)c->alpha;
        if (c->sdone) {
            x[i] = x[i] + y[i] * a;
            return;
        }
        T w = (T)c->omega;
        x[i] = (x[i] + y[i] * a) + z[i] * w;
        T rn = s[i] - t[i] * w;
        r[i] = rn;
        acc[0] += (double)rn * (double)rn;
    }
};
struct FinBicgEnd {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        if (c->sdone) {
            c->done = 1;
            c->status = JFG_OK;
            c->res_norm = c->s_norm;
            return;
        }
        c->rho_last = c->rho;
        c->iter++;
        publish(c, sqrt(t[0]));
        check(c, sqrt(t[0]));
    }
};

// GMRES pieces (GMRES.java:136-251)
template <typename T>
__global__ void k_mdot(int n, const T* __restrict__ V, const T* __restrict__ q, const Ctl* __restrict__ c,
                       double* __restrict__ part, const int* __restrict__ flag)
{
    pdl_wait();
    if (*flag) return;
    int i = blockIdx.y;
    if (i > c->j) return;
    const T* v = V + (size_t)i * n;
    double acc[1] = {0};
    for (int r = blockIdx.x * kThreads + threadIdx.x; r < n; r += gridDim.x * kThreads)
        acc[0] += (double)v[r] * (double)q[r];
    block_sum<1>(acc);
    if (threadIdx.x == 0) part[(size_t)i * gridDim.x + blockIdx.x] = acc[0];
}
__global__ void k_mdot_fin(int gx, const double* __restrict__ part, const Ctl* __restrict__ c, double* __restrict__ fac,
                           const int* __restrict__ flag)
{
    pdl_wait();
    if (*flag) return;
    int i = blockIdx.x;
    if (i > c->j) return;
    double acc[1] = {0};
    for (int k = threadIdx.x; k < gx; k += kThreads) acc[0] += part[(size_t)i * gx + k];
    block_sum<1>(acc);
    if (threadIdx.x == 0) fac[i] = acc[0];
}
template <typename T>
struct VGmresW {     // w = q - sum_i V_i fac_i; acc += w^2
    const T* V;
    const T* q;
    T* w;
    const double* fac;
    const Ctl* c;
    int n;
    template <int K> __device__ void operator()(int r, double (&acc)[K]) const
    {
        int j = c->j;
        T lc = 0;
        for (int i = 0; i <= j; i++) lc = lc + V[(size_t)i * n + r] * (T)fac[i];
        T wv = q[r] - lc;
        w[r] = wv;
        acc[0] += (double)wv * (double)wv;
    }
};
struct FinGivens {
    Ctl* c;
    double* h;
    double* gam;
    double* cs;
    double* sn;
    const double* fac;
    int ldh;
    __device__ void operator()(const double* t) const
    {
        int j = c->j;
        for (int i = 0; i <= j; i++) h[(size_t)i * ldh + j] += fac[i];
        double wn = sqrt(t[0]);
        h[(size_t)(j + 1) * ldh + j] += wn;
        for (int i = 0; i < j; i++) {
            double hij = h[(size_t)i * ldh + j], hipj = h[(size_t)(i + 1) * ldh + j];
            h[(size_t)i * ldh + j] = hij * cs[i] + hipj * sn[i];
            h[(size_t)(i + 1) * ldh + j] = -hij * sn[i] + hipj * cs[i];
        }
        double hjj = h[(size_t)j * ldh + j], hj1 = h[(size_t)(j + 1) * ldh + j];
        double beta = sqrt(hjj * hjj + hj1 * hj1);
        sn[j] = hj1 / beta;
        cs[j] = hjj / beta;
        h[(size_t)j * ldh + j] = beta;
        gam[j + 1] = -sn[j] * gam[j];
        gam[j] = cs[j] * gam[j];
        double g = fabs(gam[j + 1]);
        c->res_norm = g;
        if (c->hist && c->iter < c->hist_cap) c->hist[c->iter] = g;
        if (g < c->tol || j > c->restart_len || !isfinite(g)) {
            c->cycle_done = 1;
            c->jfin = j;
            if (!isfinite(g)) c->status = JFG_NONFINITE;
        }
    }
};
template <typename T>
struct VGmresNext {  // v_{j+1} = w / h[j+1][j] into V and vcur
    T* V;
    T* vcur;
    const T* w;
    const double* h;
    const Ctl* c;
    int n;
    int ldh;
    template <int K> __device__ void operator()(int r, double (&)[K]) const
    {
        int j = c->j;
        T inv = (T)(1.0 / h[(size_t)(j + 1) * ldh + j]);
        T v = w[r] * inv;
        V[(size_t)(j + 1) * n + r] = v;
        vcur[r] = v;
    }
};
struct GmresAdvance {
    Ctl* c;
    __device__ void operator()() const
    {
        c->iter++;
        c->j++;
        if (c->j == c->n) {
            c->cycle_done = 1;
            c->jfin = c->n - 1;
        }
    }
};
struct GmresAlpha {  // calculateAlpha (GMRES.java:239-251)
    const Ctl* c;
    const double* h;
    const double* gam;
    double* alpha;
    int ldh;
    __device__ void operator()() const
    {
        int j = c->jfin;
        for (int i = j; i >= 0; i--) {
            double s = 0;
            for (int k = i + 1; k <= j; k++) s += h[(size_t)i * ldh + k] * alpha[k];
            alpha[i] = 1.0 / h[(size_t)i * ldh + i] * (gam[i] - s);
        }
    }
};
template <typename T>
struct VGmresX {     // x = x + sum_i V_i alpha_i
    T* x;
    const T* V;
    const double* alpha;
    const Ctl* c;
    int n;
    template <int K> __device__ void operator()(int r, double (&)[K]) const
    {
        int j = c->jfin;
        T lc = 0;
        for (int i = 0; i <= j; i++) lc = lc + V[(size_t)i * n + r] * (T)alpha[i];
        x[r] = x[r] + lc;
    }
};
struct FinGamma0 {
    Ctl* c;
    double* gam;
    __device__ void operator()(const double* t) const
    {
        double g = sqrt(t[0]);
        gam[0] = g;
        c->res_norm = g;
        c->j = 0;
        c->jfin = 0;
        c->cycle_done = 0;
        if (g <= c->tol) {           // GMRES.java:77, 113: return x
            c->cycle_done = 1;
            c->done = 1;
            c->status = JFG_OK;
        }
        if (!isfinite(g)) {
            c->cycle_done = 1;
            c->done = 1;
            c->status = JFG_NONFINITE;
        }
    }
};
template <typename T>
struct VScaleInto2 {  // a = b * (1 / gam0), c = a
    T* a;
    T* cpy;
    const T* b;
    const double* gam;
    template <int K> __device__ void operator()(int i, double (&)[K]) const
    {
        T v = b[i] * (T)(1.0 / gam[0]);
        a[i] = v;
        cpy[i] = v;
    }
};
struct FinTrueRes {
    Ctl* c;
    __device__ void operator()(const double* t) const { c->true_res = sqrt(t[0]); }
};

__global__ void k_set_cond(cudaGraphConditionalHandle h, const int* flag)
{
    pdl_wait();
    cudaGraphSetConditional(h, *flag ? 0u : 1u);
}

template <typename T>
struct VAddScaled {  // x64 += s * e   (defect correction)
    double* x;
    const T* e;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { x[i] = x[i] + c->res_norm * (double)e[i]; }
};
template <typename T>
struct VScaleDown {  // r32 = r64 / ||r64||
    const double* r;
    T* o;
    const Ctl* c;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { o[i] = (T)(r[i] / c->res_norm); }
};
struct FinOuter {
    Ctl* c;
    __device__ void operator()(const double* t) const
    {
        double rn = sqrt(t[0]);
        c->res_norm = rn;
        c->rr = t[0];
        publish(c, rn);
        check(c, rn);
    }
};

inline int vec_grid_n(int n) { return vec_grid(n); }

}  // namespace

template <typename T>
void Precond<T>::apply(const T* r, T* z, const Scratch& sc, const int* done, cudaStream_t st) const
{
    if (hook) {     // multigrid + network, Schwarz, block-diagonal
        hook(hook_self, r, z, sc, done, st);
        return;
    }
    switch (kind) {
    case JFG_PREC_MG:
        if (mg32) {
            vec_launch<0>(st, n, VCast<T, float>{r, r32}, sc, done);
            mg32->apply(r32, z32, sc, done, st);
            vec_launch<0>(st, n, VCast<float, T>{z32, z}, sc, done);
        } else {
            mg->apply(r, z, sc, done, st);
        }
        break;
    case JFG_PREC_JACOBI:
        vec_launch<0>(st, n, VMul<T>{dinv, r, z}, sc, done);
        break;
    case JFG_PREC_MATRIX:
        spmv_launch<T, T, 0>(st, M, vals_of<T>(M), r, EpiStore<T>{z}, sc, done);
        break;
    default:
        vec_launch<0>(st, n, VCopy<T>{r, z}, sc, done);
        break;
    }
}
template struct Precond<double>;
template struct Precond<float>;

GraphCache::~GraphCache()
{
    for (auto& kv : execs) cudaGraphExecDestroy(kv.second);
}

void SolverWork::ensure(int n, int max_blocks, int hist_cap)
{
    ctl.alloc(2);
    hist.alloc(hist_cap > 0 ? hist_cap : 1);
    size_t need = (size_t)4 * (max_blocks > kVecGrid ? max_blocks : kVecGrid);
    if (partials.n < need) {
        // pointers baked into cached graphs change: drop them
        for (auto& kv : graphs.execs) cudaGraphExecDestroy(kv.second);
        graphs.execs.clear();
    }
    partials.alloc(need);
    if (!counter.p) {
        counter.alloc(4);
        JFG_CUDA(cudaMemset(counter.p, 0, 4 * sizeof(unsigned)));
    }
    sc.partials = partials.p;
    sc.counter = counter.p;
    (void)n;
}

static bool g_conditional_ok = true;

int run_loop(SolverWork& w, const int* flag, const std::vector<uintptr_t>& key, const std::function<void()>& iter,
             int use_graph, int chunk)
{
    cudaStream_t st = w.c->stream;
    if (chunk < 1) chunk = 8;
    if (use_graph && g_conditional_ok) {
        cudaGraphExec_t exec = nullptr;
        int nodes = 0;
        auto it = w.graphs.execs.find(key);
        if (it != w.graphs.execs.end()) {
            exec = it->second;
            nodes = w.graphs.nodes[key];
        } else {
            cudaGraph_t g = nullptr;
            bool ok = false;
            if (cudaGraphCreate(&g, 0) == cudaSuccess) {
                cudaGraphConditionalHandle h;
                if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess) {
                    cudaGraphNodeParams p = {};
                    p.type = cudaGraphNodeTypeConditional;
                    p.conditional.handle = h;
                    p.conditional.type = cudaGraphCondTypeWhile;
                    p.conditional.size = 1;
                    cudaGraphNode_t node;
                    if (cudaGraphAddNode(&node, g, nullptr, 0, &p) == cudaSuccess) {
                        cudaGraph_t body = p.conditional.phGraph_out[0];
                        JFG_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                                               cudaStreamCaptureModeThreadLocal));
                        unsigned long long before = g_launches.load();
                        try {
                            iter();
                            launch_ex(k_set_cond, dim3(1), dim3(1), 0, st, h, flag);
                            nodes = (int)(g_launches.load() - before);
                            g_launches.fetch_sub(nodes);
                        } catch (...) {
                            cudaGraph_t dummy;
                            cudaStreamEndCapture(st, &dummy);
                            cudaGraphDestroy(g);
                            throw;
                        }
                        cudaGraph_t outg = nullptr;
                        cudaError_t e = cudaStreamEndCapture(st, &outg);
                        if (e == cudaSuccess && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) ok = true;
                    }
                }
                cudaGraphDestroy(g);
            }
            cudaGetLastError();
            if (!ok) {
                g_conditional_ok = false;
                exec = nullptr;
            } else {
                w.graphs.execs[key] = exec;
                w.graphs.nodes[key] = nodes;
            }
        }
        if (exec) {
            JFG_CUDA(cudaGraphLaunch(exec, st));
            return nodes;
        }
    }
    // fallback: chunks of plain launches with a convergence poll
    int h_flag = 0;
    for (;;) {
        for (int k = 0; k < chunk; k++) iter();
        JFG_CUDA(cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        if (h_flag) break;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// the solvers
// ---------------------------------------------------------------------------
template <typename T>
static void vec_copy(cudaStream_t st, int n, const T* a, T* b, const Scratch& sc, const int* done)
{
    vec_launch<0>(st, n, VCopy<T>{a, b}, sc, done);
}

static void init_ctl(SolverWork& w, int idx, double tol, int maxit, double* hist, int hist_cap, int n, int restart)
{
    Ctl h{};
    h.tol = tol;
    h.maxit = maxit;
    h.alpha = 1;
    h.omega = 1;
    h.rho = 1;
    h.rho_last = 1;
    h.beta = 1;
    h.hist = hist;
    h.hist_cap = hist_cap;
    h.n = n;
    h.restart_len = restart;
    h.status = JFG_NOT_CONVERGED;
    JFG_CUDA(cudaMemcpyAsync(w.ctl.p + idx, &h, sizeof(Ctl), cudaMemcpyHostToDevice, w.c->stream));
    JFG_CUDA(cudaStreamSynchronize(w.c->stream));
}

static Ctl read_ctl(SolverWork& w, int idx)
{
    Ctl h;
    JFG_CUDA(cudaMemcpyAsync(&h, w.ctl.p + idx, sizeof(Ctl), cudaMemcpyDeviceToHost, w.c->stream));
    JFG_CUDA(cudaStreamSynchronize(w.c->stream));
    return h;
}

// (P)CG on device vectors of type T with matrix values of type T.
// b, x: device; x holds the start iterate.  `xzero`: x is known to be zero.
template <typename T>
int run_cg(SolverWork& w, int ci, Matrix* A, const Precond<T>& M, const T* b, T* x, T* r, T* p, T* Ap, T* z,
            bool xzero, int use_graph, int chunk)
{
    cudaStream_t st = w.c->stream;
    Ctl* c = w.ctl.p + ci;
    const int* done = &c->done;
    int n = A->rows;
    const Scratch& sc = w.sc;
    const T* val = vals_of<T>(A);
    bool pcg = M.kind != JFG_PREC_NONE;
    if (xzero) {
        vec_launch<1>(st, n, VCopyNorm<T>{b, r}, sc, nullptr, FinInit{c});
    } else {
        spmv_launch<T, T, 1>(st, A, val, x, EpiResid<T>{b, r}, sc, nullptr, FinInit{c});
    }
    if (pcg) {
        M.apply(r, z, sc, done, st);
        vec_launch<1>(st, n, VDot<T>{r, z}, sc, done, FinRZ{c});
        vec_copy<T>(st, n, z, p, sc, done);
    } else {
        vec_copy<T>(st, n, r, p, sc, done);
    }
    const bool fused32 = std::is_same<T, double>::value && M.kind == JFG_PREC_MG && M.mg32 && !M.hook;
    auto iter = [&]() {
        spmv_launch<T, T, 1>(st, A, val, p, EpiStoreDot<T>{Ap, p}, sc, done, FinAlpha{c});
        if constexpr (std::is_same<T, double>::value) {
            if (fused32) {
                vec_launch<1>(st, n, VCGUpdate32{x, p, r, Ap, M.r32, c}, sc, done, FinCGRes{c, 1});
                M.mg32->apply(M.r32, M.z32, sc, done, st);
                vec_launch<1>(st, n, VDotMixed{r, M.z32}, sc, done, FinBeta{c});
                vec_launch<0>(st, n, VXpby32{M.z32, p, c}, sc, done);
                return;
            }
        }
        vec_launch<1>(st, n, VCGUpdate<T>{x, p, r, Ap, c}, sc, done, FinCGRes{c, pcg ? 1 : 0});
        if (pcg) {
            M.apply(r, z, sc, done, st);
            vec_launch<1>(st, n, VDot<T>{r, z}, sc, done, FinBeta{c});
            vec_launch<0>(st, n, VXpby<T>{z, p, c}, sc, done);
        } else {
            vec_launch<0>(st, n, VXpby<T>{r, p, c}, sc, done);
        }
    };
    std::vector<uintptr_t> key{1, (uintptr_t)A->uid, (uintptr_t)(M.mg ? M.mg->uid : 0), (uintptr_t)M.hook_uid, (uintptr_t)(M.M ? M.M->uid : 0), (uintptr_t)(M.mg32 ? M.mg32->uid : 0), (uintptr_t)M.r32, (uintptr_t)M.dinv, (uintptr_t)b,
                               (uintptr_t)x, (uintptr_t)r, (uintptr_t)p, (uintptr_t)z, (uintptr_t)Ap, (uintptr_t)sizeof(T),
                               (uintptr_t)M.kind, (uintptr_t)done};
    return run_loop(w, done, key, iter, use_graph, chunk);
}

template <typename T>
int run_bicgstab(SolverWork& w, int ci, Matrix* A, const Precond<T>& M, const T* b, T* x, T* const* v,
                  int use_graph, int chunk)
{
    cudaStream_t st = w.c->stream;
    Ctl* c = w.ctl.p + ci;
    const int* done = &c->done;
    const int* skip = &c->skip;
    int n = A->rows;
    const Scratch& sc = w.sc;
    const T* val = vals_of<T>(A);
    bool pre = M.kind != JFG_PREC_NONE;
    T *r0 = v[0], *r = v[1], *p = v[2], *vv = v[3], *s = v[4], *t = v[5], *y = v[6], *z = v[7];
    T* pt = v[8];
    spmv_launch<T, T, 1>(st, A, val, x, EpiResid<T>{b, r0}, sc, nullptr, FinInit{c});
    vec_copy<T>(st, n, r0, r, sc, nullptr);
    vec_launch<0>(st, n, VZero<T>{p}, sc, nullptr);
    vec_launch<0>(st, n, VZero<T>{vv}, sc, nullptr);
    auto iter = [&]() {
        vec_launch<1>(st, n, VDot<T>{r, r0}, sc, done, FinRho{c});
        vec_launch<0>(st, n, VBicgP<T>{r, p, vv, c}, sc, done);
        const T* yy = p;
        if (pre) {
            M.apply(p, y, sc, done, st);
            yy = y;
        }
        spmv_launch<T, T, 1>(st, A, val, yy, EpiStoreDot<T>{vv, r0}, sc, done, FinAlphaB{c});
        vec_launch<1>(st, n, VBicgS<T>{r, vv, s, c}, sc, done, FinS{c});
        if (pre) {
            M.apply(s, z, sc, skip, st);
            spmv_launch<T, T, 0>(st, A, val, z, EpiStore<T>{t}, sc, skip);
            M.apply(t, pt, sc, skip, st);
            vec_launch<2>(st, n, VDot2<T>{pt, z}, sc, skip, FinOmega{c});
            vec_launch<1>(st, n, VBicgEnd<T>{x, y, z, s, t, r, c}, sc, done, FinBicgEnd{c});
        } else {
            spmv_launch<T, T, 2>(st, A, val, s, EpiStoreDot2<T>{t, s}, sc, skip, FinOmega{c});
            vec_launch<1>(st, n, VBicgEnd<T>{x, p, s, s, t, r, c}, sc, done, FinBicgEnd{c});
        }
    };
    std::vector<uintptr_t> key{2, (uintptr_t)A->uid, (uintptr_t)(M.mg ? M.mg->uid : 0), (uintptr_t)M.hook_uid, (uintptr_t)(M.M ? M.M->uid : 0), (uintptr_t)(M.mg32 ? M.mg32->uid : 0), (uintptr_t)M.r32, (uintptr_t)M.dinv, (uintptr_t)b,
                               (uintptr_t)x, (uintptr_t)r0, (uintptr_t)r, (uintptr_t)p, (uintptr_t)vv, (uintptr_t)s,
                               (uintptr_t)t, (uintptr_t)y, (uintptr_t)z, (uintptr_t)pt, (uintptr_t)sizeof(T),
                               (uintptr_t)M.kind, (uintptr_t)done};
    return run_loop(w, done, key, iter, use_graph, chunk);
}

// Restarted GMRES (double only).  Returns restarts done.
int run_gmres(SolverWork& w, Matrix* A, const Precond<double>& M, const double* b, double* x, int IBR,
              int max_restarts, int use_graph, int chunk)
{
    return run_gmres(w, op_of(A), M, b, x, IBR, max_restarts, use_graph, chunk);
}

int run_gmres(SolverWork& w, const Operator& op, const Precond<double>& M, const double* b, double* x, int IBR,
              int max_restarts, int use_graph, int chunk)
{
    cudaStream_t st = w.c->stream;
    Ctl* c = w.ctl.p;
    const int* cdone = &c->cycle_done;
    int n = op.n;
    const Scratch& sc = w.sc;
    bool pre = M.kind != JFG_PREC_NONE;
    int m = IBR + 3;
    int ldh = IBR + 10;
    if (w.gm_m < m || w.V.n < (size_t)m * n) {
        w.V.alloc((size_t)m * n);
        w.gm_m = m;
    }
    w.H.alloc((size_t)ldh * ldh);
    w.gam.alloc(ldh);
    w.cs.alloc(ldh);
    w.sn.alloc(ldh);
    w.fac.alloc(ldh);
    w.alpha.alloc(ldh);
    int gx = vec_grid_n(n) < 296 ? vec_grid_n(n) : 296;
    w.mdot_part.alloc((size_t)gx * m);
    double *t = w.v64[2].p, *q = w.v64[3].p, *wv = w.v64[4].p, *vcur = w.v64[5].p, *rr = w.v64[6].p;
    const double* qq = pre ? q : t;
    double* V = w.V.p;
    int restarts = 0;
    int iter_before = read_ctl(w, 0).iter;
    for (;;) {
        JFG_CUDA(cudaMemsetAsync(w.H.p, 0, sizeof(double) * ldh * ldh, st));
        JFG_CUDA(cudaMemsetAsync(w.gam.p, 0, sizeof(double) * ldh, st));
        op_launch<0>(st, op, x, EpiResid<double>{b, pre ? t : rr}, sc, nullptr);
        if (pre) M.apply(t, rr, sc, nullptr, st);
        vec_launch<1>(st, n, VNorm2<double>{rr}, sc, nullptr, FinGamma0{c, w.gam.p});
        vec_launch<0>(st, n, VScaleInto2<double>{V, vcur, rr, w.gam.p}, sc, cdone);
        auto iter = [&]() {
            op_launch<0>(st, op, vcur, EpiStore<double>{t}, sc, cdone);
            if (pre) M.apply(t, q, sc, cdone, st);
            dim3 g1(gx, m);
            launch_ex(k_mdot<double>, g1, dim3(kThreads), 0, st, n, (const double*)V, qq, (const Ctl*)c,
                      w.mdot_part.p, cdone);
            launch_ex(k_mdot_fin, dim3(m), dim3(kThreads), 0, st, gx, (const double*)w.mdot_part.p, (const Ctl*)c,
                      w.fac.p, cdone);
            vec_launch<1>(st, n, VGmresW<double>{V, qq, wv, w.fac.p, c, n}, sc, cdone,
                          FinGivens{c, w.H.p, w.gam.p, w.cs.p, w.sn.p, w.fac.p, ldh});
            vec_launch<0>(st, n, VGmresNext<double>{V, vcur, wv, w.H.p, c, n, ldh}, sc, cdone);
            scalar_launch(st, GmresAdvance{c}, cdone);
        };
        std::vector<uintptr_t> key{3, (uintptr_t)op.uid, (uintptr_t)(M.mg ? M.mg->uid : 0), (uintptr_t)M.hook_uid, (uintptr_t)(M.M ? M.M->uid : 0), (uintptr_t)(M.mg32 ? M.mg32->uid : 0), (uintptr_t)M.r32, (uintptr_t)M.dinv,
                                   (uintptr_t)x, (uintptr_t)V, (uintptr_t)M.kind, (uintptr_t)m, (uintptr_t)t,
                                   (uintptr_t)q, (uintptr_t)wv, (uintptr_t)vcur, (uintptr_t)w.H.p,
                                   (uintptr_t)w.fac.p, (uintptr_t)w.mdot_part.p, (uintptr_t)cdone};
        int nodes = run_loop(w, cdone, key, iter, use_graph, chunk);
        Ctl h = read_ctl(w, 0);
        note_launch((unsigned long long)nodes * (unsigned long long)(h.iter - iter_before + 1));
        iter_before = h.iter;
        if (h.done) break;   // converged at the cycle start (or non-finite)
        scalar_launch(st, GmresAlpha{c, w.H.p, w.gam.p, w.alpha.p, ldh}, nullptr);
        vec_launch<0>(st, n, VGmresX<double>{x, V, w.alpha.p, c, n}, sc, nullptr);
        op_launch<1>(st, op, x, EpiResid<double>{b, t}, sc, nullptr, FinTrueRes{c});
        h = read_ctl(w, 0);
        bool nonfinite = !std::isfinite(h.true_res) || h.status == JFG_NONFINITE;
        if (nonfinite) {
            Ctl hc = h;
            hc.status = JFG_NONFINITE;
            hc.done = 1;
            JFG_CUDA(cudaMemcpyAsync(w.ctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
            break;
        }
        // GMRES.java:92: restart while j > ITERATIONS_BEFORE_RESTART (bounded) or residual > tol
        if ((h.jfin > IBR && restarts < max_restarts) || h.true_res > h.tol) {
            if (restarts >= max_restarts) {
                Ctl hc = h;
                hc.status = JFG_NOT_CONVERGED;
                hc.done = 1;
                JFG_CUDA(cudaMemcpyAsync(w.ctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
                break;
            }
            restarts++;
            continue;
        }
        Ctl hc = h;
        hc.status = JFG_OK;
        hc.done = 1;
        JFG_CUDA(cudaMemcpyAsync(w.ctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
        break;
    }
    JFG_CUDA(cudaStreamSynchronize(st));
    return restarts;
}

// ---------------------------------------------------------------------------
// Flexible GMRES(m) with right preconditioning (Saad 1993): the
// preconditioner may change between iterations (the learned smoother is
// nonlinear), so z_j = M_j v_j is stored and x = x0 + Z y.  Classical
// Gram-Schmidt with one re-orthogonalisation pass.  No counterpart in the
// reference (its GMRES is left-preconditioned, GMRES.java:64-101).
// ---------------------------------------------------------------------------
namespace {
template <typename T>
struct VGmresW0 {    // w = q - sum_i V_i fac_i (no norm)
    const T* V;
    const T* q;
    T* w;
    const double* fac;
    const Ctl* c;
    int n;
    template <int K> __device__ void operator()(int r, double (&)[K]) const
    {
        int j = c->j;
        T lc = 0;
        for (int i = 0; i <= j; i++) lc = lc + V[(size_t)i * n + r] * (T)fac[i];
        w[r] = q[r] - lc;
    }
};
struct FinGivensSum {   // h column = fac + fac2, then the rotations of FinGivens
    FinGivens g;
    const double* fac2;
    double* facsum;
    __device__ void operator()(const double* t) const
    {
        int j = g.c->j;
        for (int i = 0; i <= j; i++) facsum[i] = g.fac[i] + fac2[i];
        FinGivens g2 = g;
        g2.fac = facsum;
        g2(t);
    }
};
struct VStoreCol {      // Z[:, j] = z
    double* Z;
    const double* z;
    const Ctl* c;
    int n;
    template <int K> __device__ void operator()(int r, double (&)[K]) const { Z[(size_t)c->j * n + r] = z[r]; }
};
}  // namespace

int run_fgmres(SolverWork& w, Matrix* A, const Precond<double>& M, const double* b, double* x, int m_restart,
               int max_restarts, int use_graph, int chunk)
{
    cudaStream_t st = w.c->stream;
    Ctl* c = w.ctl.p;
    const int* cdone = &c->cycle_done;
    int n = A->rows;
    const Scratch& sc = w.sc;
    const double* val = A->val.p;
    int IBR = m_restart;
    int m = IBR + 3;
    int ldh = IBR + 10;
    if (w.gm_m < m || w.V.n < (size_t)m * n) {
        w.V.alloc((size_t)m * n);
        w.gm_m = m;
    }
    w.Z.alloc((size_t)m * n);
    w.H.alloc((size_t)ldh * ldh);
    w.gam.alloc(ldh);
    w.cs.alloc(ldh);
    w.sn.alloc(ldh);
    w.fac.alloc(ldh);
    w.fac2.alloc(ldh);
    w.facsum.alloc(ldh);
    w.alpha.alloc(ldh);
    int gx = vec_grid_n(n) < 296 ? vec_grid_n(n) : 296;
    w.mdot_part.alloc((size_t)gx * m);
    double *t = w.v64[2].p, *wv = w.v64[4].p, *vcur = w.v64[5].p, *rr = w.v64[6].p, *zcur = w.v64[7].p;
    double* V = w.V.p;
    double* Z = w.Z.p;
    int restarts = 0;
    int iter_before = read_ctl(w, 0).iter;
    for (;;) {
        JFG_CUDA(cudaMemsetAsync(w.H.p, 0, sizeof(double) * ldh * ldh, st));
        JFG_CUDA(cudaMemsetAsync(w.gam.p, 0, sizeof(double) * ldh, st));
        spmv_launch<double, double, 0>(st, A, val, x, EpiResid<double>{b, rr}, sc, nullptr);
        vec_launch<1>(st, n, VNorm2<double>{rr}, sc, nullptr, FinGamma0{c, w.gam.p});
        vec_launch<0>(st, n, VScaleInto2<double>{V, vcur, rr, w.gam.p}, sc, cdone);
        auto iter = [&]() {
            M.apply(vcur, zcur, sc, cdone, st);
            vec_launch<0>(st, n, VStoreCol{Z, zcur, c, n}, sc, cdone);
            spmv_launch<double, double, 0>(st, A, val, zcur, EpiStore<double>{t}, sc, cdone);
            dim3 g1(gx, m);
            // pass 1: fac = V^T t ; w = t - V fac
            launch_ex(k_mdot<double>, g1, dim3(kThreads), 0, st, n, (const double*)V, (const double*)t,
                      (const Ctl*)c, w.mdot_part.p, cdone);
            launch_ex(k_mdot_fin, dim3(m), dim3(kThreads), 0, st, gx, (const double*)w.mdot_part.p, (const Ctl*)c,
                      w.fac.p, cdone);
            vec_launch<0>(st, n, VGmresW0<double>{V, t, wv, w.fac.p, c, n}, sc, cdone);
            // pass 2: fac2 = V^T w ; w = w - V fac2 ; ||w|| ; Givens on fac + fac2
            launch_ex(k_mdot<double>, g1, dim3(kThreads), 0, st, n, (const double*)V, (const double*)wv,
                      (const Ctl*)c, w.mdot_part.p, cdone);
            launch_ex(k_mdot_fin, dim3(m), dim3(kThreads), 0, st, gx, (const double*)w.mdot_part.p, (const Ctl*)c,
                      w.fac2.p, cdone);
            vec_launch<1>(st, n, VGmresW<double>{V, wv, wv, w.fac2.p, c, n}, sc, cdone,
                          FinGivensSum{FinGivens{c, w.H.p, w.gam.p, w.cs.p, w.sn.p, w.fac.p, ldh}, w.fac2.p,
                                       w.facsum.p});
            vec_launch<0>(st, n, VGmresNext<double>{V, vcur, wv, w.H.p, c, n, ldh}, sc, cdone);
            scalar_launch(st, GmresAdvance{c}, cdone);
        };
        std::vector<uintptr_t> key{7, (uintptr_t)A->uid, (uintptr_t)(M.mg ? M.mg->uid : 0),
                                   (uintptr_t)(M.hook_uid), (uintptr_t)(M.mg32 ? M.mg32->uid : 0),
                                   (uintptr_t)M.r32, (uintptr_t)M.kind, (uintptr_t)x, (uintptr_t)V, (uintptr_t)Z,
                                   (uintptr_t)m, (uintptr_t)t, (uintptr_t)wv, (uintptr_t)vcur, (uintptr_t)zcur,
                                   (uintptr_t)w.H.p, (uintptr_t)w.fac.p, (uintptr_t)w.fac2.p,
                                   (uintptr_t)w.mdot_part.p, (uintptr_t)cdone};
        int nodes = run_loop(w, cdone, key, iter, use_graph, chunk);
        Ctl h = read_ctl(w, 0);
        note_launch((unsigned long long)nodes * (unsigned long long)(h.iter - iter_before + 1));
        iter_before = h.iter;
        if (h.done) break;
        scalar_launch(st, GmresAlpha{c, w.H.p, w.gam.p, w.alpha.p, ldh}, nullptr);
        vec_launch<0>(st, n, VGmresX<double>{x, Z, w.alpha.p, c, n}, sc, nullptr);
        spmv_launch<double, double, 1>(st, A, val, x, EpiResid<double>{b, t}, sc, nullptr, FinTrueRes{c});
        h = read_ctl(w, 0);
        Ctl hc = h;
        hc.done = 1;
        if (!std::isfinite(h.true_res) || h.status == JFG_NONFINITE) {
            hc.status = JFG_NONFINITE;
        } else if ((h.jfin > IBR && restarts < max_restarts) || h.true_res > h.tol) {
            // the restart rule of GMRES.java:92, bounded by max_restarts
            if (restarts < max_restarts) {
                restarts++;
                continue;
            }
            hc.status = JFG_NOT_CONVERGED;
        } else {
            hc.status = JFG_OK;
        }
        JFG_CUDA(cudaMemcpyAsync(w.ctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
        break;
    }
    JFG_CUDA(cudaStreamSynchronize(st));
    return restarts;
}

template int run_cg<double>(SolverWork&, int, Matrix*, const Precond<double>&, const double*, double*, double*,
                            double*, double*, double*, bool, int, int);
template int run_cg<float>(SolverWork&, int, Matrix*, const Precond<float>&, const float*, float*, float*, float*,
                           float*, float*, bool, int, int);
template int run_bicgstab<double>(SolverWork&, int, Matrix*, const Precond<double>&, const double*, double*,
                                   double* const*, int, int);

// FP64 defect correction around FP32 inner (P)CG (x: FP64 device iterate).
// Returns the number of outer steps.
int run_mixed_cg(SolverWork& w, Matrix* A, const Precond<float>& M, const double* b, double* x, double tol,
                 int maxit, double inner_rtol, int use_graph, int chunk, int* inner_iters, double* hist, int hist_cap)
{
    cudaStream_t st = w.c->stream;
    int n = A->rows;
    const Scratch& sc = w.sc;
    matrix_ensure_fp32(A);
    Ctl* co = w.ctl.p;
    double* r64 = w.v64[2].p;
    float *b32 = w.v32[0].p, *e32 = w.v32[1].p, *r32 = w.v32[2].p, *p32 = w.v32[3].p, *Ap32 = w.v32[4].p,
          *z32 = w.v32[5].p;
    init_ctl(w, 0, tol, 1 << 30, hist, hist_cap, n, 0);
    int outer = 0, total_inner = 0;
    int max_outer = 100;
    for (;;) {
        spmv_launch<double, double, 1>(st, A, A->val.p, x, EpiResid<double>{b, r64}, sc, nullptr, FinOuter{co});
        Ctl h = read_ctl(w, 0);
        if (h.done || outer >= max_outer || total_inner >= maxit) break;
        vec_launch<0>(st, n, VScaleDown<float>{r64, b32, co}, sc, nullptr);
        vec_launch<0>(st, n, VZero<float>{e32}, sc, nullptr);
        int in_max = maxit - total_inner;
        init_ctl(w, 1, inner_rtol, in_max, nullptr, 0, n, 0);
        int nodes = run_cg<float>(w, 1, A, M, b32, e32, r32, p32, Ap32, z32, true, use_graph, chunk);
        Ctl hi = read_ctl(w, 1);
        note_launch((unsigned long long)nodes * (unsigned long long)(hi.iter > 0 ? hi.iter : 1));
        total_inner += hi.iter;
        vec_launch<0>(st, n, VAddScaled<float>{x, e32, co}, sc, nullptr);
        // iter counts outer steps in the history slot
        Ctl upd = read_ctl(w, 0);
        upd.iter++;
        JFG_CUDA(cudaMemcpyAsync(w.ctl.p, &upd, sizeof(Ctl), cudaMemcpyHostToDevice, st));
        outer++;
        if (hi.status == JFG_NONFINITE) break;
    }
    JFG_CUDA(cudaStreamSynchronize(st));
    *inner_iters = total_inner;
    return outer;
}

// ---------------------------------------------------------------------------
// GMRES2 (GMRES2.java:60-104) with its Arnoldi helper (Arnoldi.java:13-83)
// ---------------------------------------------------------------------------
namespace {
// device scalars of GMRES2 (w.g2): [0] t, [1] ||res||, [2] ||q_last||, [3] proj, [4] nn
struct FinG2T {       // t = Mres.Av / Av.Av
    double* g;
    __device__ void operator()(const double* s) const { g[0] = s[0] / s[1]; }
};
struct FinG2Store {   // g[idx] = sqrt(s) or s
    double* g;
    int idx;
    int root;
    __device__ void operator()(const double* s) const { g[idx] = root ? sqrt(s[0]) : s[0]; }
};
struct EpiG2Res {     // res -= t * (A v); acc += res^2
    double* res;
    const double* g;
    template <typename AT, int K>
    __device__ void operator()(int r, AT s, double (&acc)[K]) const
    {
        double v = res[r] - (double)s * g[0];
        res[r] = v;
        acc[0] += v * v;
    }
};
struct VG2Step {      // x += v t; Mres -= Av t
    double* x;
    const double* v;
    double* mres;
    const double* av;
    const double* g;
    template <int K> __device__ void operator()(int i, double (&)[K]) const
    {
        x[i] = x[i] + v[i] * g[0];
        mres[i] = mres[i] - av[i] * g[0];
    }
};
struct VG2Scale {     // y = a * (1 / g[idx])
    const double* a;
    double* y;
    const double* g;
    int idx;
    template <int K> __device__ void operator()(int i, double (&)[K]) const { y[i] = a[i] * (1.0 / g[idx]); }
};
struct VG2Mgs {       // apply the previous projection (if any), then acc += newAw . Av_i
    double* w;
    double* naw;
    const double* vprev;
    const double* avprev;
    const double* avi;      // null on the closing pass (then acc += naw^2)
    const double* g;
    template <int K> __device__ void operator()(int r, double (&acc)[K]) const
    {
        double nv = naw[r];
        if (vprev) {
            double p = g[3];
            w[r] = w[r] - vprev[r] * p;
            nv = nv - avprev[r] * p;
            naw[r] = nv;
        }
        acc[0] += avi ? nv * avi[r] : nv * nv;
    }
};
struct VG2New {       // V = w / nn, AV = newAw / nn
    double* v;
    double* av;
    const double* wv;
    const double* naw;
    const double* g;
    template <int K> __device__ void operator()(int i, double (&)[K]) const
    {
        v[i] = wv[i] * (1.0 / g[4]);
        av[i] = naw[i] * (1.0 / g[4]);
    }
};
}  // namespace

int run_gmres2(SolverWork& w, Matrix* A, const Precond<double>& M, const double* b, double* x, double tol, int maxit,
               int max_restarts, int basis_cap, int* iters, int* restarts_out, double* final_norm, double* hist,
               int hist_cap)
{
    cudaStream_t st = w.c->stream;
    const Scratch& sc = w.sc;
    int n = A->rows;
    const double* val = A->val.p;
    if (basis_cap < 2) basis_cap = 2;
    if (w.g2_cap < basis_cap || w.V2.n < (size_t)basis_cap * n) {
        w.V2.alloc((size_t)basis_cap * n);
        w.AV2.alloc((size_t)basis_cap * n);
        w.g2_cap = basis_cap;
    }
    w.g2.alloc(8);
    double* g = w.g2.p;
    double *res = w.v64[0].p, *mres = w.v64[1].p, *ql = w.v64[2].p, *wv = w.v64[3].p, *naw = w.v64[4].p,
           *t1 = w.v64[5].p;
    auto V = [&](int i) { return w.V2.p + (size_t)i * n; };
    auto AV = [&](int i) { return w.AV2.p + (size_t)i * n; };
    auto norm_into = [&](const double* a, int idx) {
        vec_launch<1>(st, n, VDot<double>{a, a}, sc, nullptr, FinG2Store{g, idx, 1});
    };
    auto MA = [&](const double* in, double* out) {  // out = M (A in)
        spmv_launch<double, double, 0>(st, A, val, in, EpiStore<double>{t1}, sc, nullptr);
        M.apply(t1, out, sc, nullptr, st);
    };
    auto read = [&](int idx) {
        double h = 0;
        JFG_CUDA(cudaMemcpyAsync(&h, g + idx, sizeof(double), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        return h;
    };
    int it = 0, restarts = 0, status = JFG_NOT_CONVERGED;
    double rn = 0;
    for (;;) {
        // solveInternal: res = b - A x; Mres = M res; Arnoldi(Mres, MA)
        spmv_launch<double, double, 1>(st, A, val, x, EpiResid<double>{b, res}, sc, nullptr, FinG2Store{g, 1, 1});
        M.apply(res, mres, sc, nullptr, st);
        norm_into(mres, 2);
        vec_launch<0>(st, n, VG2Scale{mres, wv, g, 2}, sc, nullptr);          // w0 = Mres / |Mres|
        MA(wv, ql);                                                            // q1 = MA w0 = Aw0
        norm_into(ql, 4);
        vec_launch<0>(st, n, VG2New{V(0), AV(0), wv, ql, g}, sc, nullptr);   // v0, Av0
        norm_into(ql, 2);
        vec_launch<0>(st, n, VG2Scale{ql, wv, g, 2}, sc, nullptr);
        MA(wv, naw);                                                           // q2 = MA(q1 / |q1|)
        vec_launch<0>(st, n, VCopy<double>{naw, ql}, sc, nullptr);
        norm_into(ql, 2);
        int nv = 1;
        rn = read(1);
        bool restart = false;
        while (rn > tol) {
            if (it >= maxit) break;
            const double* v = V(nv - 1);
            const double* av = AV(nv - 1);
            vec_launch<2>(st, n, VDot2<double>{av, mres}, sc, nullptr, FinG2T{g});
            spmv_launch<double, double, 1>(st, A, val, v, EpiG2Res{res, g}, sc, nullptr, FinG2Store{g, 1, 1});
            vec_launch<0>(st, n, VG2Step{x, v, mres, av, g}, sc, nullptr);
            rn = read(1);
            if (hist && it < hist_cap) JFG_CUDA(cudaMemcpyAsync(hist + it, g + 1, sizeof(double),
                                                                cudaMemcpyDeviceToDevice, st));
            it++;
            if (!std::isfinite(rn)) {
                status = JFG_NONFINITE;
                break;
            }
            // arnoldiStep
            vec_launch<0>(st, n, VG2Scale{ql, wv, g, 2}, sc, nullptr);       // w = q_last / |q_last|
            MA(wv, naw);                                                     // newAw = MA w
            vec_launch<0>(st, n, VCopy<double>{naw, ql}, sc, nullptr);     // q_last = newAw
            norm_into(ql, 2);
            for (int i = 0; i <= nv; i++) {
                const double* vprev = i > 0 ? V(i - 1) : nullptr;
                const double* avprev = i > 0 ? AV(i - 1) : nullptr;
                const double* avi = i < nv ? AV(i) : nullptr;
                vec_launch<1>(st, n, VG2Mgs{wv, naw, vprev, avprev, avi, g}, sc, nullptr,
                              FinG2Store{g, i < nv ? 3 : 4, i < nv ? 0 : 1});
            }
            if (nv >= basis_cap) {   // basis full: restart from the current iterate
                restart = true;
                break;
            }
            vec_launch<0>(st, n, VG2New{V(nv), AV(nv), wv, naw, g}, sc, nullptr);
            nv++;
            if (read(4) < 1e-13) {
                restart = true;
                break;
            }
        }
        if (status == JFG_NONFINITE) break;
        if (!(rn > tol)) {
            status = JFG_OK;
            break;
        }
        if (restart && restarts < max_restarts && it < maxit) {
            restarts++;
            continue;
        }
        break;
    }
    JFG_CUDA(cudaStreamSynchronize(st));
    *iters = it;
    *restarts_out = restarts;
    *final_norm = rn;
    return status;
}

// Jacobi preconditioner vectors
template <typename T>
void jacobi_apply(cudaStream_t st, int n, const T* d, const T* r, T* z, const Scratch& sc, const int* done)
{
    vec_launch<0>(st, n, VJacobiPre<T>{d, r, z}, sc, done);
}
template void jacobi_apply<double>(cudaStream_t, int, const double*, const double*, double*, const Scratch&,
                                   const int*);
template void jacobi_apply<float>(cudaStream_t, int, const float*, const float*, float*, const Scratch&, const int*);

}  // namespace jfg
