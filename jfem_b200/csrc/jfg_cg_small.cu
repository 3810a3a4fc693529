// Unpreconditioned CG (IterativeSolver.solveCG, IterativeSolver.java:48-103)
// for small systems in one launch: one 8-CTA thread-block cluster runs every
// iteration.  Each thread owns up to two rows and keeps their x, r, p and A p
// entries in registers; p is also written to global memory for the other
// rows' products; the two dot products of an iteration are reduced through
// distributed shared memory (every CTA sums the eight CTA partials in rank
// order, so every thread holds the same value and takes the same branch).
// Three cluster barriers per iteration replace the ~5 kernel launches of the
// graph-captured loop, whose launch latency dominates at this size.  The
// scalar recurrences and the stopping test are those of the multi-kernel CG
// (alpha = rz / p.Ap, beta = rr' / rr, `iter < maxit && ||r|| > tol`,
// NONFINITE on a non-finite residual); the loop is bounded by maxit.
#include <cooperative_groups.h>

#include "jfg_krylov.cuh"

namespace jfg {

namespace {

namespace cg = cooperative_groups;

constexpr int kCgCtas = 8;
constexpr int kCgThreads = 1024;
constexpr int kCgRowsPerThread = 2;

struct CgSmallArgs {
    int n;
    const int* ptr;
    const int* col;
    const double* val;
    const double* b;
    double* x;
    double* p;          // global copy of the direction (read by the products)
    Ctl* ctl;           // tol, maxit, hist, hist_cap in; iter, status, res_norm, ... out
};

// sum of one double over the cluster: warp shuffles, the CTA's warps in
// order, then the eight CTA partials (read through DSMEM) in rank order
__device__ __forceinline__ double cluster_sum(cg::cluster_group& cl, double v, double* warp_part, double* slot)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) warp_part[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < kCgThreads / 32; i++) s += warp_part[i];
        *slot = s;
    }
    cl.sync();
    double t = 0.0;
    for (int r = 0; r < kCgCtas; r++) t += *cl.map_shared_rank(slot, r);
    return t;
}

__device__ __forceinline__ double row_dot(const CgSmallArgs& a, int i, const double* v)
{
    double s = 0.0;
    for (int k = a.ptr[i]; k < a.ptr[i + 1]; k++) s += a.val[k] * __ldcg(v + a.col[k]);
    return s;
}

__device__ __forceinline__ bool stop_test(Ctl* c, double rn, int iter, int maxit, double tol, int* status)
{
    if (!isfinite(rn)) {
        *status = JFG_NONFINITE;
        return true;
    }
    if (!(rn > tol)) {
        *status = JFG_OK;
        return true;
    }
    if (iter >= maxit) {
        *status = JFG_NOT_CONVERGED;
        return true;
    }
    return false;
}

__global__ void __cluster_dims__(kCgCtas, 1, 1) __launch_bounds__(kCgThreads, 1) k_cg_small(CgSmallArgs a)
{
    __shared__ double warp_part[kCgThreads / 32];
    __shared__ double slots[2];
    cg::cluster_group cl = cg::this_cluster();
    const int tid = (int)cl.block_rank() * kCgThreads + threadIdx.x;
    const bool lead = tid == 0;
    Ctl* c = a.ctl;
    const double tol = c->tol;
    const int maxit = c->maxit;
    double* hist = c->hist;
    const int hist_cap = c->hist_cap;
    int rows[kCgRowsPerThread];
    double x[kCgRowsPerThread], r[kCgRowsPerThread], p[kCgRowsPerThread], ap[kCgRowsPerThread];
#pragma unroll
    for (int j = 0; j < kCgRowsPerThread; j++) {
        rows[j] = tid + j * kCgCtas * kCgThreads;
        x[j] = r[j] = p[j] = ap[j] = 0.0;
        if (rows[j] < a.n) x[j] = a.x[rows[j]];
    }
    // r = b - A x0, rr
    double part = 0.0;
#pragma unroll
    for (int j = 0; j < kCgRowsPerThread; j++)
        if (rows[j] < a.n) {
            r[j] = a.b[rows[j]] - row_dot(a, rows[j], a.x);
            part += r[j] * r[j];
        }
    double rr = cluster_sum(cl, part, warp_part, &slots[0]);
    double rz = rr;
    int iter = 0, status = JFG_NOT_CONVERGED, not_pd = 0;
    double res = sqrt(rr);
    bool done = stop_test(c, res, iter, maxit, tol, &status);
    // p = r
#pragma unroll
    for (int j = 0; j < kCgRowsPerThread; j++)
        if (rows[j] < a.n) {
            p[j] = r[j];
            a.p[rows[j]] = p[j];
        }
    cl.sync();
    while (!done) {
        // A p and p.Ap
        part = 0.0;
#pragma unroll
        for (int j = 0; j < kCgRowsPerThread; j++)
            if (rows[j] < a.n) {
                ap[j] = row_dot(a, rows[j], a.p);
                part += p[j] * ap[j];
            }
        const double pap = cluster_sum(cl, part, warp_part, &slots[1]);
        const double alpha = rz / pap;
        if (!(pap > 0)) not_pd = 1;
        // x += p alpha, r -= A p alpha, ||r||^2
        part = 0.0;
#pragma unroll
        for (int j = 0; j < kCgRowsPerThread; j++)
            if (rows[j] < a.n) {
                x[j] = x[j] + p[j] * alpha;
                r[j] = r[j] - ap[j] * alpha;
                part += r[j] * r[j];
            }
        const double rr_new = cluster_sum(cl, part, warp_part, &slots[0]);
        iter++;
        const double beta = rr_new / rr;
        rz = rr_new;
        rr = rr_new;
        res = sqrt(rr_new);
        if (lead && hist && iter <= hist_cap) hist[iter - 1] = res;
        done = stop_test(c, res, iter, maxit, tol, &status);
        if (done) break;
        // p = r + p beta
#pragma unroll
        for (int j = 0; j < kCgRowsPerThread; j++)
            if (rows[j] < a.n) {
                p[j] = r[j] + p[j] * beta;
                a.p[rows[j]] = p[j];
            }
        cl.sync();
    }
#pragma unroll
    for (int j = 0; j < kCgRowsPerThread; j++)
        if (rows[j] < a.n) a.x[rows[j]] = x[j];
    if (lead) {
        c->iter = iter;
        c->status = status;
        c->res_norm = res;
        c->rr = rr;
        c->rz = rz;
        c->not_pd = not_pd;
        c->done = 1;
    }
    cl.sync();      // no CTA leaves while another may still read its shared memory
}

}  // namespace

bool cg_small_fits(const Matrix* A)
{
    const char* e = getenv("JFEM_SMALL_CG");        // "0": always the multi-kernel loop
    return !(e && e[0] == '0') && A->rows <= kCgCtas * kCgThreads * kCgRowsPerThread;
}

// Runs the whole CG; the control block w.ctl[0] holds tol / maxit / history
// on entry and the results on return (as the multi-kernel loop leaves them).
void run_cg_small(SolverWork& w, Matrix* A, const double* b, double* x)
{
    cudaStream_t st = w.c->stream;
    w.v64[0].alloc((size_t)A->rows);
    CgSmallArgs a{A->rows, A->csr_ptr.p, A->csr_col.p, A->csr_val.p, b, x, w.v64[0].p, w.ctl.p};
    k_cg_small<<<kCgCtas, kCgThreads, 0, st>>>(a);
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

}  // namespace jfg
