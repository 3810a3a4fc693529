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

#include <algorithm>
#include <vector>

#include "jfg_krylov.cuh"

namespace jfg {

namespace {

namespace cg = cooperative_groups;

constexpr int kCgCtas = 8;
constexpr int kCgThreads = 1024;
constexpr int kCgRowsPerThread = 2;
constexpr int kSmThreads = 512;      // shared-memory variant: 512 threads x 4 rows
constexpr int kSmRows = 4;

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
template <int THREADS = kCgThreads>
__device__ __forceinline__ double cluster_sum(cg::cluster_group& cl, double v, double* warp_part, double* slot)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) warp_part[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < THREADS / 32; i++) s += warp_part[i];
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

// The same iteration with the matrix rows and a replica of p in shared
// memory: CTA q owns the contiguous rows [q R, (q + 1) R) and keeps their CSR
// slice; every thread stores the new p of its rows into all eight CTAs'
// replicas (DSMEM stores) before the barrier, so the products read only
// shared memory.  Used when the slice and the replica fit one CTA's shared
// memory.
struct CgSmemLayout {
    int R;              // rows per CTA
    int max_nnz;        // largest CSR slice of a CTA
    size_t bytes;       // dynamic shared memory per CTA
};

__global__ void __cluster_dims__(kCgCtas, 1, 1) __launch_bounds__(kSmThreads, 1)
    k_cg_small_smem(CgSmallArgs a, int R, int max_nnz)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double warp_part[kSmThreads / 32];
    __shared__ double slots[2];
    double* p_all = reinterpret_cast<double*>(smem);                       // n
    double* lval = p_all + a.n;                                            // max_nnz
    int* lptr = reinterpret_cast<int*>(lval + max_nnz);                    // R + 1
    int* lcol = lptr + R + 1;                                              // max_nnz
    cg::cluster_group cl = cg::this_cluster();
    const int q = (int)cl.block_rank();
    const int r0 = q * R, r1 = min(a.n, r0 + R);
    const int nr = r1 > r0 ? r1 - r0 : 0;
    const bool lead = q == 0 && threadIdx.x == 0;
    Ctl* c = a.ctl;
    const double tol = c->tol;
    const int maxit = c->maxit;
    double* hist = c->hist;
    const int hist_cap = c->hist_cap;
    // the CTA's CSR slice, with row pointers relative to its first entry
    const int e0 = nr ? a.ptr[r0] : 0;
    const int ne = nr ? a.ptr[r1] - e0 : 0;
    for (int i = threadIdx.x; i <= nr; i += kSmThreads) lptr[i] = a.ptr[r0 + i] - e0;
    for (int k = threadIdx.x; k < ne; k += kSmThreads) {
        lcol[k] = a.col[e0 + k];
        lval[k] = a.val[e0 + k];
    }
    int rows[kSmRows];
    double x[kSmRows], r[kSmRows], p[kSmRows], ap[kSmRows];
#pragma unroll
    for (int j = 0; j < kSmRows; j++) {
        rows[j] = threadIdx.x + j * kSmThreads;               // local row
        x[j] = r[j] = p[j] = ap[j] = 0.0;
        if (rows[j] < nr) x[j] = a.x[r0 + rows[j]];
    }
    __syncthreads();
    auto local_dot = [&](int lr, const double* v) {
        double s = 0.0;
        for (int k = lptr[lr]; k < lptr[lr + 1]; k++) s += lval[k] * v[lcol[k]];
        return s;
    };
    // r = b - A x0 (x0 read from global once), rr
    double part = 0.0;
#pragma unroll
    for (int j = 0; j < kSmRows; j++)
        if (rows[j] < nr) {
            double s = 0.0;
            for (int k = lptr[rows[j]]; k < lptr[rows[j] + 1]; k++) s += lval[k] * a.x[lcol[k]];
            r[j] = a.b[r0 + rows[j]] - s;
            part += r[j] * r[j];
        }
    double rr = cluster_sum<kSmThreads>(cl, part, warp_part, &slots[0]);
    double rz = rr;
    int iter = 0, status = JFG_NOT_CONVERGED, not_pd = 0;
    double res = sqrt(rr);
    bool done = stop_test(c, res, iter, maxit, tol, &status);
    auto broadcast_p = [&]() {
#pragma unroll
        for (int j = 0; j < kSmRows; j++)
            if (rows[j] < nr)
                for (int t = 0; t < kCgCtas; t++) *cl.map_shared_rank(p_all + r0 + rows[j], t) = p[j];
    };
#pragma unroll
    for (int j = 0; j < kSmRows; j++) p[j] = r[j];
    broadcast_p();
    cl.sync();
    while (!done) {
        part = 0.0;
#pragma unroll
        for (int j = 0; j < kSmRows; j++)
            if (rows[j] < nr) {
                ap[j] = local_dot(rows[j], p_all);
                part += p[j] * ap[j];
            }
        const double pap = cluster_sum<kSmThreads>(cl, part, warp_part, &slots[1]);
        const double alpha = rz / pap;
        if (!(pap > 0)) not_pd = 1;
        part = 0.0;
#pragma unroll
        for (int j = 0; j < kSmRows; j++)
            if (rows[j] < nr) {
                x[j] = x[j] + p[j] * alpha;
                r[j] = r[j] - ap[j] * alpha;
                part += r[j] * r[j];
            }
        const double rr_new = cluster_sum<kSmThreads>(cl, part, warp_part, &slots[0]);
        iter++;
        const double beta = rr_new / rr;
        rz = rr_new;
        rr = rr_new;
        res = sqrt(rr_new);
        if (lead && hist && iter <= hist_cap) hist[iter - 1] = res;
        done = stop_test(c, res, iter, maxit, tol, &status);
        if (done) break;
#pragma unroll
        for (int j = 0; j < kSmRows; j++)
            if (rows[j] < nr) p[j] = r[j] + p[j] * beta;
        broadcast_p();
        cl.sync();
    }
#pragma unroll
    for (int j = 0; j < kSmRows; j++)
        if (rows[j] < nr) a.x[r0 + rows[j]] = x[j];
    if (lead) {
        c->iter = iter;
        c->status = status;
        c->res_norm = res;
        c->rr = rr;
        c->rz = rz;
        c->not_pd = not_pd;
        c->done = 1;
    }
    cl.sync();      // no CTA leaves while another may still read or write its shared memory
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
    const int n = A->rows;
    w.v64[0].alloc((size_t)n);
    CgSmallArgs a{n, A->csr_ptr.p, A->csr_col.p, A->csr_val.p, b, x, w.v64[0].p, w.ctl.p};
    // shared-memory variant when a CTA's CSR slice and the p replica fit
    const int R = (n + kCgCtas - 1) / kCgCtas;
    if (A->cg_small_nnz < 0) {      // once per matrix: the largest row block's CSR slice
        std::vector<int> ptr((size_t)n + 1);
        JFG_CUDA(cudaMemcpyAsync(ptr.data(), A->csr_ptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
        JFG_CUDA(cudaStreamSynchronize(st));
        int mx = 0;
        for (int q = 0; q < kCgCtas; q++) {
            const int r0 = std::min(n, q * R), r1 = std::min(n, r0 + R);
            mx = std::max(mx, ptr[r1] - ptr[r0]);
        }
        A->cg_small_nnz = mx;
    }
    const int max_nnz = A->cg_small_nnz;
    const size_t bytes = sizeof(double) * ((size_t)n + max_nnz) + sizeof(int) * ((size_t)R + 1 + max_nnz) + 16;
    constexpr size_t kSmemCap = (size_t)200 * 1024;
    const char* e = getenv("JFEM_SMALL_CG_SMEM");
    const bool smem_ok = !(e && e[0] == '0') && R <= kSmThreads * kSmRows && bytes <= kSmemCap;
    if (smem_ok) {
        static int attr_dev = -1;     // the opt-in shared memory size, set once per device
        int dev = 0;
        JFG_CUDA(cudaGetDevice(&dev));
        if (attr_dev != dev) {
            JFG_CUDA(cudaFuncSetAttribute(k_cg_small_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemCap));
            attr_dev = dev;
        }
        k_cg_small_smem<<<kCgCtas, kSmThreads, bytes, st>>>(a, R, max_nnz);
    } else {
        k_cg_small<<<kCgCtas, kCgThreads, 0, st>>>(a);
    }
    JFG_CUDA(cudaGetLastError());
    note_launch();
}

}  // namespace jfg
