// Dense FP64 LU with partial pivoting on the device: the coarsest multigrid
// level, the drop-in dense solve and dense inverses.
//
// Right-looking LU: for each column k one CTA picks the pivot (largest |a_ik|,
// lowest index on ties), swaps rows and scales the column; a grid then applies
// the rank-1 update to the trailing block.  Triangular solves run one CTA per
// right-hand side, column-oriented.
#include "jfg_mg.cuh"

namespace jfg {

namespace {

__global__ void k_lu_pivot(int n, double* A, int* piv, int k, int* info)
{
    __shared__ double best[1024];
    __shared__ int bidx[1024];
    double b = -1.0;
    int bi = k;
    for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
        double v = fabs(A[(size_t)i * n + k]);
        if (v > b) { b = v; bi = i; }
    }
    best[threadIdx.x] = b;
    bidx[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            double o = best[threadIdx.x + s];
            int oi = bidx[threadIdx.x + s];
            if (o > best[threadIdx.x] || (o == best[threadIdx.x] && oi < bidx[threadIdx.x])) {
                best[threadIdx.x] = o;
                bidx[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    int p = bidx[0];
    if (threadIdx.x == 0) {
        piv[k] = p;
        if (!(best[0] > 0.0)) *info = 1;
    }
    if (!(best[0] > 0.0)) return;
    if (p != k)
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            double t = A[(size_t)k * n + j];
            A[(size_t)k * n + j] = A[(size_t)p * n + j];
            A[(size_t)p * n + j] = t;
        }
    __syncthreads();
    double inv = 1.0 / A[(size_t)k * n + k];
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + k] *= inv;
}

__global__ void k_lu_update(int n, double* A, int k, const int* info)
{
    if (*info) return;
    int m = n - k - 1;
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m * m) return;
    int i = k + 1 + (int)(idx / m);
    int j = k + 1 + (int)(idx % m);
    A[(size_t)i * n + j] -= A[(size_t)i * n + k] * A[(size_t)k * n + j];
}

// One CTA per right-hand side column c: B[:, c] <- A^-1 B[:, c], with B
// row-major n x nrhs (column c strided by nrhs).
__global__ void k_lu_solve(int n, const double* LU, const int* piv, double* B, int nrhs)
{
    int c = blockIdx.x;
    double* x = B + c;
    if (threadIdx.x == 0)
        for (int k = 0; k < n; k++)
            if (piv[k] != k) {
                double t = x[(size_t)k * nrhs];
                x[(size_t)k * nrhs] = x[(size_t)piv[k] * nrhs];
                x[(size_t)piv[k] * nrhs] = t;
            }
    __syncthreads();
    for (int k = 0; k < n; k++) {           // forward, unit lower
        double xk = x[(size_t)k * nrhs];
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) x[(size_t)i * nrhs] -= LU[(size_t)i * n + k] * xk;
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; k--) {      // backward
        if (threadIdx.x == 0) x[(size_t)k * nrhs] /= LU[(size_t)k * n + k];
        __syncthreads();
        double xk = x[(size_t)k * nrhs];
        for (int i = threadIdx.x; i < k; i += blockDim.x) x[(size_t)i * nrhs] -= LU[(size_t)i * n + k] * xk;
        __syncthreads();
    }
}

__global__ void k_identity(int n, double* B)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * n) return;
    B[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

int lu_factor(Context* c, int n, double* A, int* piv, int* info)
{
    cudaStream_t st = c->stream;
    JFG_CUDA(cudaMemsetAsync(info, 0, sizeof(int), st));
    for (int k = 0; k < n; k++) {
        k_lu_pivot<<<1, 1024, 0, st>>>(n, A, piv, k, info);
        int m = n - k - 1;
        if (m > 0) {
            int64_t tot = (int64_t)m * m;
            k_lu_update<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, A, k, info);
        }
    }
    JFG_CUDA(cudaGetLastError());
    int h = 0;
    JFG_CUDA(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    return h ? JFG_ERR_SINGULAR : JFG_OK;
}

}  // namespace

int dense_inverse_device(Context* c, int n, double* d_A, double* d_inv)
{
    if (n == 0) return JFG_OK;
    DevBuf<int> piv, info;
    piv.alloc(n);
    info.alloc(1);
    int st = lu_factor(c, n, d_A, piv.p, info.p);
    if (st != JFG_OK) return st;
    int64_t tot = (int64_t)n * n;
    k_identity<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(n, d_inv);
    k_lu_solve<<<n, 256, 0, c->stream>>>(n, d_A, piv.p, d_inv, n);
    JFG_CUDA(cudaGetLastError());
    JFG_CUDA(cudaStreamSynchronize(c->stream));
    return JFG_OK;
}

int dense_solve_device(Context* c, int n, double* d_A, const double* d_b, double* d_x)
{
    if (n == 0) return JFG_OK;
    DevBuf<int> piv, info;
    piv.alloc(n);
    info.alloc(1);
    int st = lu_factor(c, n, d_A, piv.p, info.p);
    if (st != JFG_OK) return st;
    if (d_x != d_b) JFG_CUDA(cudaMemcpyAsync(d_x, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    k_lu_solve<<<1, 1024, 0, c->stream>>>(n, d_A, piv.p, d_x, 1);
    JFG_CUDA(cudaGetLastError());
    JFG_CUDA(cudaStreamSynchronize(c->stream));
    return JFG_OK;
}

}  // namespace jfg
