// Sparse matrix-matrix products on the device (set-up of Galerkin coarse
// operators):
//
//   C = A B     SparseMatrix.mmMul (Core/src/main/java/linalg/SparseMatrix.java:549-593)
//   C = A^T B   Matrix.tmMul       (Core/src/main/java/linalg/Matrix.java:142-148)
//   C = (R A) P / (P^T A) P        AMGSpace.createSystems (multigrid/AMGSpace.java:60-78),
//                                  MGPreconditionerInterface.AMGFromMatrix
//                                  (multigrid/MGPreconditionerInterface.java:387-402)
//
// Method: expand - sort - sum.  Each row of A expands into its products
// a_ik * b_kj (one rounding each, in k-major, j-minor order), the products of
// a chunk of rows are sorted by (row, column) with a stable radix sort (equal
// keys keep their k order), and every run of equal keys is summed from 0 left
// to right by one thread, without fused multiply-adds -- each entry of C is
// sum_k (a_ik * b_kj) in ascending k, as a Java loop `contraction += row[k] *
// b` computes it.  Entries whose sum is exactly zero are dropped (the
// reference's SparseMatrix.add skips zero values, SparseMatrix.java:289).
// The reference iterates B's columns in HashMap order, so its per-entry
// summation order is hash-defined; the two agree to rounding.
//
// Rows are processed in chunks of at most chunk_products() products so that
// scratch stays bounded; chunks are row-contiguous, so their outputs
// concatenate into globally sorted keys.
#include <cub/cub.cuh>

#include <algorithm>
#include <memory>
#include <vector>

#include "jfg_kernels.cuh"

namespace jfg {

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// products per chunk: 64 Mi (1 GiB of key/value pairs); JFEM_SPGEMM_CHUNK
// overrides it (tests use small chunks to exercise the concatenation)
int64_t chunk_products()
{
    const char* e = getenv("JFEM_SPGEMM_CHUNK");
    const long long v = e ? atoll(e) : 0;
    return v > 0 ? (int64_t)v : ((int64_t)1 << 26);
}

// products of each row of A: sum over its entries k of the length of row k of B
__global__ void k_gemm_count(int rows, const int* __restrict__ aptr, const int* __restrict__ acol,
                             const int* __restrict__ bptr, int64_t* __restrict__ cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    int64_t s = 0;
    for (int p = aptr[i]; p < aptr[i + 1]; p++) {
        int k = acol[p];
        s += bptr[k + 1] - bptr[k];
    }
    cnt[i] = s;
}

// One warp per row i of [r0, r1): writes the products of row i at
// off[i] - off[r0], keyed by (i - r0) * ncols + j.
__global__ void k_gemm_expand(int r0, int r1, int ncols, const int64_t* __restrict__ off,
                              const int* __restrict__ aptr, const int* __restrict__ acol,
                              const double* __restrict__ aval, const int* __restrict__ bptr,
                              const int* __restrict__ bcol, const double* __restrict__ bval,
                              uint64_t* __restrict__ key, double* __restrict__ val)
{
    const int warp = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int i = r0 + warp;
    if (i >= r1) return;
    int64_t pos = off[i] - off[r0];
    const uint64_t rk = (uint64_t)(i - r0) * (uint64_t)ncols;
    for (int p = aptr[i]; p < aptr[i + 1]; p++) {
        const int k = acol[p];
        const double a = aval[p];
        const int b0 = bptr[k], len = bptr[k + 1] - b0;
        for (int t = lane; t < len; t += 32) {
            key[pos + t] = rk + (uint64_t)bcol[b0 + t];
            val[pos + t] = __dmul_rn(a, bval[b0 + t]);
        }
        pos += len;
    }
}

// One thread per run of equal keys: the in-order sum of its products, and a
// keep flag (the sum is not exactly zero).  Keys are shifted back to global
// row numbering.
__global__ void k_gemm_sum_runs(const int64_t* __restrict__ nruns, const int64_t* __restrict__ rstart,
                                const int* __restrict__ rlen, const uint64_t* __restrict__ ukey,
                                const double* __restrict__ val, uint64_t key_base, uint64_t* __restrict__ okey,
                                double* __restrict__ oval, char* __restrict__ keep)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= *nruns) return;
    const int64_t s0 = rstart[r];
    const int n = rlen[r];
    double s = 0.0;
    for (int t = 0; t < n; t++) s = __dadd_rn(s, val[s0 + t]);
    okey[r] = ukey[r] + key_base;
    oval[r] = s;
    keep[r] = s != 0.0;
}

int key_bits(uint64_t maxkey)
{
    int b = 1;
    while (b < 64 && (1ULL << b) < maxkey) b++;
    return b;
}

}  // namespace

// Carves aligned sub-buffers out of one workspace allocation; a first pass
// with base == nullptr measures the bytes needed.
struct Carve {
    char* base;
    size_t used = 0;
    template <typename T>
    T* take(size_t n)
    {
        used = (used + 255) & ~(size_t)255;
        T* r = base ? (T*)(base + used) : nullptr;
        used += (n ? n : 1) * sizeof(T);
        return r;
    }
};

// C = A B on the device; sell = false leaves out the SpMV layout (products
// used only as inputs of further products).  Scratch lives in the context's
// grow-only workspaces, so repeated products allocate nothing but C.
Matrix* matrix_mmmul(Matrix* A, Matrix* B, bool sell)
{
    JFG_CHECK(A->cols == B->rows, JFG_ERR_BAD_ARG, "Incompatible sizes");
    Context* c = A->ctx;
    cudaStream_t s = c->stream;
    const int rows = A->rows, ncols = B->cols;
    if (rows == 0 || ncols == 0 || A->nnz == 0 || B->nnz == 0)
        return matrix_from_sorted_keys(c, rows, ncols, 0, nullptr, nullptr, sell);

    // products per row and their offsets
    size_t scan_bytes = 0;
    JFG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (int64_t*)nullptr, (int64_t*)nullptr, rows + 1, s));
    Carve m0{nullptr};
    m0.take<int64_t>((size_t)rows + 1);
    m0.take<int64_t>((size_t)rows + 1);
    m0.take<char>(scan_bytes);
    c->gemm_rows.alloc(m0.used);
    Carve c0{c->gemm_rows.p};
    int64_t* cnt = c0.take<int64_t>((size_t)rows + 1);
    int64_t* off = c0.take<int64_t>((size_t)rows + 1);
    char* scan_tmp = c0.take<char>(scan_bytes);
    JFG_CUDA(cudaMemsetAsync(cnt + rows, 0, sizeof(int64_t), s));
    k_gemm_count<<<nblk(rows), 256, 0, s>>>(rows, A->csr_ptr.p, A->csr_col.p, B->csr_ptr.p, cnt);
    JFG_CUDA(cudaGetLastError());
    JFG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, cnt, off, rows + 1, s));
    std::vector<int64_t> h_off((size_t)rows + 1);
    JFG_CUDA(cudaMemcpyAsync(h_off.data(), off, sizeof(int64_t) * (rows + 1), cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));

    // row chunks of at most `chunk` products (a longer single row is a chunk of its own)
    const int64_t chunk = chunk_products();
    std::vector<int> cuts{0};
    for (int i = 0; i < rows;) {
        int j = i + 1;
        while (j < rows && h_off[j + 1] - h_off[i] <= chunk) j++;
        cuts.push_back(j);
        i = j;
    }
    int64_t cap = 1;
    for (size_t q = 0; q + 1 < cuts.size(); q++) cap = std::max(cap, h_off[cuts[q + 1]] - h_off[cuts[q]]);
    const bool one_chunk = cuts.size() == 2;

    // scratch of the cub passes, sized for the largest chunk
    const int max_bits = key_bits((uint64_t)std::max(1, rows) * (uint64_t)ncols);
    size_t t_sort = 0, t_rle = 0, t_scan = 0, t_sel1 = 0, t_sel2 = 0;
    {
        uint64_t* k = nullptr;
        double* v = nullptr;
        int* rl = nullptr;
        int64_t* i64 = nullptr;
        char* f = nullptr;
        JFG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, k, k, v, v, cap, 0, max_bits, s));
        JFG_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, t_rle, k, k, rl, i64, cap, s));
        JFG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, rl, i64, cap, s));
        JFG_CUDA(cub::DeviceSelect::Flagged(nullptr, t_sel1, k, f, k, i64, cap, s));
        JFG_CUDA(cub::DeviceSelect::Flagged(nullptr, t_sel2, v, f, v, i64, cap, s));
    }
    const size_t t_max = std::max({t_sort, t_rle, t_scan, t_sel1, t_sel2});
    auto layout = [&](Carve& w, uint64_t*& key, uint64_t*& key2, uint64_t*& ukey, double*& val, double*& val2,
                      int*& rlen, int64_t*& rstart, int64_t*& nrun, uint64_t*& okey, double*& oval, char*& keep,
                      char*& tmp) {
        key = w.take<uint64_t>((size_t)cap);
        key2 = w.take<uint64_t>((size_t)cap);
        ukey = w.take<uint64_t>((size_t)cap);
        val = w.take<double>((size_t)cap);
        val2 = w.take<double>((size_t)cap);
        rlen = w.take<int>((size_t)cap);
        rstart = w.take<int64_t>((size_t)cap);
        nrun = w.take<int64_t>(2);
        okey = w.take<uint64_t>((size_t)cap);
        oval = w.take<double>((size_t)cap);
        keep = w.take<char>((size_t)cap);
        tmp = w.take<char>(t_max);
    };
    uint64_t *key, *key2, *ukey, *okey;
    double *val, *val2, *oval;
    int* rlen;
    int64_t *rstart, *nrun;
    char *keep, *tmp;
    Carve m1{nullptr};
    layout(m1, key, key2, ukey, val, val2, rlen, rstart, nrun, okey, oval, keep, tmp);
    c->gemm_ws.alloc(m1.used);
    Carve w{c->gemm_ws.p};
    layout(w, key, key2, ukey, val, val2, rlen, rstart, nrun, okey, oval, keep, tmp);

    std::vector<std::unique_ptr<DevBuf<uint64_t>>> part_key;
    std::vector<std::unique_ptr<DevBuf<double>>> part_val;
    std::vector<int64_t> part_n;
    int64_t total = 0;
    for (size_t q = 0; q + 1 < cuts.size(); q++) {
        const int r0 = cuts[q], r1 = cuts[q + 1];
        const int64_t nprod = h_off[r1] - h_off[r0];
        if (nprod == 0) continue;
        k_gemm_expand<<<nblk((int64_t)(r1 - r0) * 32), 256, 0, s>>>(r0, r1, ncols, off, A->csr_ptr.p, A->csr_col.p,
                                                                    A->csr_val.p, B->csr_ptr.p, B->csr_col.p,
                                                                    B->csr_val.p, key, val);
        JFG_CUDA(cudaGetLastError());
        const int bits = key_bits((uint64_t)(r1 - r0) * (uint64_t)ncols);
        size_t tb = t_max;
        JFG_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, val, val2, nprod, 0, bits, s));
        tb = t_max;
        JFG_CUDA(cub::DeviceRunLengthEncode::Encode(tmp, tb, key2, ukey, rlen, nrun, nprod, s));
        int64_t h_runs = 0;
        JFG_CUDA(cudaMemcpyAsync(&h_runs, nrun, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        JFG_CUDA(cudaStreamSynchronize(s));
        tb = t_max;
        JFG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, rlen, rstart, h_runs, s));
        k_gemm_sum_runs<<<nblk(h_runs), 256, 0, s>>>(nrun, rstart, rlen, ukey, val2, (uint64_t)r0 * (uint64_t)ncols,
                                                    okey, oval, keep);
        JFG_CUDA(cudaGetLastError());
        // keep the nonzero sums
        tb = t_max;
        JFG_CUDA(cub::DeviceSelect::Flagged(tmp, tb, okey, keep, key, nrun + 1, h_runs, s));
        tb = t_max;
        JFG_CUDA(cub::DeviceSelect::Flagged(tmp, tb, oval, keep, val, nrun + 1, h_runs, s));
        int64_t h_keep = 0;
        JFG_CUDA(cudaMemcpyAsync(&h_keep, nrun + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        JFG_CUDA(cudaStreamSynchronize(s));
        if (one_chunk) return matrix_from_sorted_keys(c, rows, ncols, h_keep, key, val, sell);
        if (!h_keep) continue;
        part_key.emplace_back(new DevBuf<uint64_t>());
        part_val.emplace_back(new DevBuf<double>());
        part_key.back()->alloc((size_t)h_keep);
        part_val.back()->alloc((size_t)h_keep);
        JFG_CUDA(cudaMemcpyAsync(part_key.back()->p, key, sizeof(uint64_t) * h_keep, cudaMemcpyDeviceToDevice, s));
        JFG_CUDA(cudaMemcpyAsync(part_val.back()->p, val, sizeof(double) * h_keep, cudaMemcpyDeviceToDevice, s));
        part_n.push_back(h_keep);
        total += h_keep;
    }
    DevBuf<uint64_t> all_key;
    DevBuf<double> all_val;
    all_key.alloc(total ? (size_t)total : 1);
    all_val.alloc(total ? (size_t)total : 1);
    int64_t at = 0;
    for (size_t q = 0; q < part_n.size(); q++) {
        JFG_CUDA(cudaMemcpyAsync(all_key.p + at, part_key[q]->p, sizeof(uint64_t) * part_n[q],
                                 cudaMemcpyDeviceToDevice, s));
        JFG_CUDA(cudaMemcpyAsync(all_val.p + at, part_val[q]->p, sizeof(double) * part_n[q],
                                 cudaMemcpyDeviceToDevice, s));
        at += part_n[q];
    }
    JFG_CUDA(cudaStreamSynchronize(s));
    return matrix_from_sorted_keys(c, rows, ncols, total, all_key.p, all_val.p, sell);
}

// C = A^T B (Matrix.tmMul: transpose().mmMul(B)).
Matrix* matrix_tmmul(Matrix* A, Matrix* B, bool sell)
{
    JFG_CHECK(A->rows == B->rows, JFG_ERR_BAD_ARG, "Incompatible sizes");
    return matrix_mmmul(matrix_transpose(A), B, sell);
}

// C = (R A) P, with R = P^T when R is null (the association of the reference:
// P.tmMul(A).mmMul(P), resp. R.mmMul(A).mmMul(P)).
Matrix* matrix_galerkin(Matrix* R, Matrix* A, Matrix* P)
{
    JFG_CHECK(A->rows == A->cols, JFG_ERR_BAD_ARG, "Galerkin product of a non-square matrix");
    JFG_CHECK(P->rows == A->cols, JFG_ERR_BAD_ARG, "Incompatible sizes");
    JFG_CHECK(!R || (R->cols == A->rows && R->rows == P->cols), JFG_ERR_BAD_ARG, "Incompatible sizes");
    Matrix* S = R ? matrix_mmmul(R, A, false) : matrix_tmmul(P, A, false);
    Matrix* C = nullptr;
    try {
        C = matrix_mmmul(S, P, true);
    } catch (...) {
        delete S;
        throw;
    }
    delete S;
    return C;
}

}  // namespace jfg
