// COO -> row-block CSR conversion on the device, transposes, precision
// copies and the plain SpMV entry points.
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>

#include "jfg_kernels.cuh"

namespace jfg {

namespace {

__global__ void k_make_keys(int64_t nnz, const int* ri, const int* ci, int rows, int cols, uint64_t* key,
                            int* bad)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    int r = ri[k], c = ci[k];
    if (r < 0 || r >= rows || c < 0 || c >= cols) {
        atomicExch(bad, 1);
        r = 0;
        c = 0;
    }
    key[k] = (uint64_t)r * (uint64_t)cols + (uint64_t)c;
}

__global__ void k_nonzero_flags(int64_t m, const double* v, char* f)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) f[i] = v[i] != 0.0;
}

__global__ void k_row_counts(int64_t m, const uint64_t* key, int cols, int* cnt)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    atomicAdd(cnt + (int)(key[k] / (uint64_t)cols), 1);
}

__global__ void k_scatter_padded(int64_t m, const uint64_t* key, const double* v, int cols, const int64_t* oldptr,
                                 const int* newptr, int* col, double* val)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    int r = (int)(key[k] / (uint64_t)cols);
    int c = (int)(key[k] % (uint64_t)cols);
    int64_t pos = newptr[r] + (k - oldptr[r]);
    col[pos] = c;
    val[pos] = v[k];
}

__global__ void k_diag(int rows, int cols, const int* rowptr, const int* col, const double* val, double* d)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double s = 0;
    if (r < cols)
        for (int k = rowptr[r]; k < rowptr[r + 1]; k++)
            if (col[k] == r) s += val[k];
    d[r] = s;
}

__global__ void k_expand_rows(int rows, const int* rowptr, int* ri_out, const int64_t* dense_off)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    int64_t o = dense_off[r];
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) ri_out[o + (k - rowptr[r])] = r;
}

__global__ void k_compact(int rows, const int* rowptr, const int* col, const double* val, const int64_t* dense_off,
                          int* ci_out, double* v_out)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    int64_t o = dense_off[r];
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) {
        ci_out[o + (k - rowptr[r])] = col[k];
        v_out[o + (k - rowptr[r])] = val[k];
    }
}

__global__ void k_to_f32(int64_t n, const double* a, float* b)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void k_to_bf16(int64_t n, const double* a, __nv_bfloat16* b)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn((float)a[i]);
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

int choose_lpr_log2(double avg)
{
    if (avg <= 3) return 1;
    if (avg <= 12) return 2;
    if (avg <= 24) return 3;
    if (avg <= 48) return 4;
    return 5;
}

}  // namespace

std::atomic<unsigned long long> g_launches{0};

bool use_pdl()
{
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("JFEM_PDL");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

uint64_t next_uid()
{
    static std::atomic<uint64_t> ctr{1};
    return ctr.fetch_add(1);
}

Matrix::Matrix() : uid(next_uid()) {}
Matrix::~Matrix() { delete transposed; }

// Builds the padded row-block layout from merged, sorted, zero-free COO that
// is already on the device (keys = row*cols+col, ascending).
static Matrix* build_from_sorted(Context* c, int rows, int cols, int64_t m, const uint64_t* d_key,
                                 const double* d_val)
{
    cudaStream_t s = c->stream;
    auto* M = new Matrix();
    M->ctx = c;
    M->rows = rows;
    M->cols = cols;
    M->nnz = m;
    DevBuf<int> cnt;
    cnt.alloc((size_t)rows + 1);
    JFG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * ((size_t)rows + 1), s));
    if (m) k_row_counts<<<nblk(m), 256, 0, s>>>(m, d_key, cols, cnt.p);
    JFG_CUDA(cudaGetLastError());
    std::vector<int> h_cnt(rows + 1);
    JFG_CUDA(cudaMemcpyAsync(h_cnt.data(), cnt.p, sizeof(int) * rows, cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));
    // merged offsets and the padded row-block layout
    std::vector<int64_t> oldptr(rows + 1, 0);
    for (int r = 0; r < rows; r++) oldptr[r + 1] = oldptr[r] + h_cnt[r];
    std::vector<int> rb;
    std::vector<int> newptr(rows + 1, 0);
    int64_t off = 0;
    int r = 0;
    rb.push_back(0);
    // Greedy partition into row blocks of <= kBlockRows rows and
    // <= kBlockNnz - 8 nonzeros (a longer row forms a block of its own).  Each
    // block starts on an 8-element boundary (16-byte aligned bulk copies for
    // every value type); the <= 7 padding slots before it hold column 0 /
    // value 0 and are summed into the previous block's last row as exact zeros.
    while (r < rows) {
        off = (off + 7) & ~int64_t(7);
        int start = r;
        int64_t bnnz = 0;
        while (r < rows && r - start < kBlockRows) {
            int len = h_cnt[r];
            if (r > start && bnnz + len > kBlockNnz - 8) break;
            newptr[r] = (int)(off + bnnz);
            bnnz += len;
            r++;
            if (bnnz > kBlockNnz - 8) break;
        }
        off += bnnz;
        rb.push_back(r);
    }
    if (rows == 0) rb.push_back(0);
    newptr[rows] = (int)off;
    JFG_CHECK(off < (int64_t)INT32_MAX - 64, JFG_ERR_UNSUPPORTED, "matrix has more than 2^31 nonzeros");
    M->nblocks = (int)rb.size() - 1;
    M->nnz_padded = off + 16;   // slack: bulk copies round the last block up to 8 elements
    M->rb.alloc(rb.size());
    M->rowptr.alloc((size_t)rows + 1);
    M->col.alloc((size_t)M->nnz_padded);
    M->val.alloc((size_t)M->nnz_padded);
    JFG_CUDA(cudaMemcpyAsync(M->rb.p, rb.data(), sizeof(int) * rb.size(), cudaMemcpyHostToDevice, s));
    JFG_CUDA(cudaMemcpyAsync(M->rowptr.p, newptr.data(), sizeof(int) * (rows + 1), cudaMemcpyHostToDevice, s));
    JFG_CUDA(cudaMemsetAsync(M->col.p, 0, sizeof(int) * M->nnz_padded, s));
    JFG_CUDA(cudaMemsetAsync(M->val.p, 0, sizeof(double) * M->nnz_padded, s));
    DevBuf<int64_t> d_old;
    d_old.alloc((size_t)rows + 1);
    JFG_CUDA(cudaMemcpyAsync(d_old.p, oldptr.data(), sizeof(int64_t) * (rows + 1), cudaMemcpyHostToDevice, s));
    if (m) k_scatter_padded<<<nblk(m), 256, 0, s>>>(m, d_key, d_val, cols, d_old.p, M->rowptr.p, M->col.p, M->val.p);
    JFG_CUDA(cudaGetLastError());
    M->diag.alloc((size_t)rows);
    if (rows) k_diag<<<nblk(rows), 256, 0, s>>>(rows, cols, M->rowptr.p, M->col.p, M->val.p, M->diag.p);
    JFG_CUDA(cudaGetLastError());
    M->lpr = 1 << choose_lpr_log2(rows ? (double)m / rows : 1.0);
    JFG_CUDA(cudaStreamSynchronize(s));
    return M;
}

// COO on the device -> Matrix (sort, merge duplicates, drop zeros).
static Matrix* from_device_coo(Context* c, int rows, int cols, int64_t nnz, const int* d_ri, const int* d_ci,
                               const double* d_v, bool keep_zeros)
{
    cudaStream_t s = c->stream;
    DevBuf<uint64_t> key, key2, ukey;
    DevBuf<double> v2, uval;
    DevBuf<int> bad;
    DevBuf<int64_t> nrun;
    size_t cap = nnz ? (size_t)nnz : 1;
    key.alloc(cap);
    key2.alloc(cap);
    v2.alloc(cap);
    ukey.alloc(cap);
    uval.alloc(cap);
    bad.alloc(1);
    nrun.alloc(2);
    JFG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    if (nnz) k_make_keys<<<nblk(nnz), 256, 0, s>>>(nnz, d_ri, d_ci, rows, cols, key.p, bad.p);
    JFG_CUDA(cudaGetLastError());
    int h_bad = 0;
    JFG_CUDA(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));
    JFG_CHECK(!h_bad, JFG_ERR_BAD_ARG, "COO index out of bounds");
    int end_bit = 1;
    uint64_t maxkey = (uint64_t)rows * (uint64_t)cols;
    while (end_bit < 64 && (1ULL << end_bit) < maxkey) end_bit++;
    int64_t m = 0;
    if (nnz) {
        size_t tmp_bytes = 0, tmp2 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.p, key2.p, d_v, v2.p, (int64_t)nnz, 0, end_bit, s);
        cub::DeviceReduce::ReduceByKey(nullptr, tmp2, key2.p, ukey.p, v2.p, uval.p, nrun.p, cub::Sum(), (int64_t)nnz, s);
        DevBuf<char> tmp;
        tmp.alloc(std::max(tmp_bytes, tmp2) + 64);
        JFG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, key.p, key2.p, d_v, v2.p, (int64_t)nnz, 0, end_bit, s));
        JFG_CUDA(cub::DeviceReduce::ReduceByKey(tmp.p, tmp2, key2.p, ukey.p, v2.p, uval.p, nrun.p, cub::Sum(),
                                                (int64_t)nnz, s));
        int64_t h_runs = 0;
        JFG_CUDA(cudaMemcpyAsync(&h_runs, nrun.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        JFG_CUDA(cudaStreamSynchronize(s));
        m = h_runs;
        if (!keep_zeros && m) {
            // keep the merged entries whose value is nonzero
            DevBuf<char> flags;
            flags.alloc((size_t)m);
            k_nonzero_flags<<<nblk(m), 256, 0, s>>>(m, uval.p, flags.p);
            JFG_CUDA(cudaGetLastError());
            size_t t1 = 0, t2 = 0;
            cub::DeviceSelect::Flagged(nullptr, t1, ukey.p, flags.p, key.p, nrun.p + 1, m, s);
            cub::DeviceSelect::Flagged(nullptr, t2, uval.p, flags.p, v2.p, nrun.p + 1, m, s);
            DevBuf<char> tmp4;
            tmp4.alloc(std::max(t1, t2) + 64);
            JFG_CUDA(cub::DeviceSelect::Flagged(tmp4.p, t1, ukey.p, flags.p, key.p, nrun.p + 1, m, s));
            JFG_CUDA(cub::DeviceSelect::Flagged(tmp4.p, t2, uval.p, flags.p, v2.p, nrun.p + 1, m, s));
            int64_t h_sel = 0;
            JFG_CUDA(cudaMemcpyAsync(&h_sel, nrun.p + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            JFG_CUDA(cudaStreamSynchronize(s));
            return build_from_sorted(c, rows, cols, h_sel, key.p, v2.p);
        }
    }
    return build_from_sorted(c, rows, cols, m, ukey.p, uval.p);
}

Matrix* matrix_from_coo(Context* c, int rows, int cols, int64_t nnz, const int* ri, const int* ci, const double* v,
                        bool keep_zeros)
{
    JFG_CHECK(rows >= 0 && cols >= 0 && nnz >= 0, JFG_ERR_BAD_ARG, "negative matrix dimension or nnz");
    JFG_CHECK(nnz == 0 || (ri && ci && v), JFG_ERR_BAD_ARG, "null COO array");
    cudaStream_t s = c->stream;
    DevBuf<int> d_ri, d_ci;
    DevBuf<double> d_v;
    size_t cap = nnz ? (size_t)nnz : 1;
    d_ri.alloc(cap);
    d_ci.alloc(cap);
    d_v.alloc(cap);
    if (nnz) {
        JFG_CUDA(cudaMemcpyAsync(d_ri.p, ri, sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
        JFG_CUDA(cudaMemcpyAsync(d_ci.p, ci, sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
        JFG_CUDA(cudaMemcpyAsync(d_v.p, v, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    return from_device_coo(c, rows, cols, nnz, d_ri.p, d_ci.p, d_v.p, keep_zeros);
}

Matrix* matrix_from_csr_host(Context* c, int rows, int cols, const std::vector<int64_t>& rp,
                             const std::vector<int>& ci, const std::vector<double>& v)
{
    std::vector<int> ri(ci.size());
    for (int r = 0; r < rows; r++)
        for (int64_t k = rp[r]; k < rp[r + 1]; k++) ri[k] = r;
    return matrix_from_coo(c, rows, cols, (int64_t)ci.size(), ri.data(), ci.data(), v.data(), false);
}

// Expands the padded layout back to COO on the device and rebuilds with rows
// and columns exchanged.
Matrix* matrix_transpose(Matrix* M)
{
    if (M->transposed) return M->transposed;
    Context* c = M->ctx;
    cudaStream_t s = c->stream;
    std::vector<int> hptr(M->rows + 1);
    JFG_CUDA(cudaMemcpyAsync(hptr.data(), M->rowptr.p, sizeof(int) * (M->rows + 1), cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> doff(M->rows + 1, 0);
    for (int r = 0; r < M->rows; r++) doff[r + 1] = doff[r] + (hptr[r + 1] - hptr[r]);
    int64_t m = doff[M->rows];
    DevBuf<int64_t> d_off;
    DevBuf<int> ri, ci;
    DevBuf<double> v;
    d_off.alloc((size_t)M->rows + 1);
    ri.alloc(m ? (size_t)m : 1);
    ci.alloc(m ? (size_t)m : 1);
    v.alloc(m ? (size_t)m : 1);
    JFG_CUDA(cudaMemcpyAsync(d_off.p, doff.data(), sizeof(int64_t) * (M->rows + 1), cudaMemcpyHostToDevice, s));
    if (M->rows) {
        k_expand_rows<<<nblk(M->rows), 256, 0, s>>>(M->rows, M->rowptr.p, ri.p, d_off.p);
        k_compact<<<nblk(M->rows), 256, 0, s>>>(M->rows, M->rowptr.p, M->col.p, M->val.p, d_off.p, ci.p, v.p);
    }
    JFG_CUDA(cudaGetLastError());
    M->transposed = from_device_coo(c, M->cols, M->rows, m, ci.p, ri.p, v.p, false);
    return M->transposed;
}

void matrix_ensure_fp32(Matrix* M)
{
    if (M->has32) return;
    M->val32.alloc((size_t)M->nnz_padded);
    k_to_f32<<<nblk(M->nnz_padded), 256, 0, M->ctx->stream>>>(M->nnz_padded, M->val.p, M->val32.p);
    JFG_CUDA(cudaGetLastError());
    M->has32 = 1;
}

void matrix_ensure_bf16(Matrix* M)
{
    if (M->has16) return;
    M->val16.alloc((size_t)M->nnz_padded);
    k_to_bf16<<<nblk(M->nnz_padded), 256, 0, M->ctx->stream>>>(M->nnz_padded, M->val.p, M->val16.p);
    JFG_CUDA(cudaGetLastError());
    M->has16 = 1;
}

}  // namespace jfg
