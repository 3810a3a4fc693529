// COO -> CSR -> SELL-32-sigma conversion on the device, transposes and
// precision copies.
#include <cub/cub.cuh>

#include <climits>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <numeric>

#include "jfg_kernels.cuh"

namespace jfg {

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

bool spmv_pipe()
{
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("JFEM_SPMV_PIPE");
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

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

__global__ void k_make_keys(int64_t nnz, const int* ri, const int* ci, int rows, int cols, uint64_t* key, int* bad)
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

// merged sorted keys -> CSR column indices (values are already in CSR order)
__global__ void k_key_cols(int64_t m, const uint64_t* key, int cols, int* col)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) col[k] = (int)(key[k] % (uint64_t)cols);
}

__global__ void k_diag(int rows, int cols, const int* ptr, const int* col, const double* val, double* d)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double s = 0;
    if (r < cols)
        for (int k = ptr[r]; k < ptr[r + 1]; k++)
            if (col[k] == r) s += val[k];
    d[r] = s;
}

// one thread per SELL slot: copies its row into the slice column-major and
// pads with (last column of the row, 0.0)
__global__ void k_fill_sell(int nslots, const int* perm, const int* off, const int* ptr, const int* ccol,
                            const double* cval, int* col, double* val)
{
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslots) return;
    int s = slot >> 5, lane = slot & 31;
    int o = off[s];
    int len = (off[s + 1] - o) >> 5;
    int r = perm[slot];
    int a = 0, e = 0;
    if (r >= 0) {
        a = ptr[r];
        e = ptr[r + 1];
    }
    int pad_col = e > a ? ccol[e - 1] : 0;
    for (int k = 0; k < len; k++) {
        int64_t dst = (int64_t)o + (int64_t)k * 32 + lane;
        if (a + k < e) {
            col[dst] = ccol[a + k];
            val[dst] = cval[a + k];
        } else {
            col[dst] = pad_col;
            val[dst] = 0.0;
        }
    }
}

// 16-bit column offsets relative to the slot's row (FE matrices couple rows
// to nearby columns); flags an entry that does not fit
__global__ void k_make_col16(int nslots, const int* perm, const int* off, const int* col, int16_t* col16, int* bad)
{
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslots) return;
    int s = slot >> 5, lane = slot & 31;
    int o = off[s];
    int len = (off[s + 1] - o) >> 5;
    int base = max(perm[slot], 0);
    for (int k = 0; k < len; k++) {
        int64_t at = (int64_t)o + (int64_t)k * 32 + lane;
        int d = col[at] - base;
        if (d < -32768 || d > 32767) {
            atomicOr(bad, 1);
            return;
        }
        col16[at] = (int16_t)d;
    }
}

// 16-bit column offsets from a per-slice base column (matrices whose columns
// are far from their rows, e.g. transfers between grids): one warp per slice,
// base = (smallest column of the slice's rows) + 32768, so a span of up to
// 65,535 columns fits; padding slots (no row) point at the smallest column.
__global__ void k_make_col16_slice(int nslots, const int* perm, const int* off, const int* col, int16_t* col16,
                                   int* cbase, int* bad)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = slot < nslots;                      // nslots is a multiple of 32: warp-uniform
    if (!in) return;
    const int s = slot >> 5, lane = slot & 31;
    const int o = off[s];
    const int len = (off[s + 1] - o) >> 5;
    const bool real = perm[slot] >= 0;
    int mn = INT_MAX, mx = INT_MIN;
    if (real)
        for (int k = 0; k < len; k++) {
            const int c = col[(int64_t)o + (int64_t)k * 32 + lane];
            mn = min(mn, c);
            mx = max(mx, c);
        }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (mn == INT_MAX) mn = mx = 0;                     // a slice of padding slots only
    if ((int64_t)mx - mn > 65535) {
        if (lane == 0) atomicOr(bad, 1);
        return;
    }
    const int base = mn + 32768;
    if (lane == 0) cbase[s] = base;
    for (int k = 0; k < len; k++) {
        const int64_t at = (int64_t)o + (int64_t)k * 32 + lane;
        col16[at] = (int16_t)((real ? col[at] : mn) - base);
    }
}

__global__ void k_expand_rows(int rows, const int* ptr, int* ri)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    for (int k = ptr[r]; k < ptr[r + 1]; k++) ri[k] = r;
}

// Point layouts (Matrix::st): row r is regular when its entries all sit at
// center(r) + off_k for the layout's offsets and all those columns exist.
//   kind 0 (9-point stencil):    center = r, offsets (a - 1) S + (b - 1), a, b in 0..2
//   kind 1 (prolongation, rows = fine nodes with grid stride S, columns =
//     coarse nodes with stride S2): center = (g / 2) S2 + h / 2 for
//     (g, h) = (r / S, r % S), offsets {0, 1, S2, S2 + 1}
//   kind 2 (restriction, rows = coarse nodes with stride S, columns = fine
//     nodes with stride S2): center = 2 g S2 + 2 h, offsets (a - 1) S2 + (b - 1)
__device__ __forceinline__ int pt_center(int kind, int S, int S2, int r)
{
    if (kind == 0) return r;
    const int g = r / S, h = r - g * S;
    return kind == 1 ? (g >> 1) * S2 + (h >> 1) : 2 * g * S2 + 2 * h;
}
// offset d -> slot (ascending column order), -1 when d is not an offset
__device__ __forceinline__ int pt_slot(int kind, int S, int S2, int d)
{
    if (kind == 1) return d == 0 ? 0 : d == 1 ? 1 : d == S2 ? 2 : d == S2 + 1 ? 3 : -1;
    const int X = kind == 0 ? S : S2;
    if (d >= -1 && d <= 1) return d + 4;
    if (d >= -X - 1 && d <= -X + 1) return d + X + 1;
    if (d >= X - 1 && d <= X + 1) return d - X + 7;
    return -1;
}

__global__ void k_st_classify(int rows, int cols, int kind, int S, int S2, const int* __restrict__ ptr,
                              const int* __restrict__ col, unsigned char* __restrict__ reg)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int c = pt_center(kind, S, S2, r);
    const int X = kind == 0 ? S : S2;
    const int lo = kind == 1 ? 0 : -X - 1, hi = kind == 1 ? S2 + 1 : X + 1;
    bool ok = c + lo >= 0 && c + hi < cols;
    for (int k = ptr[r]; ok && k < ptr[r + 1]; k++) ok = pt_slot(kind, S, S2, col[k] - c) >= 0;
    reg[r] = ok ? 1 : 0;
}

__global__ void k_st_fill(int kind, int lo, int nreg, int ld, int S, int S2, const int* __restrict__ ptr,
                          const int* __restrict__ col, const double* __restrict__ val, double* __restrict__ st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nreg) return;
    const int r = lo + i;
    const int c = pt_center(kind, S, S2, r);
    for (int k = ptr[r]; k < ptr[r + 1]; k++) st[(int64_t)pt_slot(kind, S, S2, col[k] - c) * ld + i] = val[k];
}

// CSR copy of the irregular rows (their entries in column order)
__global__ void k_st_irregular(int nirr, const int* __restrict__ irow, const int* __restrict__ iptr,
                               const int* __restrict__ ptr, const int* __restrict__ col,
                               const double* __restrict__ val, int* __restrict__ icol, double* __restrict__ ival)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nirr) return;
    const int r = irow[j];
    int o = iptr[j];
    for (int k = ptr[r]; k < ptr[r + 1]; k++, o++) {
        icol[o] = col[k];
        ival[o] = val[k];
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

}  // namespace

// JFEM_STENCIL=0 keeps every matrix built afterwards in SELL-32 only (read
// at each build: products of one matrix in both layouts can be compared)
bool stencil_enabled()
{
    const char* e = getenv("JFEM_STENCIL");
    return !(e && e[0] == '0');
}

// JFEM_ST_STAGED=1 gives the 9-point layouts built afterwards the staged
// kernel k_spmv_pt instead of the register kernel k_spmv_st (read at each build)
static bool st_staged_enabled()
{
    const char* e = getenv("JFEM_ST_STAGED");
    return e && e[0] == '1';
}

// Point layout of M (see Matrix::st) for the rows whose entries fit it:
// kind 0 detects the 9-point stencil's stride S off a few middle rows
// (largest column offset - 1); kinds 1 and 2 (grid transfers) take S and S2
// from the level matrices.  The layout is kept when the contiguous run of
// regular rows around the middle row leaves at most a quarter of the rows
// outside it.
static void build_point_layout(Matrix* M, const std::vector<int>& len, int kind, int S, int S2)
{
    const int n = M->rows;
    if (n < 256 || M->st || !stencil_enabled()) return;
    if (kind == 0 && M->rows != M->cols) return;
    cudaStream_t s = M->ctx->stream;
    if (kind == 0) {
        std::vector<int> hp(n + 1);
        JFG_CUDA(cudaMemcpyAsync(hp.data(), M->csr_ptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
        JFG_CUDA(cudaStreamSynchronize(s));
        S = 0;
        for (int j = 0; j < 16 && !S; j++) {
            const int r = n / 2 + j;
            const int a = hp[r], e = hp[r + 1];
            if (e - a < 2 || e - a > 9) continue;
            std::vector<int> c(e - a);
            JFG_CUDA(cudaMemcpyAsync(c.data(), M->csr_col.p + a, sizeof(int) * (e - a), cudaMemcpyDeviceToHost, s));
            JFG_CUDA(cudaStreamSynchronize(s));
            const int cand = c.back() - r - 1;
            if (cand < 3) continue;
            bool ok = true;
            for (int v : c) {
                const int d = std::abs(v - r);
                ok = ok && (d <= 1 || (d >= cand - 1 && d <= cand + 1));
            }
            if (ok) S = cand;
        }
        S2 = 0;
    }
    if (S < 3 || (kind != 0 && S2 < 3)) return;
    const int K = kind == 1 ? 4 : 9;
    DevBuf<unsigned char> reg;
    reg.alloc((size_t)n);
    k_st_classify<<<nblk(n), 256, 0, s>>>(n, M->cols, kind, S, S2, M->csr_ptr.p, M->csr_col.p, reg.p);
    JFG_CUDA(cudaGetLastError());
    std::vector<unsigned char> hr(n);
    JFG_CUDA(cudaMemcpyAsync(hr.data(), reg.p, (size_t)n, cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));
    // the range: from the row after the last irregular row of the first half
    // to the first irregular row of the second half (on 2-D grids numbered by
    // first appearance the irregular rows are the first and the last grid
    // lines; the regular Dirichlet rows among them go to CSR)
    const int mid = n / 2;
    int lo = mid, hi = mid;
    while (lo > 0 && hr[lo - 1]) lo--;
    while (hi < n && hr[hi]) hi++;
    if (hi - lo < 64) return;
    const int nreg = hi - lo, nirr = n - nreg;
    if ((int64_t)nirr * 4 > n) return;
    std::vector<int> irow, iptr{0};
    irow.reserve(nirr);
    for (int r = 0; r < n; r++)
        if (r < lo || r >= hi) {
            irow.push_back(r);
            iptr.push_back(iptr.back() + len[r]);
        }
    const int64_t irr_nnz = iptr.back();
    const int ld = (nreg + 7) / 8 * 8;
    M->st_kind = kind;
    M->st_staged = st_staged_enabled() ? 1 : 0;
    M->st_err.alloc(1);
    JFG_CUDA(cudaMemsetAsync(M->st_err.p, 0, sizeof(int), s));
    M->st_K = K;
    M->st_S = S;
    M->st_S2 = S2;
    M->st_lo = lo;
    M->st_hi = hi;
    M->st_nirr = nirr;
    M->st_ld = ld;
    M->st_len = (int64_t)K * ld + irr_nnz;
    M->st_val.alloc((size_t)M->st_len);
    M->st_irow.alloc(nirr ? (size_t)nirr : 1);
    M->st_iptr.alloc((size_t)nirr + 1);
    M->st_icol.alloc(irr_nnz ? (size_t)irr_nnz : 1);
    JFG_CUDA(cudaMemsetAsync(M->st_val.p, 0, sizeof(double) * K * (size_t)ld, s));
    k_st_fill<<<nblk(nreg), 256, 0, s>>>(kind, lo, nreg, ld, S, S2, M->csr_ptr.p, M->csr_col.p, M->csr_val.p,
                                        M->st_val.p);
    JFG_CUDA(cudaGetLastError());
    if (nirr) {
        JFG_CUDA(cudaMemcpyAsync(M->st_irow.p, irow.data(), sizeof(int) * nirr, cudaMemcpyHostToDevice, s));
        JFG_CUDA(cudaMemcpyAsync(M->st_iptr.p, iptr.data(), sizeof(int) * (nirr + 1), cudaMemcpyHostToDevice, s));
        k_st_irregular<<<nblk(nirr), 256, 0, s>>>(nirr, M->st_irow.p, M->st_iptr.p, M->csr_ptr.p, M->csr_col.p,
                                                 M->csr_val.p, M->st_icol.p, M->st_val.p + (int64_t)K * ld);
        JFG_CUDA(cudaGetLastError());
    }
    // the 9-point kernel takes rows in pairs (its launch caps the grid); the transfer kernel one row per thread
    M->st_nb_reg = (int)nblk(nreg, kind == 0 ? kThreads * 2 : kThreads);
    M->st_nb_irr = (int)nblk(nirr, kThreads);
    M->nblocks = std::max(M->nblocks, M->st_nb_reg + M->st_nb_irr);
    JFG_CUDA(cudaStreamSynchronize(s));
    M->st = 1;
}

// Row lengths of a matrix's CSR on the host.
static std::vector<int> row_lengths(const Matrix* M)
{
    std::vector<int> hp(M->rows + 1), len(M->rows + 1, 0);
    JFG_CUDA(cudaMemcpyAsync(hp.data(), M->csr_ptr.p, sizeof(int) * (M->rows + 1), cudaMemcpyDeviceToHost,
                             M->ctx->stream));
    JFG_CUDA(cudaStreamSynchronize(M->ctx->stream));
    for (int r = 0; r < M->rows; r++) len[r] = hp[r + 1] - hp[r];
    return len;
}

void matrix_build_transfer_layout(Matrix* M, int kind, int S, int S2)
{
    if (M->st || M->csr_only || M->has32 || M->has16 || M->hash) return;   // precision copies follow the layout
    build_point_layout(M, row_lengths(M), kind, S, S2);
}

// Builds CSR and SELL-32-sigma from merged, sorted, zero-free COO that is
// already on the device (keys = row*cols+col ascending, values alongside).
static Matrix* build_from_sorted(Context* c, int rows, int cols, int64_t m, const uint64_t* d_key,
                                 const double* d_val, bool sell = true)
{
    cudaStream_t s = c->stream;
    JFG_CHECK(m < (int64_t)INT32_MAX - 64, JFG_ERR_UNSUPPORTED, "matrix has more than 2^31 nonzeros");
    auto* M = new Matrix();
    M->ctx = c;
    M->rows = rows;
    M->cols = cols;
    M->nnz = m;
    // row counts -> CSR row pointers
    DevBuf<int> cnt;
    cnt.alloc((size_t)rows + 1);
    JFG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * ((size_t)rows + 1), s));
    if (m) k_row_counts<<<nblk(m), 256, 0, s>>>(m, d_key, cols, cnt.p);
    JFG_CUDA(cudaGetLastError());
    std::vector<int> len(rows + 1, 0);
    JFG_CUDA(cudaMemcpyAsync(len.data(), cnt.p, sizeof(int) * rows, cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));
    std::vector<int> ptr(rows + 1, 0);
    for (int r = 0; r < rows; r++) ptr[r + 1] = ptr[r] + len[r];
    M->csr_ptr.alloc((size_t)rows + 1);
    M->csr_col.alloc(m ? (size_t)m : 1);
    M->csr_val.alloc(m ? (size_t)m : 1);
    JFG_CUDA(cudaMemcpyAsync(M->csr_ptr.p, ptr.data(), sizeof(int) * (rows + 1), cudaMemcpyHostToDevice, s));
    if (m) {
        k_key_cols<<<nblk(m), 256, 0, s>>>(m, d_key, cols, M->csr_col.p);
        JFG_CUDA(cudaMemcpyAsync(M->csr_val.p, d_val, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
    }
    M->diag.alloc((size_t)rows);
    if (rows) k_diag<<<nblk(rows), 256, 0, s>>>(rows, cols, M->csr_ptr.p, M->csr_col.p, M->csr_val.p, M->diag.p);
    JFG_CUDA(cudaGetLastError());
    if (!sell) {
        M->csr_only = 1;
        JFG_CUDA(cudaStreamSynchronize(s));
        return M;
    }
    // SELL-32-sigma: sort rows by length (descending, stable) inside windows
    int nslices = (rows + kSliceRows - 1) / kSliceRows;
    std::vector<int> perm((size_t)nslices * kSliceRows, -1);
    std::vector<int> idx(rows);
    std::iota(idx.begin(), idx.end(), 0);
    for (int w0 = 0; w0 < rows; w0 += kSellSigma) {
        int w1 = std::min(rows, w0 + kSellSigma);
        std::stable_sort(idx.begin() + w0, idx.begin() + w1, [&](int a, int b) { return len[a] > len[b]; });
    }
    std::copy(idx.begin(), idx.end(), perm.begin());
    std::vector<int> off(nslices + 1, 0);
    int64_t total = 0;
    for (int sl = 0; sl < nslices; sl++) {
        int mx = 0;
        for (int l = 0; l < kSliceRows; l++) {
            int r = perm[(size_t)sl * kSliceRows + l];
            if (r >= 0) mx = std::max(mx, len[r]);
        }
        off[sl] = (int)total;
        total += (int64_t)mx * kSliceRows;
        JFG_CHECK(total < (int64_t)INT32_MAX - 64, JFG_ERR_UNSUPPORTED, "padded matrix exceeds 2^31 entries");
    }
    off[nslices] = (int)total;
    M->nslices = nslices;
    M->sell_len = total;
    // threads per row: 1 from 262,144 rows (the staged one-thread-per-row
    // kernel), 4 from 32,768 rows or with short rows, 8 on small matrices with
    // rows of 10 or more entries (measured on the Q2 multigrid levels;
    // JFEM_TPR overrides)
    double avg = rows ? (double)m / rows : 0.0;
    int tl = rows >= 262144 ? 0 : (avg >= 10.0 ? (rows >= 32768 ? 2 : 3) : 2);
    if (const char* e = getenv("JFEM_TPR")) {
        int v = atoi(e);
        tl = v <= 0 ? 0 : (v <= 2 ? 2 : 3);   // the SpMV is instantiated for 1, 4 and 8 threads per row
    }
    M->tpr_log2 = tl;
    M->nblocks = std::max(1, (int)((((int64_t)nslices * kSliceRows << tl) + kThreads - 1) / kThreads));
    M->off.alloc((size_t)nslices + 1);
    M->perm.alloc(perm.size() ? perm.size() : 1);
    M->col.alloc(total ? (size_t)total : 1);
    M->val.alloc(total ? (size_t)total : 1);
    JFG_CUDA(cudaMemcpyAsync(M->off.p, off.data(), sizeof(int) * (nslices + 1), cudaMemcpyHostToDevice, s));
    if (!perm.empty())
        JFG_CUDA(cudaMemcpyAsync(M->perm.p, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, s));
    if (nslices)
        k_fill_sell<<<nblk((int64_t)nslices * kSliceRows), 256, 0, s>>>(nslices * kSliceRows, M->perm.p, M->off.p,
                                                                         M->csr_ptr.p, M->csr_col.p, M->csr_val.p,
                                                                         M->col.p, M->val.p);
    JFG_CUDA(cudaGetLastError());
    const char* e16 = getenv("JFEM_IDX16");
    if (nslices && !(e16 && e16[0] == '0')) {
        DevBuf<int> bad;
        bad.alloc(1);
        JFG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
        M->col16.alloc((size_t)total);
        k_make_col16<<<nblk((int64_t)nslices * kSliceRows), 256, 0, s>>>(nslices * kSliceRows, M->perm.p, M->off.p,
                                                                          M->col.p, M->col16.p, bad.p);
        JFG_CUDA(cudaGetLastError());
        int hb = 0;
        JFG_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        JFG_CUDA(cudaStreamSynchronize(s));
        M->idx16 = hb ? 0 : 1;
        if (hb) {       // columns far from the rows: try offsets from a base column per slice
            JFG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
            M->cbase.alloc((size_t)nslices);
            k_make_col16_slice<<<nblk((int64_t)nslices * kSliceRows), 256, 0, s>>>(
                nslices * kSliceRows, M->perm.p, M->off.p, M->col.p, M->col16.p, M->cbase.p, bad.p);
            JFG_CUDA(cudaGetLastError());
            JFG_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            JFG_CUDA(cudaStreamSynchronize(s));
            M->idx16 = hb ? 0 : 2;
            if (hb) {
                M->col16.release();
                M->cbase.release();
            }
        }
    }
    JFG_CUDA(cudaStreamSynchronize(s));
    build_point_layout(M, len, 0, 0, 0);
    return M;
}

Matrix* matrix_from_sorted_keys(Context* c, int rows, int cols, int64_t m, const uint64_t* d_key,
                                const double* d_val, bool sell)
{
    return build_from_sorted(c, rows, cols, m, d_key, d_val, sell);
}

// COO on the device -> Matrix (sort, merge duplicates, drop zeros).
static Matrix* from_device_coo(Context* c, int rows, int cols, int64_t nnz, const int* d_ri, const int* d_ci,
                               const double* d_v)
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
    if (!nnz) return build_from_sorted(c, rows, cols, 0, ukey.p, uval.p);
    int end_bit = 1;
    uint64_t maxkey = (uint64_t)rows * (uint64_t)cols;
    while (end_bit < 64 && (1ULL << end_bit) < maxkey) end_bit++;
    size_t tmp_bytes = 0, tmp2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.p, key2.p, d_v, v2.p, (int64_t)nnz, 0, end_bit, s);
    cub::DeviceReduce::ReduceByKey(nullptr, tmp2, key2.p, ukey.p, v2.p, uval.p, nrun.p, cub::Sum(), (int64_t)nnz, s);
    DevBuf<char> tmp;
    tmp.alloc(std::max(tmp_bytes, tmp2) + 64);
    JFG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, key.p, key2.p, d_v, v2.p, (int64_t)nnz, 0, end_bit, s));
    JFG_CUDA(cub::DeviceReduce::ReduceByKey(tmp.p, tmp2, key2.p, ukey.p, v2.p, uval.p, nrun.p, cub::Sum(),
                                            (int64_t)nnz, s));
    int64_t m = 0;
    JFG_CUDA(cudaMemcpyAsync(&m, nrun.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    JFG_CUDA(cudaStreamSynchronize(s));
    if (!m) return build_from_sorted(c, rows, cols, 0, ukey.p, uval.p);
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

Matrix* matrix_from_device_coo(Context* c, int rows, int cols, int64_t nnz, const int* d_ri, const int* d_ci,
                               const double* d_v)
{
    return from_device_coo(c, rows, cols, nnz, d_ri, d_ci, d_v);
}

Matrix* matrix_from_coo(Context* c, int rows, int cols, int64_t nnz, const int* ri, const int* ci, const double* v,
                        bool keep_zeros)
{
    (void)keep_zeros;
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
    return from_device_coo(c, rows, cols, nnz, d_ri.p, d_ci.p, d_v.p);
}

Matrix* matrix_from_csr_host(Context* c, int rows, int cols, const std::vector<int64_t>& rp,
                             const std::vector<int>& ci, const std::vector<double>& v)
{
    std::vector<int> ri(ci.size());
    for (int r = 0; r < rows; r++)
        for (int64_t k = rp[r]; k < rp[r + 1]; k++) ri[k] = r;
    return matrix_from_coo(c, rows, cols, (int64_t)ci.size(), ri.data(), ci.data(), v.data(), false);
}

// CSR -> COO with rows and columns exchanged -> Matrix.
Matrix* matrix_transpose(Matrix* M)
{
    if (M->transposed) return M->transposed;
    Context* c = M->ctx;
    cudaStream_t s = c->stream;
    int64_t m = M->nnz;
    DevBuf<int> ri;
    ri.alloc(m ? (size_t)m : 1);
    if (M->rows) k_expand_rows<<<nblk(M->rows), 256, 0, s>>>(M->rows, M->csr_ptr.p, ri.p);
    JFG_CUDA(cudaGetLastError());
    M->transposed = from_device_coo(c, M->cols, M->rows, m, M->csr_col.p, ri.p, M->csr_val.p);
    return M->transposed;
}

void matrix_ensure_fp32(Matrix* M)
{
    if (M->has32) return;
    M->val32.alloc(M->sell_len ? (size_t)M->sell_len : 1);
    if (M->sell_len) k_to_f32<<<nblk(M->sell_len), 256, 0, M->ctx->stream>>>(M->sell_len, M->val.p, M->val32.p);
    JFG_CUDA(cudaGetLastError());
    if (M->st) {
        M->st_val32.alloc((size_t)M->st_len);
        k_to_f32<<<nblk(M->st_len), 256, 0, M->ctx->stream>>>(M->st_len, M->st_val.p, M->st_val32.p);
        JFG_CUDA(cudaGetLastError());
    }
    M->has32 = 1;
}

namespace {
__global__ void k_absmax(int64_t n, const double* __restrict__ a, unsigned long long* __restrict__ out)
{
    // |a| of finite doubles orders like its bit pattern: one atomicMax on the bits
    unsigned long long m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(a[i]));
        m = b > m ? b : m;
    }
    atomicMax(out, m);
}
__global__ void k_to_f16(int64_t n, const double* __restrict__ a, double s, __half* __restrict__ b)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __double2half(a[i] * s);       // exact scaling by 2^k, one rounding
}
}  // namespace

// FP16 copy of the SpMV values scaled by s = 2^k with max |a| * s in
// [2^14, 2^15]: the small entries (mass terms ~h^2) stay out of the FP16
// subnormal range; the SpMV multiplies its row sums by 1/s (exact).
void matrix_ensure_fp16(Matrix* M)
{
    if (M->hash) return;
    cudaStream_t st = M->ctx->stream;
    DevBuf<unsigned long long> mx;
    mx.alloc(1);
    JFG_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(unsigned long long), st));
    if (M->nnz) k_absmax<<<std::min<int64_t>(nblk(M->nnz), 1184), 256, 0, st>>>(M->nnz, M->csr_val.p, mx.p);
    JFG_CUDA(cudaGetLastError());
    unsigned long long hb = 0;
    JFG_CUDA(cudaMemcpyAsync(&hb, mx.p, sizeof(hb), cudaMemcpyDeviceToHost, st));
    JFG_CUDA(cudaStreamSynchronize(st));
    double amax;
    memcpy(&amax, &hb, sizeof(amax));
    int e = 0;
    if (amax > 0 && std::isfinite(amax)) {
        std::frexp(amax, &e);                       // amax in [2^(e-1), 2^e)
        e = 15 - e;                                 // amax * 2^e in [2^14, 2^15)
        e = std::max(-120, std::min(120, e));
    }
    const double s = std::ldexp(1.0, e);
    M->hscale_inv = (float)std::ldexp(1.0, -e);
    M->valh.alloc(M->sell_len ? (size_t)M->sell_len : 1);
    if (M->sell_len) k_to_f16<<<nblk(M->sell_len), 256, 0, st>>>(M->sell_len, M->val.p, s, M->valh.p);
    JFG_CUDA(cudaGetLastError());
    if (M->st) {
        M->st_valh.alloc((size_t)M->st_len);
        k_to_f16<<<nblk(M->st_len), 256, 0, st>>>(M->st_len, M->st_val.p, s, M->st_valh.p);
        JFG_CUDA(cudaGetLastError());
    }
    M->hash = 1;
}

void matrix_ensure_bf16(Matrix* M)
{
    if (M->has16) return;
    M->val16.alloc(M->sell_len ? (size_t)M->sell_len : 1);
    if (M->sell_len) k_to_bf16<<<nblk(M->sell_len), 256, 0, M->ctx->stream>>>(M->sell_len, M->val.p, M->val16.p);
    JFG_CUDA(cudaGetLastError());
    if (M->st) {
        M->st_val16.alloc((size_t)M->st_len);
        k_to_bf16<<<nblk(M->st_len), 256, 0, M->ctx->stream>>>(M->st_len, M->st_val.p, M->st_val16.p);
        JFG_CUDA(cudaGetLastError());
    }
    M->has16 = 1;
}

}  // namespace jfg
