/*
 * jfem_oracle.c -- CPU restatement (FP64) of JFEM's linear-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline.  It is never linked into the product library (libjfem_gpu.so);
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Every routine restates one Java routine of the reference (paths relative to
 * the JFEM project root, Core/src/main/java/...):
 *   - COO storage and scatter SpMV ........ linalg/SparseMatrix.java:22-27, 274-294, 480-501
 *   - row/column bucketed SpMV ............ linalg/SparseMvMul.java:21-116
 *   - vector inner / norm ................. linalg/DenseVector.java:104-121, linalg/Vector.java:80-94
 *   - CG / PCG ............................ linalg/IterativeSolver.java:48-162
 *   - BiCGStab / PBiCGStab ................ linalg/IterativeSolver.java:234-402
 *   - restarted GMRES (Givens) ............ linalg/GMRES.java:40-251
 *   - GMRES2 + Arnoldi .................... linalg/GMRES2.java:34-104, linalg/Arnoldi.java:13-83
 *   - Jacobi / Richardson smoothers ....... multigrid/JacobiSmoother.java:12-50,
 *                                           multigrid/RichardsonSmoother.java:13-50
 *   - V-cycle, FMG, preconditioner mvMul .. multigrid/MGPreconditionerInterface.java:125-198, 293-379
 *   - transfers with zero boundary ........ multigrid/MGPreconditionerSpace.java:59-109
 *   - dense LU solve / inverse ............ linalg/DenseMatrix.java:491-519 (UJMP) and
 *                                           JSparse/src/native/sparseSolver.cpp:10-113 (LAPACK);
 *     both are restated as textbook partial-pivot LU: the pivot order of
 *     UJMP/LAPACK is not reproduced bit-for-bit.
 *   - java.util.Random (48-bit LCG, nextDouble) for the seeded fixtures of the
 *     reference tests (linalg/SparseMvMulTest.java:12-113).
 *
 * Threads: the loops the reference runs as Java parallel streams when
 * PerformanceArguments.parallelizeThreads is set (PerformanceArguments.java:24)
 * run as OpenMP loops here -- SparseMvMul.mvMul/tvMul rows/columns
 * (SparseMvMul.java:81-84, 103-106), the GMRES orthogonality factors
 * (GMRES.java:203-210) and the patches of one colour
 * (ColoredMultiplicativeSubspaceCorrection.java:91-111).  Each output element
 * is computed by one thread in the serial order, so the results do not depend
 * on the thread count.  Everything else, the COO scatter SpMV included, is
 * serial as in the reference.  or_set_threads() sets the count.
 *
 * Deviations, all documented: solvers carry an iteration/restart cap so that no
 * call can run forever (the reference's GMRES restarts without bound while the
 * true residual exceeds tol, GMRES.java:92; GMRES2 loops without bound,
 * GMRES2.java:70).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_OK 0
#define OR_MAXITER 1
#define OR_BREAKDOWN 2
#define OR_NONFINITE 3
#define OR_BADARG 4
#define OR_SINGULAR 5

/* ------------------------------------------------------------------ */
/* java.util.Random: the documented 48-bit linear congruential generator */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t seed; } or_jrand;

static void jr_init(or_jrand* r, int64_t seed)
{
    r->seed = ((uint64_t)seed ^ 0x5DEECE66DULL) & ((1ULL << 48) - 1);
}
static int32_t jr_next(or_jrand* r, int bits)
{
    r->seed = (r->seed * 0x5DEECE66DULL + 0xBULL) & ((1ULL << 48) - 1);
    return (int32_t)(uint32_t)(r->seed >> (48 - bits));
}
static double jr_next_double(or_jrand* r)
{
    int64_t hi = (int64_t)jr_next(r, 26);
    int64_t lo = (int64_t)jr_next(r, 27);
    return (double)((hi << 27) + lo) * (1.0 / 9007199254740992.0);
}

/* Fills out[0..count) with successive nextDouble() values of new Random(seed). */
void or_jrandom_doubles(long long seed, long long count, double* out)
{
    or_jrand r;
    jr_init(&r, (int64_t)seed);
    for (long long i = 0; i < count; i++) out[i] = jr_next_double(&r);
}

/* ------------------------------------------------------------------ */
/* COO matrix (SparseMatrix.java) and merged CSR/CSC (SparseMvMul.java) */
/* ------------------------------------------------------------------ */
typedef struct or_mat {
    int rows, cols;
    long long nnz;
    int* ri;       /* sparseYs: row index of each stored triple */
    int* ci;       /* sparseXs: column index */
    double* v;     /* sparseValues */
    /* merged (duplicates summed) row and column buckets, SparseMvMul semantics */
    long long* rp; int* rc; double* rv;
    long long* cp; int* cr; double* cv;
} or_mat;

static int cmp_pair(const void* a, const void* b)
{
    const long long* x = (const long long*)a;
    const long long* y = (const long long*)b;
    if (x[0] != y[0]) return (x[0] > y[0]) - (x[0] < y[0]);
    return (x[1] > y[1]) - (x[1] < y[1]);
}

/* Merged row and column buckets: SparseMvMul.java:21-60 builds them from
 * getCoordinateEntryList(), i.e. with duplicates summed. */
static void build_buckets(or_mat* m)
{
    long long nnz = m->nnz, cap = nnz ? nnz : 1;
    long long* key = (long long*)malloc(sizeof(long long) * cap * 2);
    for (long long k = 0; k < nnz; k++) {
        key[2 * k] = (long long)m->ri[k] * m->cols + m->ci[k];
        key[2 * k + 1] = k;
    }
    qsort(key, nnz, 2 * sizeof(long long), cmp_pair);
    long long u = 0;
    long long* ukey = (long long*)malloc(sizeof(long long) * cap);
    double* uval = (double*)malloc(sizeof(double) * cap);
    for (long long k = 0; k < nnz; k++) {
        long long kk = key[2 * k];
        double val = m->v[key[2 * k + 1]];
        if (u > 0 && ukey[u - 1] == kk) uval[u - 1] += val;
        else { ukey[u] = kk; uval[u] = val; u++; }
    }
    m->rp = (long long*)calloc((size_t)m->rows + 1, sizeof(long long));
    m->cp = (long long*)calloc((size_t)m->cols + 1, sizeof(long long));
    m->rc = (int*)malloc(sizeof(int) * (u ? u : 1));
    m->rv = (double*)malloc(sizeof(double) * (u ? u : 1));
    m->cr = (int*)malloc(sizeof(int) * (u ? u : 1));
    m->cv = (double*)malloc(sizeof(double) * (u ? u : 1));
    for (long long k = 0; k < u; k++) {
        int r = (int)(ukey[k] / m->cols), c = (int)(ukey[k] % m->cols);
        m->rp[r + 1]++; m->cp[c + 1]++;
    }
    for (int i = 0; i < m->rows; i++) m->rp[i + 1] += m->rp[i];
    for (int i = 0; i < m->cols; i++) m->cp[i + 1] += m->cp[i];
    long long* cfill = (long long*)malloc(sizeof(long long) * ((size_t)m->cols + 1));
    memcpy(cfill, m->cp, sizeof(long long) * ((size_t)m->cols + 1));
    for (long long k = 0; k < u; k++) {
        int r = (int)(ukey[k] / m->cols), c = (int)(ukey[k] % m->cols);
        m->rc[k] = c; m->rv[k] = uval[k];
        long long p = cfill[c]++;
        m->cr[p] = r; m->cv[p] = uval[k];
    }
    free(cfill); free(key); free(ukey); free(uval);
}

or_mat* or_mat_new(int rows, int cols, long long nnz, const int* ri, const int* ci, const double* v)
{
    if (rows < 0 || cols < 0 || nnz < 0) return NULL;
    for (long long k = 0; k < nnz; k++)
        if (ri[k] < 0 || ri[k] >= rows || ci[k] < 0 || ci[k] >= cols) return NULL;
    or_mat* m = (or_mat*)calloc(1, sizeof(or_mat));
    m->rows = rows; m->cols = cols; m->nnz = nnz;
    long long cap = nnz ? nnz : 1;
    m->ri = (int*)malloc(sizeof(int) * cap);
    m->ci = (int*)malloc(sizeof(int) * cap);
    m->v = (double*)malloc(sizeof(double) * cap);
    if (nnz) {
        memcpy(m->ri, ri, sizeof(int) * nnz);
        memcpy(m->ci, ci, sizeof(int) * nnz);
        memcpy(m->v, v, sizeof(double) * nnz);
    }
    build_buckets(m);
    return m;
}

void or_mat_free(or_mat* m)
{
    if (!m) return;
    free(m->ri); free(m->ci); free(m->v);
    free(m->rp); free(m->rc); free(m->rv);
    free(m->cp); free(m->cr); free(m->cv);
    free(m);
}

int or_mat_rows(const or_mat* m) { return m->rows; }
int or_mat_cols(const or_mat* m) { return m->cols; }

static int cmp_int_asc(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* SparseMatrix.mvMul (SparseMatrix.java:480-489): COO scatter in storage order. */
void or_mat_mvmul(const or_mat* m, const double* x, double* y)
{
    memset(y, 0, sizeof(double) * m->rows);
    for (long long k = 0; k < m->nnz; k++) y[m->ri[k]] += m->v[k] * x[m->ci[k]];
}

long long or_mat_nnz(const or_mat* m) { return m->nnz; }

/* The stored COO triples (for a product: row-major, columns ascending). */
void or_mat_coo(const or_mat* m, int* ri, int* ci, double* v)
{
    if (!m->nnz) return;
    memcpy(ri, m->ri, sizeof(int) * m->nnz);
    memcpy(ci, m->ci, sizeof(int) * m->nnz);
    memcpy(v, m->v, sizeof(double) * m->nnz);
}

/* SparseMatrix.mmMul (SparseMatrix.java:549-593): for every merged row i of A
 * and every column j of B, contraction = sum over column j's entries (k, b_kj)
 * of row_i[k] * b_kj, added with SparseMatrix.add (zero sums are not stored,
 * SparseMatrix.java:289).  The reference visits a column's entries in HashMap
 * order; here they are visited in ascending k, row by row with a dense
 * accumulator (the sums of the touched columns are the column contractions;
 * untouched columns contract to zero and are not stored). */
or_mat* or_mat_mmmul(const or_mat* A, const or_mat* B)
{
    if (A->cols != B->rows) return NULL;
    int n = B->cols;
    double* acc = (double*)calloc(n > 0 ? n : 1, sizeof(double));
    char* touched = (char*)calloc(n > 0 ? n : 1, 1);
    int* list = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    long long cap = 1024, m = 0;
    int* ri = (int*)malloc(sizeof(int) * cap);
    int* ci = (int*)malloc(sizeof(int) * cap);
    double* v = (double*)malloc(sizeof(double) * cap);
    for (int i = 0; i < A->rows; i++) {
        int cnt = 0;
        for (long long p = A->rp[i]; p < A->rp[i + 1]; p++) {
            int k = A->rc[p];
            double a = A->rv[p];
            for (long long q = B->rp[k]; q < B->rp[k + 1]; q++) {
                int j = B->rc[q];
                if (!touched[j]) { touched[j] = 1; list[cnt++] = j; acc[j] = 0.0; }
                double prod = a * B->rv[q];
                acc[j] = acc[j] + prod;
            }
        }
        qsort(list, cnt, sizeof(int), cmp_int_asc);
        for (int t = 0; t < cnt; t++) {
            int j = list[t];
            touched[j] = 0;
            if (acc[j] == 0.0) continue;
            if (m == cap) {
                cap *= 2;
                ri = (int*)realloc(ri, sizeof(int) * cap);
                ci = (int*)realloc(ci, sizeof(int) * cap);
                v = (double*)realloc(v, sizeof(double) * cap);
            }
            ri[m] = i; ci[m] = j; v[m] = acc[j]; m++;
        }
    }
    or_mat* C = or_mat_new(A->rows, n, m, ri, ci, v);
    free(acc); free(touched); free(list); free(ri); free(ci); free(v);
    return C;
}

/* SparseMatrix.tvMul (SparseMatrix.java:492-501). */
void or_mat_tvmul(const or_mat* m, const double* x, double* y)
{
    memset(y, 0, sizeof(double) * m->cols);
    for (long long k = 0; k < m->nnz; k++) y[m->ci[k]] += m->v[k] * x[m->ri[k]];
}

void or_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int or_threads(void) { return omp_get_max_threads(); }

/* SparseMvMul.mvMul (SparseMvMul.java:73-94): row-bucketed dot per row. */
void or_mat_mvmul_rows(const or_mat* m, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m->rows; r++) {
        double s = 0;
        for (long long p = m->rp[r]; p < m->rp[r + 1]; p++) s += m->rv[p] * x[m->rc[p]];
        y[r] = s;
    }
}

/* SparseMvMul.tvMul (SparseMvMul.java:96-116): column-bucketed dot per column. */
void or_mat_tvmul_cols(const or_mat* m, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for (int c = 0; c < m->cols; c++) {
        double s = 0;
        for (long long p = m->cp[c]; p < m->cp[c + 1]; p++) s += m->cv[p] * x[m->cr[p]];
        y[c] = s;
    }
}

/* Matrix.diag (Matrix.java:157-175): diagonal with duplicates summed. */
void or_mat_diag(const or_mat* m, double* d)
{
    int n = m->rows < m->cols ? m->rows : m->cols;
    memset(d, 0, sizeof(double) * n);
    for (long long k = 0; k < m->nnz; k++)
        if (m->ri[k] == m->ci[k]) d[m->ri[k]] += m->v[k];
}

/* Densify, row-major, duplicates summed (sparseSolver.cpp:27-31 densifies the same way). */
void or_mat_dense(const or_mat* m, double* a)
{
    memset(a, 0, sizeof(double) * (size_t)m->rows * m->cols);
    for (long long k = 0; k < m->nnz; k++) a[(size_t)m->ri[k] * m->cols + m->ci[k]] += m->v[k];
}

/* ------------------------------------------------------------------ */
/* vectors (DenseVector.java:104-121, 203-260)                          */
/* ------------------------------------------------------------------ */
static double vdot(int n, const double* a, const double* b)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}
static double vnorm(int n, const double* a) { return sqrt(vdot(n, a, a)); }
static double* vnew(int n) { return (double*)calloc(n > 0 ? n : 1, sizeof(double)); }
static double* vdup(int n, const double* a)
{
    double* r = vnew(n);
    memcpy(r, a, sizeof(double) * n);
    return r;
}

double or_dot(int n, const double* a, const double* b) { return vdot(n, a, b); }

/* ------------------------------------------------------------------ */
/* dense LU with partial pivoting (textbook Doolittle)                  */
/* ------------------------------------------------------------------ */
typedef struct { int n; double* lu; int* piv; } or_lu;

static int lu_factor(or_lu* f, int n, const double* a)
{
    f->n = n;
    f->lu = (double*)malloc(sizeof(double) * (size_t)n * n + 8);
    f->piv = (int*)malloc(sizeof(int) * (n ? n : 1));
    memcpy(f->lu, a, sizeof(double) * (size_t)n * n);
    double* A = f->lu;
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(A[(size_t)i * n + k]) > best) { best = fabs(A[(size_t)i * n + k]); p = i; }
        f->piv[k] = p;
        if (best == 0.0) return OR_SINGULAR;
        if (p != k)
            for (int j = 0; j < n; j++) {
                double t = A[(size_t)k * n + j];
                A[(size_t)k * n + j] = A[(size_t)p * n + j];
                A[(size_t)p * n + j] = t;
            }
        double inv = 1.0 / A[(size_t)k * n + k];
        for (int i = k + 1; i < n; i++) {
            double l = A[(size_t)i * n + k] * inv;
            A[(size_t)i * n + k] = l;
            for (int j = k + 1; j < n; j++) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
        }
    }
    return OR_OK;
}

static void lu_solve(const or_lu* f, const double* b, double* x)
{
    int n = f->n;
    const double* A = f->lu;
    if (x != b) memcpy(x, b, sizeof(double) * n);
    for (int k = 0; k < n; k++)
        if (f->piv[k] != k) { double t = x[k]; x[k] = x[f->piv[k]]; x[f->piv[k]] = t; }
    for (int i = 0; i < n; i++) {
        double s = x[i];
        for (int j = 0; j < i; j++) s -= A[(size_t)i * n + j] * x[j];
        x[i] = s;
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int j = i + 1; j < n; j++) s -= A[(size_t)i * n + j] * x[j];
        x[i] = s / A[(size_t)i * n + i];
    }
}

static void lu_free(or_lu* f) { free(f->lu); free(f->piv); f->lu = NULL; f->piv = NULL; }

/* DenseMatrix.solve / sparseSolver.cpp iSolve: A row-major n x n. */
int or_dense_solve(int n, const double* a, const double* b, double* x)
{
    or_lu f;
    int st = lu_factor(&f, n, a);
    if (st == OR_OK) lu_solve(&f, b, x);
    lu_free(&f);
    return st;
}

/* DenseMatrix.inverse / sparseSolver.cpp iInverse. */
int or_dense_inverse(int n, const double* a, double* ainv)
{
    or_lu f;
    int st = lu_factor(&f, n, a);
    if (st == OR_OK) {
        double* e = vnew(n);
        double* col = vnew(n);
        for (int j = 0; j < n; j++) {
            memset(e, 0, sizeof(double) * n);
            e[j] = 1;
            lu_solve(&f, e, col);
            for (int i = 0; i < n; i++) ainv[(size_t)i * n + j] = col[i];
        }
        free(e); free(col);
    }
    lu_free(&f);
    return st;
}

/* ------------------------------------------------------------------ */
/* operators (VectorMultiplyable.java:8-17)                             */
/* ------------------------------------------------------------------ */
typedef struct or_op or_op;
struct or_op {
    int n;
    void (*mv)(const or_op* self, const double* x, double* y);
    const void* data;
    double* tmp;       /* scratch of length n for composed operators */
    const or_op* inner1;
    const or_op* inner2;
};

static void op_mat_mv(const or_op* o, const double* x, double* y) { or_mat_mvmul((const or_mat*)o->data, x, y); }
static void op_id_mv(const or_op* o, const double* x, double* y) { memcpy(y, x, sizeof(double) * o->n); }
/* VectorMultiplyable.concatenate(M, A): x -> M(A x) (VectorMultiplyable.java:114-151). */
static void op_concat_mv(const or_op* o, const double* x, double* y)
{
    o->inner2->mv(o->inner2, x, o->tmp);
    o->inner1->mv(o->inner1, o->tmp, y);
}

or_op* or_op_matrix(const or_mat* m)
{
    or_op* o = (or_op*)calloc(1, sizeof(or_op));
    o->n = m->rows; o->mv = op_mat_mv; o->data = m;
    return o;
}
or_op* or_op_identity(int n)
{
    or_op* o = (or_op*)calloc(1, sizeof(or_op));
    o->n = n; o->mv = op_id_mv;
    return o;
}
static or_op* op_concat(const or_op* M, const or_op* A)
{
    or_op* o = (or_op*)calloc(1, sizeof(or_op));
    o->n = A->n; o->mv = op_concat_mv; o->inner1 = M; o->inner2 = A; o->tmp = vnew(A->n);
    return o;
}
void or_op_free(or_op* o)
{
    if (!o) return;
    free(o->tmp);
    free(o);
}

/* Block-diagonal saddle-point preconditioner: y[0, nv) = vel(x[0, nv)),
 * y[nv, n) = pinv * x[nv, n) (tmp holds pinv, inner1 the velocity operator). */
static void op_blockdiag_mv(const or_op* o, const double* x, double* y)
{
    int nv = o->inner1->n;
    o->inner1->mv(o->inner1, x, y);
    for (int i = nv; i < o->n; i++) y[i] = o->tmp[i - nv] * x[i];
}
or_op* or_op_blockdiag(const or_op* vel, int np, const double* pinv)
{
    or_op* o = (or_op*)calloc(1, sizeof(or_op));
    o->n = vel->n + np; o->mv = op_blockdiag_mv; o->inner1 = vel;
    o->tmp = vnew(np);
    memcpy(o->tmp, pinv, sizeof(double) * np);
    return o;
}
void or_op_apply(const or_op* o, const double* x, double* y) { o->mv(o, x, y); }

/* ------------------------------------------------------------------ */
/* solver bookkeeping                                                   */
/* ------------------------------------------------------------------ */
typedef struct {
    int iterations;      /* IterativeSolver.iterations */
    int restarts;
    int status;
    double final_norm;   /* last published residual norm */
    int hist_len;
} or_info;

typedef struct { double* h; int cap; int len; } hist_t;
static void hist_push(hist_t* h, double v)
{
    if (h->h && h->len < h->cap) h->h[h->len] = v;
    h->len++;
}

/* IterativeSolver.solveCG (IterativeSolver.java:48-100).  x holds the start
 * iterate on entry (e0 or the previous solution, lines 69-72) and the result
 * on exit.  The loop runs while iter < n and ||r|| > tol (line 78). */
int or_solve_cg(const or_op* A, const double* b, double* x, double tol, int maxit,
                or_info* info, double* hist, int hist_cap)
{
    int n = A->n;
    hist_t H = {hist, hist_cap, 0};
    if (maxit <= 0) maxit = n;
    double* z = vnew(n);
    double* r = vnew(n);
    double* d = vnew(n);
    A->mv(A, x, z);
    for (int i = 0; i < n; i++) r[i] = b[i] - z[i];
    memcpy(d, r, sizeof(double) * n);
    int it = 0, st = OR_MAXITER;
    double rn = vnorm(n, r);
    for (int iter = 0; iter < maxit; iter++) {
        if (!(rn > tol)) { st = OR_OK; break; }
        if (!isfinite(rn)) { st = OR_NONFINITE; break; }
        A->mv(A, d, z);
        double rr = vdot(n, r, r);
        double alpha = rr / vdot(n, d, z);
        for (int i = 0; i < n; i++) x[i] += d[i] * alpha;
        for (int i = 0; i < n; i++) r[i] = r[i] - z[i] * alpha;   /* newResiduum */
        double beta = vdot(n, r, r) / rr;
        for (int i = 0; i < n; i++) d[i] = r[i] + d[i] * beta;
        rn = vnorm(n, r);
        hist_push(&H, rn);
        it++;
    }
    if (st == OR_MAXITER && !(rn > tol)) st = OR_OK;
    if (info) { info->iterations = it; info->status = st; info->final_norm = rn; info->hist_len = H.len; info->restarts = 0; }
    free(z); free(r); free(d);
    return st;
}

/* IterativeSolver.solvePCG (IterativeSolver.java:102-162). */
int or_solve_pcg(const or_op* A, const or_op* M, const double* b, double* x, double tol, int maxit,
                 or_info* info, double* hist, int hist_cap)
{
    int n = A->n;
    hist_t H = {hist, hist_cap, 0};
    if (maxit <= 0) maxit = n;
    double* Ap = vnew(n);
    double* r = vnew(n);
    double* z = vnew(n);
    double* p = vnew(n);
    A->mv(A, x, Ap);
    for (int i = 0; i < n; i++) r[i] = b[i] - Ap[i];
    M->mv(M, r, z);
    memcpy(p, z, sizeof(double) * n);
    int it = 0, st = OR_MAXITER;
    double rn = vnorm(n, r);
    for (int iter = 0; iter < maxit; iter++) {
        if (!(rn > tol)) { st = OR_OK; break; }
        if (!isfinite(rn)) { st = OR_NONFINITE; break; }
        A->mv(A, p, Ap);
        double rz = vdot(n, r, z);
        double alpha = rz / vdot(n, p, Ap);
        for (int i = 0; i < n; i++) x[i] += p[i] * alpha;
        for (int i = 0; i < n; i++) r[i] = r[i] - Ap[i] * alpha;
        M->mv(M, r, z);                         /* newZ */
        double beta = vdot(n, r, z) / rz;
        for (int i = 0; i < n; i++) p[i] = z[i] + p[i] * beta;
        rn = vnorm(n, r);
        hist_push(&H, rn);
        it++;
    }
    if (st == OR_MAXITER && !(rn > tol)) st = OR_OK;
    if (info) { info->iterations = it; info->status = st; info->final_norm = rn; info->hist_len = H.len; info->restarts = 0; }
    free(Ap); free(r); free(z); free(p);
    return st;
}

/* ------------------------------------------------------------------ */
/* GMRES (GMRES.java)                                                   */
/* ------------------------------------------------------------------ */
/* calculateAlpha (GMRES.java:239-251): back substitution on the rotated
 * Hessenberg matrix; h is (ldh x ldh) row-major. */
static void gm_alpha(const double* gamma, const double* h, int ldh, int j, double* alpha)
{
    for (int i = j; i >= 0; i--) {
        double s = 0;
        for (int k = i + 1; k <= j; k++) s += h[(size_t)i * ldh + k] * alpha[k];
        alpha[i] = 1.0 / h[(size_t)i * ldh + i] * (gamma[i] - s);
    }
}

/* One GMRES cycle plus the restart rule (GMRES.java:64-134).  M may be NULL
 * (unpreconditioned solve, GMRES.java:103-134).  Restarts are iterative here
 * rather than recursive; total restarts are capped at max_restarts. */
int or_solve_gmres(const or_op* A, const or_op* M, const double* b, double* x, double tol,
                   int restart_len, int max_restarts, or_info* info, double* hist, int hist_cap)
{
    int n = A->n;
    hist_t H = {hist, hist_cap, 0};
    int IBR = restart_len > 0 ? restart_len : 150;   /* ITERATIONS_BEFORE_RESTART */
    if (max_restarts < 0) max_restarts = 200;       /* MAX_RESTARTS */
    int ldh = IBR + 10;
    double* h = (double*)calloc((size_t)ldh * ldh, sizeof(double));
    double* gamma = vnew(ldh);
    double* cs = vnew(ldh);
    double* sn = vnew(ldh);
    double* alpha = vnew(ldh);
    int vcap = IBR + 3;
    double** V = (double**)calloc(vcap, sizeof(double*));
    double* q = vnew(n);
    double* t = vnew(n);
    double* w = vnew(n);
    double* res = vnew(n);
    double* fac = vnew(vcap);
    int restarts = 0, total_it = 0, st = OR_MAXITER;
    double last_norm = 0;
    for (;;) {
        /* r = M(b - A x) or b - A x */
        A->mv(A, x, t);
        for (int i = 0; i < n; i++) t[i] = b[i] - t[i];
        if (M) M->mv(M, t, res); else memcpy(res, t, sizeof(double) * n);
        double rn = vnorm(n, res);
        if (rn <= tol) { st = OR_OK; last_norm = rn; break; }
        if (!isfinite(rn)) { st = OR_NONFINITE; break; }
        memset(h, 0, sizeof(double) * (size_t)ldh * ldh);
        memset(gamma, 0, sizeof(double) * ldh);
        gamma[0] = rn;
        if (!V[0]) V[0] = vnew(n);
        for (int i = 0; i < n; i++) V[0][i] = res[i] * (1.0 / gamma[0]);
        int nv = 1;
        /* innerGMRES (GMRES.java:136-176) */
        int j;
        for (j = 0; j < n; j++) {
            A->mv(A, V[j], t);
            if (M) M->mv(M, t, q); else memcpy(q, t, sizeof(double) * n);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < nv; i++) fac[i] = vdot(n, V[i], q);     /* calculateOrthogonalityFactors */
            memset(w, 0, sizeof(double) * n);                         /* linearCombination */
            for (int i = 0; i < nv; i++)
                for (int k = 0; k < n; k++) w[k] = w[k] + V[i][k] * fac[i];
            for (int k = 0; k < n; k++) w[k] = q[k] - w[k];
            for (int i = 0; i < nv; i++) h[(size_t)i * ldh + j] += fac[i];  /* addColumn */
            double wn = vnorm(n, w);
            h[(size_t)(j + 1) * ldh + j] += wn;
            for (int i = 0; i < j; i++) {                               /* calculateGivens */
                double hij = h[(size_t)i * ldh + j], hipj = h[(size_t)(i + 1) * ldh + j];
                h[(size_t)i * ldh + j] = hij * cs[i] + hipj * sn[i];
                h[(size_t)(i + 1) * ldh + j] = -hij * sn[i] + hipj * cs[i];
            }
            double hjj = h[(size_t)j * ldh + j], hj1 = h[(size_t)(j + 1) * ldh + j];
            double beta = sqrt(hjj * hjj + hj1 * hj1);
            sn[j] = hj1 / beta;
            cs[j] = hjj / beta;
            h[(size_t)j * ldh + j] = beta;
            gamma[j + 1] = -sn[j] * gamma[j];
            gamma[j] = cs[j] * gamma[j];
            last_norm = fabs(gamma[j + 1]);
            hist_push(&H, last_norm);
            if (fabs(gamma[j + 1]) < tol || j > IBR) break;
            if (!isfinite(gamma[j + 1])) break;
            if (!V[j + 1]) V[j + 1] = vnew(n);
            double inv = 1.0 / h[(size_t)(j + 1) * ldh + j];
            for (int k = 0; k < n; k++) V[j + 1][k] = w[k] * inv;
            nv++;
            total_it++;
        }
        if (j == n) j--;
        gm_alpha(gamma, h, ldh, j, alpha);
        for (int i = 0; i <= j; i++)
            for (int k = 0; k < n; k++) x[k] = x[k] + V[i][k] * alpha[i];   /* x.add(alphaV) */
        A->mv(A, x, t);
        for (int i = 0; i < n; i++) t[i] = t[i] - b[i];
        double residual = vnorm(n, t);
        last_norm = residual;
        if (!isfinite(residual)) { st = OR_NONFINITE; break; }
        if ((j > IBR && restarts < max_restarts) || residual > tol) {
            if (restarts >= max_restarts) { st = OR_MAXITER; break; }
            restarts++;
            continue;
        }
        st = OR_OK;
        break;
    }
    if (info) { info->iterations = total_it; info->restarts = restarts; info->status = st; info->final_norm = last_norm; info->hist_len = H.len; }
    for (int i = 0; i < vcap; i++) free(V[i]);
    free(V); free(h); free(gamma); free(cs); free(sn); free(alpha);
    free(q); free(t); free(w); free(res); free(fac);
    return st;
}

/* ------------------------------------------------------------------ */
/* BiCGStab (IterativeSolver.java:256-323) and PBiCGStab (:325-402)     */
/* ------------------------------------------------------------------ */
int or_solve_bicgstab(const or_op* A, const double* b, double* x, double tol, int maxit,
                      or_info* info, double* hist, int hist_cap)
{
    int n = A->n;
    hist_t H = {hist, hist_cap, 0};
    if (maxit <= 0) maxit = n;
    double* v = vnew(n);
    double* s = vnew(n);
    double* t = vnew(n);
    double* r0 = vnew(n);
    double* r = vnew(n);
    double* p = vnew(n);
    double* x0 = vdup(n, x);
    A->mv(A, x, t);
    for (int i = 0; i < n; i++) r0[i] = b[i] - t[i];
    memcpy(r, r0, sizeof(double) * n);
    double alpha = 1, omega = 1, rho = 1, rhoLast = 1, beta = 1;
    int it = 0, st = OR_MAXITER;
    double rn = vnorm(n, r);
    for (int iter = 0; iter < maxit; iter++) {
        if (!(rn > tol)) { st = OR_OK; break; }
        rho = vdot(n, r, r0);
        if (fabs(rhoLast) < tol) {
            /* breakdown: falls back to solveGMRES (line 294) from the start iterate */
            memcpy(x, x0, sizeof(double) * n);
            or_info gi;
            int gst = or_solve_gmres(A, NULL, b, x, tol, 150, 200, &gi, NULL, 0);
            if (info) { info->iterations = it + gi.iterations; info->status = gst == OR_OK ? OR_BREAKDOWN : gst; info->final_norm = gi.final_norm; info->hist_len = H.len; info->restarts = gi.restarts; }
            free(v); free(s); free(t); free(r0); free(r); free(p); free(x0);
            return gst == OR_OK ? OR_BREAKDOWN : gst;
        }
        beta = alpha / omega * rho / rhoLast;
        for (int i = 0; i < n; i++) p[i] = (r[i] + p[i] * beta) - v[i] * (omega * beta);
        A->mv(A, p, v);
        alpha = rho / vdot(n, v, r0);
        for (int i = 0; i < n; i++) s[i] = r[i] - v[i] * alpha;
        double sn = vnorm(n, s);
        if (sn < tol) {
            for (int i = 0; i < n; i++) x[i] = x[i] + p[i] * alpha;
            rn = sn;
            st = OR_OK;
            break;
        }
        A->mv(A, s, t);
        omega = vdot(n, t, s) / vdot(n, t, t);
        for (int i = 0; i < n; i++) x[i] = (x[i] + p[i] * alpha) + s[i] * omega;
        for (int i = 0; i < n; i++) r[i] = s[i] - t[i] * omega;
        rhoLast = rho;
        rn = vnorm(n, r);
        hist_push(&H, rn);
        it++;
        if (!isfinite(rn)) { st = OR_NONFINITE; break; }
    }
    if (st == OR_MAXITER && !(rn > tol)) st = OR_OK;
    if (info) { info->iterations = it; info->status = st; info->final_norm = rn; info->hist_len = H.len; info->restarts = 0; }
    free(v); free(s); free(t); free(r0); free(r); free(p); free(x0);
    return st;
}

int or_solve_pbicgstab(const or_op* A, const or_op* M, const double* b, double* x, double tol, int maxit,
                       or_info* info, double* hist, int hist_cap)
{
    int n = A->n;
    hist_t H = {hist, hist_cap, 0};
    if (maxit <= 0) maxit = 10 * n;      /* line 366: iter < n * 10 */
    double* v = vnew(n);
    double* y = vnew(n);
    double* z = vnew(n);
    double* pt = vnew(n);
    double* p = vnew(n);
    double* s = vnew(n);
    double* t = vnew(n);
    double* r0 = vnew(n);
    double* r = vnew(n);
    A->mv(A, x, t);
    for (int i = 0; i < n; i++) r0[i] = b[i] - t[i];
    memcpy(r, r0, sizeof(double) * n);
    double alpha = 1, omega = 1, rho = 1, rhoLast = 1, beta = 1;
    int it = 0, st = OR_MAXITER;
    double rn = vnorm(n, r);
    for (int iter = 0; iter < maxit; iter++) {
        if (!(rn > tol)) { st = OR_OK; break; }
        rho = vdot(n, r, r0);
        if (fabs(rhoLast) < tol) {
            /* breakdown: falls back to solvePGMRES (line 370), which starts from zero */
            memset(x, 0, sizeof(double) * n);
            or_info gi;
            int gst = or_solve_gmres(A, M, b, x, tol, 150, 200, &gi, NULL, 0);
            if (info) { info->iterations = it + gi.iterations; info->status = gst == OR_OK ? OR_BREAKDOWN : gst; info->final_norm = gi.final_norm; info->hist_len = H.len; info->restarts = gi.restarts; }
            free(v); free(y); free(z); free(pt); free(p); free(s); free(t); free(r0); free(r);
            return gst == OR_OK ? OR_BREAKDOWN : gst;
        }
        beta = alpha / omega * rho / rhoLast;
        for (int i = 0; i < n; i++) p[i] = (r[i] + p[i] * beta) - v[i] * (omega * beta);
        M->mv(M, p, y);
        A->mv(A, y, v);
        alpha = rho / vdot(n, v, r0);
        for (int i = 0; i < n; i++) s[i] = r[i] - v[i] * alpha;
        double sn = vnorm(n, s);
        if (sn < tol) {
            for (int i = 0; i < n; i++) x[i] = x[i] + y[i] * alpha;
            rn = sn;
            st = OR_OK;
            break;
        }
        M->mv(M, s, z);
        A->mv(A, z, t);
        M->mv(M, t, pt);
        omega = vdot(n, pt, z) / vdot(n, pt, pt);
        for (int i = 0; i < n; i++) x[i] = (x[i] + y[i] * alpha) + z[i] * omega;
        for (int i = 0; i < n; i++) r[i] = s[i] - t[i] * omega;
        rhoLast = rho;
        rn = vnorm(n, r);
        hist_push(&H, rn);
        it++;
        if (!isfinite(rn)) { st = OR_NONFINITE; break; }
    }
    if (st == OR_MAXITER && !(rn > tol)) st = OR_OK;
    if (info) { info->iterations = it; info->status = st; info->final_norm = rn; info->hist_len = H.len; info->restarts = 0; }
    free(v); free(y); free(z); free(pt); free(p); free(s); free(t); free(r0); free(r);
    return st;
}

/* ------------------------------------------------------------------ */
/* GMRES2 (GMRES2.java:60-104) with Arnoldi (Arnoldi.java:13-83)        */
/* ------------------------------------------------------------------ */
static void normalized(int n, const double* a, double* out)
{
    double inv = 1.0 / vnorm(n, a);
    for (int i = 0; i < n; i++) out[i] = a[i] * inv;
}

int or_solve_gmres2(const or_op* A, const or_op* M, const double* b, double* x, double tol,
                    int maxit, int max_restarts, or_info* info, double* hist, int hist_cap)
{
    int n = A->n;
    hist_t H = {hist, hist_cap, 0};
    if (maxit <= 0) maxit = 10 * n + 10;
    if (max_restarts < 0) max_restarts = 200;
    or_op* Mid = NULL;
    if (!M) { Mid = or_op_identity(n); M = Mid; }
    or_op* MA = op_concat(M, A);
    int vcap = 16;
    double** Vs = (double**)calloc(vcap, sizeof(double*));
    double** AVs = (double**)calloc(vcap, sizeof(double*));
    double* res = vnew(n);
    double* Mres = vnew(n);
    double* qlast = vnew(n);   /* the latest q of the Arnoldi object */
    double* wq = vnew(n);
    double* w = vnew(n);
    double* naw = vnew(n);
    double* t = vnew(n);
    int it = 0, restarts = 0, st = OR_MAXITER;
    double rn = 0;
    for (;;) {
        /* solveInternal (GMRES2.java:60-69) */
        A->mv(A, x, t);
        for (int i = 0; i < n; i++) res[i] = b[i] - t[i];
        M->mv(M, res, Mres);
        int nv = 0;
        /* Arnoldi(Mres, MA) constructor (Arnoldi.java:13-31) */
        normalized(n, Mres, wq);                 /* w0 = latestQNormalized() */
        MA->mv(MA, wq, qlast);                   /* addQ(): q1 = MA(w0) */
        double an = vnorm(n, qlast);             /* Aw0 = latestQ() */
        if (!Vs[0]) { Vs[0] = vnew(n); AVs[0] = vnew(n); }
        for (int i = 0; i < n; i++) { Vs[0][i] = wq[i] * (1.0 / an); AVs[0][i] = qlast[i] * (1.0 / an); }
        nv = 1;
        normalized(n, qlast, wq);
        MA->mv(MA, wq, t);                       /* addQ(): q2 = MA(q1 normalized) */
        memcpy(qlast, t, sizeof(double) * n);
        rn = vnorm(n, res);
        int restart = 0;
        while (rn > tol) {
            if (it >= maxit) break;
            const double* v = Vs[nv - 1];
            const double* Av = AVs[nv - 1];
            double tt = vdot(n, Mres, Av) / vdot(n, Av, Av);
            for (int i = 0; i < n; i++) x[i] = x[i] + v[i] * tt;
            A->mv(A, v, t);
            for (int i = 0; i < n; i++) res[i] = res[i] - t[i] * tt;
            for (int i = 0; i < n; i++) Mres[i] = Mres[i] - Av[i] * tt;
            rn = vnorm(n, res);
            hist_push(&H, rn);
            it++;
            if (!isfinite(rn)) { st = OR_NONFINITE; break; }
            /* arnoldiStep (Arnoldi.java:63-82) */
            normalized(n, qlast, w);             /* w = latestQNormalized() */
            MA->mv(MA, w, naw);                  /* addQ(); newAw = latestQ() */
            memcpy(qlast, naw, sizeof(double) * n);
            for (int i = 0; i < nv; i++) {
                double proj = vdot(n, naw, AVs[i]);
                for (int k = 0; k < n; k++) w[k] = w[k] - Vs[i][k] * proj;
                for (int k = 0; k < n; k++) naw[k] = naw[k] - AVs[i][k] * proj;
            }
            double nn = vnorm(n, naw);
            if (nv == vcap) {
                vcap *= 2;
                Vs = (double**)realloc(Vs, sizeof(double*) * vcap);
                AVs = (double**)realloc(AVs, sizeof(double*) * vcap);
                for (int i = nv; i < vcap; i++) { Vs[i] = NULL; AVs[i] = NULL; }
            }
            if (!Vs[nv]) { Vs[nv] = vnew(n); AVs[nv] = vnew(n); }
            for (int k = 0; k < n; k++) { Vs[nv][k] = w[k] * (1.0 / nn); AVs[nv][k] = naw[k] * (1.0 / nn); }
            nv++;
            if (nn < 1e-13) { restart = 1; break; }
        }
        if (st == OR_NONFINITE) break;
        if (!(rn > tol)) { st = OR_OK; break; }
        if (restart && restarts < max_restarts) { restarts++; continue; }
        st = OR_MAXITER;
        break;
    }
    if (info) { info->iterations = it; info->restarts = restarts; info->status = st; info->final_norm = rn; info->hist_len = H.len; }
    for (int i = 0; i < vcap; i++) { free(Vs[i]); free(AVs[i]); }
    free(Vs); free(AVs); free(res); free(Mres); free(qlast); free(wq); free(w); free(naw); free(t);
    or_op_free(MA);
    or_op_free(Mid);
    return st;
}

/* ------------------------------------------------------------------ */
/* Schwarz subspace corrections (schwarz/*.java)                        */
/* ------------------------------------------------------------------ */
#define OR_SCHWARZ_MULT 0
#define OR_SCHWARZ_COLORED 1
#define OR_SCHWARZ_ADDITIVE 2

typedef struct or_schwarz {
    const or_mat* A;
    int n, kind, np, nc;
    double omega;
    long long* pptr; int* dofs;       /* patch DOF lists, ascending (TreeSet by global index) */
    int* cptr; int* cpat;             /* colours: ascending patch lists (IntRBTreeSet) */
    double** inv;                     /* DirectSolver cache: dense inverse of R A R^T per patch */
    int status;
} or_schwarz;

static int cmp_int(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* UpFrontSchwarz.build (UpFrontSchwarz.java:25-59) with
 * RestrictionMatrix.selectFrom (RestrictionMatrix.java:22-43): the local
 * operator keeps the merged entries whose row and column both lie in the
 * patch; DirectSolver.solve (DirectSolver.java:22-38) caches its inverse. */
or_schwarz* or_schwarz_new(const or_mat* A, int kind, double omega, int np, const long long* pptr,
                           const int* dofs, int nc, const int* cptr, const int* cpat)
{
    or_schwarz* S = (or_schwarz*)calloc(1, sizeof(or_schwarz));
    S->A = A; S->n = A->rows; S->kind = kind; S->omega = omega; S->np = np; S->nc = nc;
    S->pptr = (long long*)malloc(sizeof(long long) * (np + 1));
    memcpy(S->pptr, pptr, sizeof(long long) * (np + 1));
    S->dofs = (int*)malloc(sizeof(int) * (pptr[np] ? pptr[np] : 1));
    memcpy(S->dofs, dofs, sizeof(int) * pptr[np]);
    for (int p = 0; p < np; p++)
        qsort(S->dofs + pptr[p], (size_t)(pptr[p + 1] - pptr[p]), sizeof(int), cmp_int);
    if (kind == OR_SCHWARZ_COLORED) {
        S->cptr = (int*)malloc(sizeof(int) * (nc + 1));
        memcpy(S->cptr, cptr, sizeof(int) * (nc + 1));
        S->cpat = (int*)malloc(sizeof(int) * (cptr[nc] ? cptr[nc] : 1));
        memcpy(S->cpat, cpat, sizeof(int) * cptr[nc]);
        for (int c = 0; c < nc; c++) qsort(S->cpat + cptr[c], (size_t)(cptr[c + 1] - cptr[c]), sizeof(int), cmp_int);
    }
    S->inv = (double**)calloc(np, sizeof(double*));
    int* loc = (int*)malloc(sizeof(int) * (S->n ? S->n : 1));
    for (int i = 0; i < S->n; i++) loc[i] = -1;
    for (int p = 0; p < np && S->status == OR_OK; p++) {
        int m = (int)(pptr[p + 1] - pptr[p]);
        const int* d = S->dofs + pptr[p];
        for (int i = 0; i < m; i++) loc[d[i]] = i;
        double* a = (double*)calloc((size_t)m * m, sizeof(double));
        for (int i = 0; i < m; i++) {
            int g = d[i];
            for (long long k = A->rp[g]; k < A->rp[g + 1]; k++) {
                int j = loc[A->rc[k]];
                if (j >= 0) a[(size_t)i * m + j] += A->rv[k];
            }
        }
        S->inv[p] = (double*)malloc(sizeof(double) * (size_t)m * m);
        if (or_dense_inverse(m, a, S->inv[p]) != OR_OK) S->status = OR_SINGULAR;
        free(a);
        for (int i = 0; i < m; i++) loc[d[i]] = -1;
    }
    free(loc);
    return S;
}

int or_schwarz_status(const or_schwarz* S) { return S->status; }

void or_schwarz_free(or_schwarz* S)
{
    if (!S) return;
    for (int p = 0; p < S->np; p++) free(S->inv[p]);
    free(S->inv); free(S->pptr); free(S->dofs); free(S->cptr); free(S->cpat);
    free(S);
}

/* getGlobalVector(p, solveLocalSystem(p, getLocalVector(p, r))) as a dense
 * global vector comp (zero outside the patch). */
static void patch_component(const or_schwarz* S, int p, const double* r, double* comp)
{
    int m = (int)(S->pptr[p + 1] - S->pptr[p]);
    const int* d = S->dofs + S->pptr[p];
    double* loc = vnew(m);
    for (int i = 0; i < m; i++) loc[i] = r[d[i]];
    memset(comp, 0, sizeof(double) * S->n);
    const double* iv = S->inv[p];
    for (int i = 0; i < m; i++) {
        double acc = 0;
        for (int j = 0; j < m; j++) acc += iv[(size_t)i * m + j] * loc[j];
        comp[d[i]] = acc;
    }
    free(loc);
}

static void residual(const or_schwarz* S, const double* rhs, const double* x, double* r)
{
    or_mat_mvmul(S->A, x, r);
    for (int i = 0; i < S->n; i++) r[i] = rhs[i] - r[i];
}

/* MultiplicativeSubspaceCorrection.upgradePatch (:61-81) and
 * ColoredMultiplicativeSubspaceCorrection.colorSetUpgrade (:84-123). */
static void colour_upgrade(const or_schwarz* S, const int* patches, int count, double om, const double* rhs,
                           double* x, double* r, double* comp)
{
    residual(S, rhs, x, r);
    double** comps = (double**)malloc(sizeof(double*) * (count ? count : 1));
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < count; q++) {
        comps[q] = vnew(S->n);
        patch_component(S, patches[q], r, comps[q]);
    }
    for (int q = 0; q < count; q++) {
        for (int i = 0; i < S->n; i++) x[i] = x[i] + comps[q][i] * om;
        free(comps[q]);
    }
    free(comps);
    (void)comp;
}

/* SubspaceCorrection.apply: x <- new iterate. */
void or_schwarz_apply(const or_schwarz* S, double* x, const double* rhs)
{
    int n = S->n;
    double* r = vnew(n);
    double* comp = vnew(n);
    if (S->kind == OR_SCHWARZ_MULT) {           /* MultiplicativeSubspaceCorrection.apply (:46-59) */
        for (int p = 0; p < S->np; p++) {
            residual(S, rhs, x, r);
            patch_component(S, p, r, comp);
            for (int i = 0; i < n; i++) x[i] = x[i] + comp[i];
        }
        for (int p = S->np - 1; p >= 0; p--) {
            residual(S, rhs, x, r);
            patch_component(S, p, r, comp);
            for (int i = 0; i < n; i++) x[i] = x[i] + comp[i];
        }
    } else if (S->kind == OR_SCHWARZ_COLORED) { /* ColoredMultiplicativeSubspaceCorrection.apply (:68-82) */
        for (int c = 0; c < S->nc; c++)
            colour_upgrade(S, S->cpat + S->cptr[c], S->cptr[c + 1] - S->cptr[c], S->omega, rhs, x, r, comp);
        for (int c = S->nc - 1; c >= 0; c--)
            colour_upgrade(S, S->cpat + S->cptr[c], S->cptr[c + 1] - S->cptr[c], S->omega, rhs, x, r, comp);
    } else {                                    /* SubspaceCorrection.apply default (:11-18) */
        residual(S, rhs, x, r);
        double* sol = vnew(n);
        for (int p = 0; p < S->np; p++) {       /* AdditiveSubspaceCorrection.solve (:22-46) */
            patch_component(S, p, r, comp);
            for (int i = 0; i < n; i++) sol[i] = sol[i] + comp[i] * S->omega;
        }
        for (int i = 0; i < n; i++) x[i] = x[i] + sol[i];
        free(sol);
    }
    free(r); free(comp);
}

/* SubspaceCorrection.solve = AbstractSchwarz.mvMul. */
void or_schwarz_solve(const or_schwarz* S, const double* rhs, double* out)
{
    int n = S->n;
    double* r = vnew(n);
    double* comp = vnew(n);
    memset(out, 0, sizeof(double) * n);
    if (S->kind == OR_SCHWARZ_ADDITIVE) {
        for (int p = 0; p < S->np; p++) {
            patch_component(S, p, rhs, comp);
            for (int i = 0; i < n; i++) out[i] = out[i] + comp[i] * S->omega;
        }
    } else {
        patch_component(S, 0, rhs, out);        /* the first patch alone (:32-35 of both) */
        if (S->kind == OR_SCHWARZ_MULT) {
            for (int p = 1; p < S->np; p++) {
                residual(S, rhs, out, r);
                patch_component(S, p, r, comp);
                for (int i = 0; i < n; i++) out[i] = out[i] + comp[i];
            }
        } else {
            for (int c = 0; c < S->nc; c++)
                colour_upgrade(S, S->cpat + S->cptr[c], S->cptr[c + 1] - S->cptr[c], S->omega, rhs, out, r, comp);
        }
    }
    free(r); free(comp);
}

/* SchwarzSmoother.smooth (SchwarzSmoother.java:21-43). */
void or_schwarz_smooth(const or_schwarz* S, int runs, const double* rhs, double* x)
{
    for (int i = 0; i < runs; i++) or_schwarz_apply(S, x, rhs);
}

/* the cached inverse of patch p (m*m, row-major) */
const double* or_schwarz_inverse(const or_schwarz* S, int p, int* m)
{
    *m = (int)(S->pptr[p + 1] - S->pptr[p]);
    return S->inv[p];
}

/* ------------------------------------------------------------------ */
/* smoothers                                                            */
/* ------------------------------------------------------------------ */
#define OR_SMOOTH_JACOBI 0
#define OR_SMOOTH_RICHARDSON 1

#define OR_SMOOTH_SCHWARZ 2
#define OR_SMOOTH_FBGS 3
#define OR_SMOOTH_GS 4

typedef struct {
    int kind, runs;
    double omega;
    double* dinv;      /* Jacobi: 1/diag with |d| < 1e-10 -> 1 (JacobiSmoother.java:16-24) */
    const or_schwarz* schwarz;   /* SchwarzSmoother: its own decomposition and global operator */
    const int* rank;   /* Gauss-Seidel: position of each row in the ordering (NULL: natural) */
} or_smoother;

/* Triangular solve of the lower (lower != 0) or upper triangle of A with the
 * diagonal, rows visited in rank order (upper: reverse), each row as
 * LowerTriangularSparseMatrix.backsubstituteRow / UpperTriangularSparseMatrix.
 * forwardsubstituteRow do (LowerTriangularSparseMatrix.java:188-212,
 * UpperTriangularSparseMatrix.java:197-221): sol_i = rhs_i / d, then
 * sol_i += (-sol_j / d) * a_ij over the row's other triangle entries, here in
 * ascending column order (the reference: HashMap order of its row bucket).
 * scale != 0 uses d_i * rhs_i as the right-hand side (D.mvMul first). */
static void gs_trsv(const or_mat* A, int lower, const int* rank, const int* order, const double* diag,
                    const double* rhs, int scale, double* sol)
{
    int n = A->rows;
    for (int p = 0; p < n; p++) {
        int i = order[lower ? p : n - 1 - p];
        double d = diag[i];
        double r = scale ? d * rhs[i] : rhs[i];
        double s = r / d;
        for (long long q = A->rp[i]; q < A->rp[i + 1]; q++) {
            int j = A->rc[q];
            if (j == i) continue;
            int in = lower ? rank[j] < rank[i] : rank[j] > rank[i];
            if (!in) continue;
            double t = -sol[j] / d;
            s = s + t * A->rv[q];
        }
        sol[i] = s;
    }
}

/* ForwardBackwardGaussSeidelSmoother.smooth (ForwardBackwardGaussSeidelSmoother.java:23-44):
 * runs x { x += L^-1 D U^-1 (b - A x) };  GaussSeidelSmoother.smooth
 * (GaussSeidelSmoother.java:24-32): runs x { x = (L + D)^-1 (b - R x) }, the
 * dense inverse of L + D restated as a forward substitution.  rank == NULL:
 * the natural row order.  Returns OR_SINGULAR for a zero diagonal entry. */
int or_gs_smooth(const or_mat* A, int kind, int runs, const int* rank_in, const double* rhs, double* x)
{
    int n = A->rows;
    if (A->rows != A->cols) return OR_BADARG;
    int* rank = (int*)malloc(sizeof(int) * (n ? n : 1));
    int* order = (int*)malloc(sizeof(int) * (n ? n : 1));
    double* diag = vnew(n);
    for (int i = 0; i < n; i++) rank[i] = rank_in ? rank_in[i] : i;
    for (int i = 0; i < n; i++) order[rank[i]] = i;
    or_mat_diag(A, diag);
    int st = OR_OK;
    for (int i = 0; i < n; i++)
        if (diag[i] == 0.0) st = OR_SINGULAR;
    double* r = vnew(n);
    double* y = vnew(n);
    double* w = vnew(n);
    for (int it = 0; st == OR_OK && it < runs; it++) {
        if (kind == OR_SMOOTH_FBGS) {
            or_mat_mvmul(A, x, r);
            for (int i = 0; i < n; i++) r[i] = rhs[i] - r[i];
            gs_trsv(A, 0, rank, order, diag, r, 0, y);
            gs_trsv(A, 1, rank, order, diag, y, 1, w);
            for (int i = 0; i < n; i++) x[i] = x[i] + w[i];
        } else {
            for (int i = 0; i < n; i++) {
                double s = 0;
                for (long long q = A->rp[i]; q < A->rp[i + 1]; q++) {
                    int j = A->rc[q];
                    if (j != i && rank[j] > rank[i]) s = s + A->rv[q] * x[j];
                }
                r[i] = rhs[i] - s;
            }
            gs_trsv(A, 1, rank, order, diag, r, 0, x);
        }
    }
    free(rank); free(order); free(diag); free(r); free(y); free(w);
    return st;
}

/* JacobiSmoother.smooth (JacobiSmoother.java:28-50) and RichardsonSmoother.smooth
 * (RichardsonSmoother.java:31-50, unpreconditioned form).  x is updated in place. */
static void smooth(const or_smoother* s, const or_mat* A, const double* rhs, double* x, double* r)
{
    int n = A->rows;
    if (s->kind == OR_SMOOTH_SCHWARZ) {
        or_schwarz_smooth(s->schwarz, s->runs, rhs, x);
        return;
    }
    if (s->kind == OR_SMOOTH_FBGS || s->kind == OR_SMOOTH_GS) {
        or_gs_smooth(A, s->kind, s->runs, s->rank, rhs, x);
        return;
    }
    for (int it = 0; it < s->runs; it++) {
        or_mat_mvmul(A, x, r);
        for (int i = 0; i < n; i++) r[i] = rhs[i] - r[i];
        if (s->kind == OR_SMOOTH_JACOBI) {
            for (int i = 0; i < n; i++) x[i] = x[i] + (s->dinv[i] * r[i]) * s->omega;
        } else {
            if (vnorm(n, r) < 1e-10) break;
            for (int i = 0; i < n; i++) x[i] = x[i] + r[i] * s->omega;
        }
    }
}

static void smoother_init(or_smoother* s, int kind, int runs, double omega, const or_mat* A)
{
    s->kind = kind; s->runs = runs; s->omega = omega; s->dinv = NULL; s->schwarz = NULL; s->rank = NULL;
    if (kind == OR_SMOOTH_JACOBI) {
        s->dinv = vnew(A->rows);
        or_mat_diag(A, s->dinv);
        for (int i = 0; i < A->rows; i++) {
            double d = s->dinv[i];
            if (fabs(d) < 1e-10) d = 1;
            s->dinv[i] = 1.0 / d;
        }
    }
}

/* Standalone smoother call: Smoother.smooth(A, rhs, x). */
void or_smooth(const or_mat* A, int kind, int runs, double omega, const double* rhs, double* x)
{
    or_smoother s;
    smoother_init(&s, kind, runs, omega, A);
    double* r = vnew(A->rows);
    smooth(&s, A, rhs, x, r);
    free(r);
    free(s.dinv);
}

/* ------------------------------------------------------------------ */
/* geometric multigrid (MGPreconditionerInterface / MGPreconditionerSpace) */
/* ------------------------------------------------------------------ */
typedef struct or_mg {
    int L;                  /* number of levels; level L-1 is the finest */
    const or_mat** A;       /* systems per level */
    const or_mat** P;       /* P[l]: n_{l+1} x n_l nodal prolongation */
    int** bd; int* nbd;     /* boundary node lists per level */
    or_smoother* sm;        /* smoothers per level (index 0 unused) */
    or_lu coarse;           /* factorised level-0 matrix */
    int coarse_status;
    int cycles;
} or_mg;

static void zero_bc(const or_mg* g, int l, double* v)
{
    for (int i = 0; i < g->nbd[l]; i++) v[g->bd[l][i]] = 0;
}

/* Prolongation operator mvMul: P v, then zero boundary on the fine level
 * (MGPreconditionerSpace.java:92-100). */
static void mg_prolong(const or_mg* g, int l, const double* vc, double* vf)
{
    or_mat_mvmul(g->P[l], vc, vf);
    zero_bc(g, l + 1, vf);
}
/* Prolongation operator tvMul: SparseMvMul.tvMul, then zero boundary on the
 * coarse level (MGPreconditionerSpace.java:101-107). */
static void mg_restrict(const or_mg* g, int l, const double* vf, double* vc)
{
    or_mat_tvmul_cols(g->P[l], vf, vc);
    zero_bc(g, l, vc);
}

or_mg* or_mg_new(int L, const or_mat** A, const or_mat** P, const int** bd, const int* nbd,
                 const int* kind, const int* runs, const double* omega, int cycles)
{
    if (L < 1) return NULL;
    or_mg* g = (or_mg*)calloc(1, sizeof(or_mg));
    g->L = L; g->cycles = cycles;
    g->A = (const or_mat**)calloc(L, sizeof(or_mat*));
    g->P = (const or_mat**)calloc(L, sizeof(or_mat*));
    g->bd = (int**)calloc(L, sizeof(int*));
    g->nbd = (int*)calloc(L, sizeof(int));
    g->sm = (or_smoother*)calloc(L, sizeof(or_smoother));
    for (int l = 0; l < L; l++) {
        g->A[l] = A[l];
        if (l < L - 1) g->P[l] = P[l];
        g->nbd[l] = nbd[l];
        g->bd[l] = (int*)malloc(sizeof(int) * (nbd[l] ? nbd[l] : 1));
        if (nbd[l]) memcpy(g->bd[l], bd[l], sizeof(int) * nbd[l]);
        if (l > 0) smoother_init(&g->sm[l], kind[l], runs[l], omega[l], A[l]);
    }
    int n0 = A[0]->rows;
    double* dense = (double*)malloc(sizeof(double) * (size_t)n0 * n0 + 8);
    or_mat_dense(A[0], dense);
    g->coarse_status = lu_factor(&g->coarse, n0, dense);
    free(dense);
    return g;
}

/* Level l smooths with SchwarzSmoother(runs, S). */
void or_mg_set_schwarz(or_mg* g, int l, const or_schwarz* S, int runs)
{
    free(g->sm[l].dinv);
    g->sm[l].dinv = NULL;
    g->sm[l].kind = OR_SMOOTH_SCHWARZ;
    g->sm[l].runs = runs;
    g->sm[l].schwarz = S;
}

void or_mg_free(or_mg* g)
{
    if (!g) return;
    for (int l = 0; l < g->L; l++) { free(g->bd[l]); free(g->sm[l].dinv); }
    lu_free(&g->coarse);
    free(g->A); free(g->P); free(g->bd); free(g->nbd); free(g->sm);
    free(g);
}

/* mgStepV (MGPreconditionerInterface.java:125-198); guess is updated in place. */
static void mg_step_v(const or_mg* g, int level, double* guess, const double* rhs)
{
    int n = g->A[level]->rows;
    if (level == 0) {
        lu_solve(&g->coarse, rhs, guess);      /* DenseMatrix(A0).solve(rhs), line 136 */
        return;
    }
    double* r = vnew(n);
    smooth(&g->sm[level], g->A[level], rhs, guess, r);          /* pre-smooth, lines 153-154 */
    or_mat_mvmul(g->A[level], guess, r);
    for (int i = 0; i < n; i++) r[i] = rhs[i] - r[i];
    int nc = g->A[level - 1]->rows;
    double* rc = vnew(nc);
    mg_restrict(g, level - 1, r, rc);                          /* lines 156-159 */
    double* cc = vnew(nc);                                     /* zero start, line 169 */
    mg_step_v(g, level - 1, cc, rc);
    mg_prolong(g, level - 1, cc, r);                           /* lines 171-172 */
    for (int i = 0; i < n; i++) guess[i] = guess[i] + r[i];    /* line 174 */
    smooth(&g->sm[level], g->A[level], rhs, guess, r);          /* post-smooth, lines 189-190 */
    free(r); free(rc); free(cc);
}

/* mgStepW (MGPreconditionerInterface.java:200-291); guess is updated in
 * place.  Despite its name the reference recurses through mgStepV: on the
 * level it is called on it smooths, applies two coarse-grid corrections in a
 * row (each a restricted defect of the current guess, one mgStepV on level-1
 * from a zero start, prolonged and added), then smooths again. */
static void mg_step_w(const or_mg* g, int level, double* guess, const double* rhs)
{
    int n = g->A[level]->rows;
    if (level == 0) {
        lu_solve(&g->coarse, rhs, guess);      /* lines 203-218 */
        return;
    }
    double* r = vnew(n);
    smooth(&g->sm[level], g->A[level], rhs, guess, r);          /* pre-smooth, lines 226-227 */
    int nc = g->A[level - 1]->rows;
    double* rc = vnew(nc);
    double* cc = vnew(nc);
    for (int pass = 0; pass < 2; pass++) {                     /* lines 229-247 and 249-267 */
        or_mat_mvmul(g->A[level], guess, r);
        for (int i = 0; i < n; i++) r[i] = rhs[i] - r[i];
        mg_restrict(g, level - 1, r, rc);
        memset(cc, 0, sizeof(double) * nc);
        mg_step_v(g, level - 1, cc, rc);
        mg_prolong(g, level - 1, cc, r);
        for (int i = 0; i < n; i++) guess[i] = guess[i] + r[i];
    }
    smooth(&g->sm[level], g->A[level], rhs, guess, r);          /* post-smooth, lines 282-283 */
    free(r); free(rc); free(cc);
}

/* wCycle (MGPreconditionerInterface.java:300-305). */
void or_mg_wcycle(const or_mg* g, const double* x0, const double* rhs, double* out)
{
    int n = g->A[g->L - 1]->rows;
    memcpy(out, x0, sizeof(double) * n);
    mg_step_w(g, g->L - 1, out, rhs);
}

/* vCycle (MGPreconditionerInterface.java:293-298). */
void or_mg_vcycle(const or_mg* g, const double* x0, const double* rhs, double* out)
{
    int n = g->A[g->L - 1]->rows;
    memcpy(out, x0, sizeof(double) * n);
    mg_step_v(g, g->L - 1, out, rhs);
}

/* fullVCycleCorrection (MGPreconditionerInterface.java:307-326).  The
 * prolongation between FMG stages uses the raw matrix P without boundary
 * zeroing (getProlongationMatrix, line 323). */
void or_mg_fmg(const or_mg* g, const double* defect, double* out)
{
    int L = g->L;
    double** rh = (double**)calloc(L, sizeof(double*));
    rh[L - 1] = vdup(g->A[L - 1]->rows, defect);
    for (int l = L - 2; l >= 0; l--) {
        rh[l] = vnew(g->A[l]->rows);
        mg_restrict(g, l, rh[l + 1], rh[l]);
    }
    double* it = vnew(g->A[0]->rows);
    for (int l = 0; l < L - 1; l++) {
        mg_step_v(g, l, it, rh[l]);
        double* nx = vnew(g->A[l + 1]->rows);
        or_mat_mvmul(g->P[l], it, nx);
        free(it);
        it = nx;
    }
    memcpy(out, it, sizeof(double) * g->A[L - 1]->rows);
    free(it);
    for (int l = 0; l < L; l++) free(rh[l]);
    free(rh);
}

/* Preconditioner application mvMul (MGPreconditionerInterface.java:352-379):
 * boundary values copied into a zero start, FMG correction of the defect,
 * then `cycles` V-cycles.  use_fmg = 0 replaces the FMG correction by a zero
 * start (plain V-cycle preconditioner).  wcycle = 1 is mvMulW
 * (MGPreconditionerSpace.java:165-183): the same with wCycle in place of
 * vCycle. */
void or_mg_apply_kind(const or_mg* g, int use_fmg, int cycles, int wcycle, const double* v, double* out)
{
    int L = g->L, n = g->A[L - 1]->rows;
    double* initial = vnew(n);
    for (int i = 0; i < g->nbd[L - 1]; i++) initial[g->bd[L - 1][i]] = v[g->bd[L - 1][i]];
    double* defect = vnew(n);
    or_mat_mvmul(g->A[L - 1], initial, defect);
    for (int i = 0; i < n; i++) defect[i] = v[i] - defect[i];
    double* iter = vnew(n);
    if (use_fmg) or_mg_fmg(g, defect, iter);
    for (int c = 0; c < cycles; c++) {
        if (wcycle) mg_step_w(g, L - 1, iter, defect);
        else mg_step_v(g, L - 1, iter, defect);
    }
    for (int i = 0; i < n; i++) out[i] = initial[i] + iter[i];
    free(initial); free(defect); free(iter);
}

void or_mg_apply_ex(const or_mg* g, int use_fmg, int cycles, const double* v, double* out)
{
    or_mg_apply_kind(g, use_fmg, cycles, 0, v, out);
}

void or_mg_apply(const or_mg* g, const double* v, double* out) { or_mg_apply_ex(g, 1, g->cycles, v, out); }

typedef struct { const or_mg* g; int use_fmg; int cycles; int wcycle; } mg_op_data;
static void op_mg_mv(const or_op* o, const double* x, double* y)
{
    const mg_op_data* d = (const mg_op_data*)o->data;
    or_mg_apply_kind(d->g, d->use_fmg, d->cycles, d->wcycle, x, y);
}
static void op_mg_free_data(or_op* o) { free((void*)o->data); }

/* The MG preconditioner as an operator.  use_fmg=1, cycles=g->cycles is the
 * reference's mvMul; use_fmg=0, cycles=1 is a single V-cycle from zero with
 * the boundary copy. */
or_op* or_op_mg_kind(const or_mg* g, int use_fmg, int cycles, int wcycle)
{
    or_op* o = (or_op*)calloc(1, sizeof(or_op));
    mg_op_data* d = (mg_op_data*)malloc(sizeof(mg_op_data));
    d->g = g; d->use_fmg = use_fmg; d->cycles = cycles; d->wcycle = wcycle;
    o->n = g->A[g->L - 1]->rows; o->mv = op_mg_mv; o->data = d;
    return o;
}
or_op* or_op_mg(const or_mg* g, int use_fmg, int cycles) { return or_op_mg_kind(g, use_fmg, cycles, 0); }
void or_op_mg_free(or_op* o)
{
    if (!o) return;
    op_mg_free_data(o);
    free(o);
}

int or_mg_coarse_status(const or_mg* g) { return g->coarse_status; }
