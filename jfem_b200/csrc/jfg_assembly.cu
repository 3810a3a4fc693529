// Finite-element assembly of Q_p Lagrange spaces on uniform Cartesian grids,
// on the device: the producer of the systems the solvers take
// (basic/MatrixFESpace.java:29-131 with tensorproduct/TPCellIntegral.java:78-159
// and basic/AcceptsMatrixBoundaryValues.java:25-44).
//
//   numbering   first appearance of a node while the cells are visited with
//               the last coordinate fastest and the local functions x-fastest
//               (the node's key is the smallest (cell, local index) visiting
//               it; the keys are ranked with a radix sort)
//   matrix      one COO triple per (cell, local pair) with the cell integral
//               kappa_c * GG_ab + mass * VV_ab (GG, VV: the 5x5-Gauss element
//               tables, computed once on the host), Dirichlet rows and columns
//               zeroed and a unit diagonal appended; the triples are merged by
//               the COO path of the matrix builder (sort, sum, drop zeros)
//   rhs         per node, the cell integrals sum_q f(c, q) w_q phi_a(q) of the
//               cells containing it, added in ascending cell order
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "jfg_kernels.cuh"

namespace jfg {

Matrix* matrix_from_device_coo(Context* c, int rows, int cols, int64_t nnz, const int* d_ri, const int* d_ci,
                               const double* d_v);

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

constexpr int kMaxP = 3;

struct TPGrid {
    int p, cx, cy, nx, ny, nl;
};

__device__ __forceinline__ bool on_boundary(const TPGrid& g, int gx, int gy)
{
    return gx == 0 || gx == g.nx - 1 || gy == 0 || gy == g.ny - 1;
}

// key of grid node gid: (first cell visiting it) * nl + local index there
__global__ void k_tp_keys(TPGrid g, uint64_t* __restrict__ key, int* __restrict__ gid)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)g.nx * g.ny) return;
    const int gx = (int)(t / g.ny), gy = (int)(t % g.ny);
    const int ix = gx == 0 ? 0 : (gx - 1) / g.p;
    const int iy = gy == 0 ? 0 : (gy - 1) / g.p;
    const int lx = gx - ix * g.p, ly = gy - iy * g.p;
    key[t] = ((uint64_t)ix * g.cy + iy) * g.nl + (uint64_t)(lx + ly * (g.p + 1));
    gid[t] = (int)t;
}

__global__ void k_iota(int64_t n, int* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = (int)t;
}

__global__ void k_tp_number(int64_t n, const int* __restrict__ gid_sorted, int* __restrict__ node_of_grid)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) node_of_grid[gid_sorted[t]] = (int)t;
}

// one triple per (cell, a, b); Dirichlet rows / columns get 0 (dropped by the merge)
__global__ void k_tp_triples(TPGrid g, const int* __restrict__ node_of_grid, const double* __restrict__ GG,
                             const double* __restrict__ VV, double grad_coef, double mass_coef,
                             const double* __restrict__ kappa, int dirichlet, int* __restrict__ ri,
                             int* __restrict__ ci, double* __restrict__ v)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per = (int64_t)g.nl * g.nl;
    if (t >= (int64_t)g.cx * g.cy * per) return;
    const int64_t c = t / per;
    const int ab = (int)(t % per), a = ab / g.nl, b = ab % g.nl;
    const int ix = (int)(c / g.cy), iy = (int)(c % g.cy);
    const int gxa = ix * g.p + a % (g.p + 1), gya = iy * g.p + a / (g.p + 1);
    const int gxb = ix * g.p + b % (g.p + 1), gyb = iy * g.p + b / (g.p + 1);
    const double kc = kappa ? kappa[c] : grad_coef;
    // kappa * GG + mass * VV, each product and the sum rounded on their own
    double val = __dadd_rn(__dmul_rn(kc, GG[ab]), __dmul_rn(mass_coef, VV[ab]));
    if (dirichlet && (on_boundary(g, gxa, gya) || on_boundary(g, gxb, gyb))) val = 0.0;
    ri[t] = node_of_grid[gxa * g.ny + gya];
    ci[t] = node_of_grid[gxb * g.ny + gyb];
    v[t] = val;
}

// unit diagonal of the boundary dofs, and their flags
__global__ void k_tp_boundary(TPGrid g, const int* __restrict__ node_of_grid, int64_t base, int* __restrict__ ri,
                              int* __restrict__ ci, double* __restrict__ v, char* __restrict__ bflag)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)g.nx * g.ny) return;
    const int gx = (int)(t / g.ny), gy = (int)(t % g.ny);
    const int dof = node_of_grid[t];
    const bool bd = on_boundary(g, gx, gy);
    bflag[dof] = bd;
    if (!bd || !ri) return;
    // position of this boundary node among the boundary nodes in grid order
    int64_t k;
    if (gx == 0) k = gy;
    else if (gx == g.nx - 1) k = g.ny + 2 * (int64_t)(g.nx - 2) + gy;
    else k = g.ny + 2 * (int64_t)(gx - 1) + (gy == 0 ? 0 : 1);
    ri[base + k] = dof;
    ci[base + k] = dof;
    v[base + k] = 1.0;
}

// rhs of each dof: cell integrals of its cells in ascending cell order
__global__ void k_tp_rhs(TPGrid g, const int* __restrict__ node_of_grid, const double* __restrict__ f,
                         const double* __restrict__ bw, int dirichlet, double* __restrict__ rhs)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)g.nx * g.ny) return;
    const int gx = (int)(t / g.ny), gy = (int)(t % g.ny);
    const int dof = node_of_grid[t];
    double s = 0.0;
    if (!(dirichlet && on_boundary(g, gx, gy)) && f) {
        const int ix0 = gx == 0 ? 0 : (gx - 1) / g.p, ix1 = min(gx / g.p, g.cx - 1);
        const int iy0 = gy == 0 ? 0 : (gy - 1) / g.p, iy1 = min(gy / g.p, g.cy - 1);
        for (int ix = ix0; ix <= ix1; ix++)
            for (int iy = iy0; iy <= iy1; iy++) {
                const int64_t c = (int64_t)ix * g.cy + iy;
                const int a = (gx - ix * g.p) + (gy - iy * g.p) * (g.p + 1);
                double ci = 0.0;
                for (int q = 0; q < 25; q++) ci = __dadd_rn(ci, __dmul_rn(f[c * 25 + q], bw[q * g.nl + a]));
                s = __dadd_rn(s, ci);
            }
    }
    rhs[dof] = s;
}

// Equidistant Lagrange functions on [0, 1] and their derivatives at t
// (LagrangeBasisFunction1D, tensorproduct/LagrangeBasisFunction1D.java:14-20).
void lagrange(int p, double t, double* val, double* der)
{
    for (int i = 0; i <= p; i++) {
        const double xi = (double)i / p;
        double denom = 1.0, v = 1.0, d = 0.0;
        for (int j = 0; j <= p; j++)
            if (j != i) denom *= xi - (double)j / p;
        for (int j = 0; j <= p; j++)
            if (j != i) v *= t - (double)j / p;
        for (int k = 0; k <= p; k++) {
            if (k == i) continue;
            double term = 1.0;
            for (int j = 0; j <= p; j++)
                if (j != i && j != k) term *= t - (double)j / p;
            d += term;
        }
        val[i] = v / denom;
        der[i] = d / denom;
    }
}

}  // namespace

// Element tables of one cell: GG, VV (nl x nl) and bw (25 x nl, basis value
// times quadrature weight) with the 5-point Gauss rule mapped to [0, 1].
static void tp_tables(int p, double hx, double hy, std::vector<double>& GG, std::vector<double>& VV,
                      std::vector<double>& bw)
{
    const double s70 = std::sqrt(70.0);
    const double gw[5] = {(322.0 - 13 * s70) / 900, (322.0 + 13 * s70) / 900, 128.0 / 225,
                          (322.0 + 13 * s70) / 900, (322.0 - 13 * s70) / 900};
    const double a = std::sqrt(5.0 + 2 * std::sqrt(10.0 / 7)) / 3, b = std::sqrt(5.0 - 2 * std::sqrt(10.0 / 7)) / 3;
    const double gp[5] = {-a, -b, 0.0, b, a};
    double qt[5], qw[5], V[kMaxP + 1][5], D[kMaxP + 1][5];
    for (int q = 0; q < 5; q++) {
        qt[q] = 0.5 * (gp[q] + 1.0);
        qw[q] = 0.5 * gw[q];
        double v[kMaxP + 1], d[kMaxP + 1];
        lagrange(p, qt[q], v, d);
        for (int i = 0; i <= p; i++) {
            V[i][q] = v[i];
            D[i][q] = d[i];
        }
    }
    const int nl = (p + 1) * (p + 1);
    GG.assign((size_t)nl * nl, 0.0);
    VV.assign((size_t)nl * nl, 0.0);
    bw.assign((size_t)25 * nl, 0.0);
    for (int Q = 0; Q < 25; Q++) {
        const int qi = Q / 5, qj = Q % 5;                     // x index slowest
        const double w = qw[qi] * qw[qj] * hx * hy;
        for (int u = 0; u < nl; u++) {
            const int ux = u % (p + 1), uy = u / (p + 1);
            const double val_u = V[ux][qi] * V[uy][qj];
            const double gx_u = D[ux][qi] / hx * V[uy][qj];
            const double gy_u = V[ux][qi] * D[uy][qj] / hy;
            bw[(size_t)Q * nl + u] = val_u * w;
            for (int v = 0; v < nl; v++) {
                const int vx = v % (p + 1), vy = v / (p + 1);
                const double val_v = V[vx][qi] * V[vy][qj];
                const double gx_v = D[vx][qi] / hx * V[vy][qj];
                const double gy_v = V[vx][qi] * D[vy][qj] / hy;
                GG[(size_t)u * nl + v] += (gx_u * gx_v + gy_u * gy_v) * w;
                VV[(size_t)u * nl + v] += (val_u * val_v) * w;
            }
        }
    }
}

Matrix* assemble_tp(Context* c, const jfg_tp_desc& d, const double* h_kappa, const double* h_f, double* h_rhs,
                    int* h_node_of_grid, int* h_boundary)
{
    JFG_CHECK(d.p >= 1 && d.p <= kMaxP, JFG_ERR_UNSUPPORTED, "polynomial degree must be 1..3");
    JFG_CHECK(d.cx >= 1 && d.cy >= 1 && d.x1 > d.x0 && d.y1 > d.y0, JFG_ERR_BAD_ARG, "empty grid");
    cudaStream_t s = c->stream;
    TPGrid g{d.p, d.cx, d.cy, d.p * d.cx + 1, d.p * d.cy + 1, (d.p + 1) * (d.p + 1)};
    const int64_t nn = (int64_t)g.nx * g.ny;
    JFG_CHECK(nn < INT32_MAX, JFG_ERR_UNSUPPORTED, "more than 2^31 nodes");
    const int64_t ncell = (int64_t)g.cx * g.cy;
    const int64_t ntrip = ncell * g.nl * g.nl;
    const int64_t nbd = 2 * (int64_t)(g.nx + g.ny) - 4;
    std::vector<double> GG, VV, bw;
    tp_tables(d.p, (d.x1 - d.x0) / d.cx, (d.y1 - d.y0) / d.cy, GG, VV, bw);

    DevBuf<double> dGG, dVV, dbw, dkappa, df, drhs;
    dGG.alloc(GG.size());
    dVV.alloc(VV.size());
    dbw.alloc(bw.size());
    JFG_CUDA(cudaMemcpyAsync(dGG.p, GG.data(), sizeof(double) * GG.size(), cudaMemcpyHostToDevice, s));
    JFG_CUDA(cudaMemcpyAsync(dVV.p, VV.data(), sizeof(double) * VV.size(), cudaMemcpyHostToDevice, s));
    JFG_CUDA(cudaMemcpyAsync(dbw.p, bw.data(), sizeof(double) * bw.size(), cudaMemcpyHostToDevice, s));
    if (h_kappa) {
        dkappa.alloc((size_t)ncell);
        JFG_CUDA(cudaMemcpyAsync(dkappa.p, h_kappa, sizeof(double) * ncell, cudaMemcpyHostToDevice, s));
    }
    if (h_f) {
        df.alloc((size_t)ncell * 25);
        JFG_CUDA(cudaMemcpyAsync(df.p, h_f, sizeof(double) * ncell * 25, cudaMemcpyHostToDevice, s));
    }

    // numbering
    DevBuf<uint64_t> key, key2;
    DevBuf<int> gid, gid2, nog;
    key.alloc((size_t)nn);
    key2.alloc((size_t)nn);
    gid.alloc((size_t)nn);
    gid2.alloc((size_t)nn);
    nog.alloc((size_t)nn);
    k_tp_keys<<<nblk(nn), 256, 0, s>>>(g, key.p, gid.p);
    JFG_CUDA(cudaGetLastError());
    int bits = 1;
    while (bits < 64 && (1ULL << bits) < (uint64_t)ncell * g.nl) bits++;
    size_t tb = 0;
    JFG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, key2.p, gid.p, gid2.p, nn, 0, bits, s));
    DevBuf<char> tmp;
    tmp.alloc(tb + 16);
    JFG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, key2.p, gid.p, gid2.p, nn, 0, bits, s));
    k_tp_number<<<nblk(nn), 256, 0, s>>>(nn, gid2.p, nog.p);
    JFG_CUDA(cudaGetLastError());

    // triples: cell pairs, then the boundary unit diagonal
    const int64_t total = ntrip + (d.dirichlet ? nbd : 0);
    DevBuf<int> ri, ci;
    DevBuf<double> v;
    DevBuf<char> bflag;
    ri.alloc((size_t)total);
    ci.alloc((size_t)total);
    v.alloc((size_t)total);
    bflag.alloc((size_t)nn);
    k_tp_triples<<<nblk(ntrip), 256, 0, s>>>(g, nog.p, dGG.p, dVV.p, d.grad_coef, d.mass_coef,
                                             h_kappa ? dkappa.p : nullptr, d.dirichlet, ri.p, ci.p, v.p);
    JFG_CUDA(cudaGetLastError());
    k_tp_boundary<<<nblk(nn), 256, 0, s>>>(g, nog.p, ntrip, d.dirichlet ? ri.p : nullptr, ci.p, v.p, bflag.p);
    JFG_CUDA(cudaGetLastError());

    // rhs
    drhs.alloc((size_t)nn);
    k_tp_rhs<<<nblk(nn), 256, 0, s>>>(g, nog.p, h_f ? df.p : nullptr, dbw.p, d.dirichlet, drhs.p);
    JFG_CUDA(cudaGetLastError());
    if (h_rhs) JFG_CUDA(cudaMemcpyAsync(h_rhs, drhs.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
    if (h_node_of_grid)
        JFG_CUDA(cudaMemcpyAsync(h_node_of_grid, nog.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, s));
    if (h_boundary) {
        // ascending boundary dofs: select the flagged dof indices
        DevBuf<int> iota, sel;
        DevBuf<int64_t> nsel;
        iota.alloc((size_t)nn);
        sel.alloc((size_t)nbd);
        nsel.alloc(1);
        k_iota<<<nblk(nn), 256, 0, s>>>(nn, iota.p);
        JFG_CUDA(cudaGetLastError());
        size_t t1 = 0;
        JFG_CUDA(cub::DeviceSelect::Flagged(nullptr, t1, iota.p, bflag.p, sel.p, nsel.p, nn, s));
        DevBuf<char> tmp2;
        tmp2.alloc(t1 + 16);
        JFG_CUDA(cub::DeviceSelect::Flagged(tmp2.p, t1, iota.p, bflag.p, sel.p, nsel.p, nn, s));
        JFG_CUDA(cudaMemcpyAsync(h_boundary, sel.p, sizeof(int) * nbd, cudaMemcpyDeviceToHost, s));
        JFG_CUDA(cudaStreamSynchronize(s));
    }
    JFG_CUDA(cudaStreamSynchronize(s));
    return matrix_from_device_coo(c, (int)nn, (int)nn, total, ri.p, ci.p, v.p);
}

// ---------------------------------------------------------------------------
// Taylor-Hood Q2/Q1 Stokes system on the unit square (cx x cy cells): unknowns
// [u0 (Q2 grid, x-major), u1, p (Q1 grid, x-major)]; blocks nu * GRAD_GRAD on
// each velocity component, -B_c (pressure rows) and -B_c^T (velocity rows),
// B_c = int q d(phi)/dx_c; Dirichlet velocity on the whole boundary with u0 = 1
// on the top lid when lid != 0, and the first pressure unknown fixed when
// pin != 0 (AcceptsMatrixBoundaryValues: fixed rows / columns zeroed, a unit
// diagonal, the lifted boundary values moved to the rhs).
// ---------------------------------------------------------------------------
namespace {

struct THGrid {
    int cx, cy, vnx, vny, pnx, pny, nv1, nv, n;
    int lid, pin;
};

__device__ __forceinline__ bool th_fixed(const THGrid& g, int dof)
{
    if (dof >= g.nv) return g.pin && dof == g.nv;
    const int v = dof % g.nv1;
    const int gx = v / g.vny, gy = v % g.vny;
    return gx == 0 || gx == g.vnx - 1 || gy == 0 || gy == g.vny - 1;
}

// boundary value of a fixed dof (u0 = 1 on the lid y = 1, else 0)
__device__ __forceinline__ double th_g(const THGrid& g, int dof)
{
    if (!g.lid || dof >= g.nv1) return 0.0;
    return (dof % g.vny) == g.vny - 1 ? 1.0 : 0.0;
}

// 306 triples per cell: per component 81 (K), 36 (pressure rows), 36 (velocity rows)
__global__ void k_th_triples(THGrid g, const double* __restrict__ K, const double* __restrict__ B, double nu,
                             int* __restrict__ ri, int* __restrict__ ci, double* __restrict__ v,
                             int* __restrict__ lrow, double* __restrict__ lval)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ncell = (int64_t)g.cx * g.cy;
    if (t >= ncell * 306) return;
    const int64_t cell = t / 306;
    int e = (int)(t % 306);
    const int ix = (int)(cell / g.cy), iy = (int)(cell % g.cy);
    const int comp = e / 153;
    e %= 153;
    int row, col;
    double val;
    auto vnode = [&](int a) { return (2 * ix + a % 3) * g.vny + (2 * iy + a / 3) + comp * g.nv1; };
    auto pnode = [&](int q) { return (ix + q % 2) * g.pny + (iy + q / 2) + g.nv; };
    if (e < 81) {
        const int a = e / 9, b = e % 9;
        row = vnode(a);
        col = vnode(b);
        val = __dmul_rn(nu, K[e]);
    } else if (e < 117) {
        const int q = (e - 81) / 9, j = (e - 81) % 9;
        row = pnode(q);
        col = vnode(j);
        val = -B[comp * 36 + q * 9 + j];
    } else {
        const int j = (e - 117) / 4, q = (e - 117) % 4;      // B^T: row = velocity j, col = pressure q
        row = vnode(j);
        col = pnode(q);
        val = -B[comp * 36 + q * 9 + j];
    }
    const bool fr = th_fixed(g, row), fc = th_fixed(g, col);
    lrow[t] = row;
    lval[t] = (fc && !fr) ? -(val * th_g(g, col)) : 0.0;     // lifted boundary value
    ri[t] = row;
    ci[t] = col;
    v[t] = (fr || fc) ? 0.0 : val;
}

__global__ void k_th_fixed(THGrid g, int64_t base, int* __restrict__ ri, int* __restrict__ ci, double* __restrict__ v,
                           char* __restrict__ flag)
{
    const int dof = blockIdx.x * blockDim.x + threadIdx.x;
    if (dof >= g.n) return;
    const bool f = th_fixed(g, dof);
    flag[dof] = f;
    ri[base + dof] = dof;
    ci[base + dof] = dof;
    v[base + dof] = f ? 1.0 : 0.0;       // unit diagonal of the fixed rows (zeros are dropped by the merge)
}

// rhs: velocity rows gather their cells' force integrals in ascending cell
// order, then the lifted boundary values (summed per row in triple order);
// fixed rows take their boundary value
__global__ void k_th_rhs(THGrid g, const double* __restrict__ f, const double* __restrict__ rw, double* __restrict__ rhs)
{
    const int dof = blockIdx.x * blockDim.x + threadIdx.x;
    if (dof >= g.n) return;
    double s = 0.0;
    if (f && dof < g.nv) {
        const int comp = dof / g.nv1, v = dof % g.nv1;
        const int gx = v / g.vny, gy = v % g.vny;
        const int ix0 = gx == 0 ? 0 : (gx - 1) / 2, ix1 = min(gx / 2, g.cx - 1);
        const int iy0 = gy == 0 ? 0 : (gy - 1) / 2, iy1 = min(gy / 2, g.cy - 1);
        for (int ix = ix0; ix <= ix1; ix++)
            for (int iy = iy0; iy <= iy1; iy++) {
                const int64_t c = (int64_t)ix * g.cy + iy;
                const int a = (gx - 2 * ix) + (gy - 2 * iy) * 3;
                double ci = 0.0;
                for (int q = 0; q < 25; q++)
                    ci = __dadd_rn(ci, __dmul_rn(f[((int64_t)comp * g.cx * g.cy + c) * 25 + q], rw[a * 25 + q]));
                s = __dadd_rn(s, ci);
            }
    }
    rhs[dof] = s;
}

__global__ void k_th_lift(const int* __restrict__ urow, const double* __restrict__ usum,
                          const int64_t* __restrict__ nruns, double* __restrict__ rhs)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nruns) return;
    rhs[urow[t]] = __dadd_rn(rhs[urow[t]], usum[t]);
}

__global__ void k_th_set_fixed(THGrid g, double* __restrict__ rhs)
{
    const int dof = blockIdx.x * blockDim.x + threadIdx.x;
    if (dof < g.n && th_fixed(g, dof)) rhs[dof] = th_g(g, dof);
}

}  // namespace

// Element tables of the Taylor-Hood pair: K (9 x 9), B (2 x 4 x 9: q x j) and
// the Q2 rhs weights rw (9 x 25), 5x5 Gauss.
static void th_tables(double hx, double hy, std::vector<double>& K, std::vector<double>& B, std::vector<double>& rw)
{
    const double s70 = std::sqrt(70.0);
    const double gw[5] = {(322.0 - 13 * s70) / 900, (322.0 + 13 * s70) / 900, 128.0 / 225,
                          (322.0 + 13 * s70) / 900, (322.0 - 13 * s70) / 900};
    const double a = std::sqrt(5.0 + 2 * std::sqrt(10.0 / 7)) / 3, b = std::sqrt(5.0 - 2 * std::sqrt(10.0 / 7)) / 3;
    const double gp[5] = {-a, -b, 0.0, b, a};
    double V2[3][5], D2[3][5], V1[2][5], qw[5];
    for (int q = 0; q < 5; q++) {
        const double t = 0.5 * (gp[q] + 1.0);
        qw[q] = 0.5 * gw[q];
        double v[4], d[4];
        lagrange(2, t, v, d);
        for (int i = 0; i < 3; i++) {
            V2[i][q] = v[i];
            D2[i][q] = d[i];
        }
        lagrange(1, t, v, d);
        for (int i = 0; i < 2; i++) V1[i][q] = v[i];
    }
    K.assign(81, 0.0);
    B.assign(72, 0.0);
    rw.assign(9 * 25, 0.0);
    for (int Q = 0; Q < 25; Q++) {
        const int qi = Q / 5, qj = Q % 5;
        const double w = qw[qi] * qw[qj] * hx * hy;
        double val2[9], gx[9], gy[9], val1[4];
        for (int u = 0; u < 9; u++) {
            const int ux = u % 3, uy = u / 3;
            val2[u] = V2[ux][qi] * V2[uy][qj];
            gx[u] = D2[ux][qi] / hx * V2[uy][qj];
            gy[u] = V2[ux][qi] * D2[uy][qj] / hy;
            rw[u * 25 + Q] = val2[u] * w;
        }
        for (int q = 0; q < 4; q++) val1[q] = V1[q % 2][qi] * V1[q / 2][qj];
        for (int i = 0; i < 9; i++)
            for (int j = 0; j < 9; j++) K[i * 9 + j] += gx[i] * gx[j] * w + gy[i] * gy[j] * w;
        for (int q = 0; q < 4; q++)
            for (int j = 0; j < 9; j++) {
                B[q * 9 + j] += val1[q] * gx[j] * w;
                B[36 + q * 9 + j] += val1[q] * gy[j] * w;
            }
    }
}

Matrix* assemble_th(Context* c, int cx, int cy, double nu, const double* h_force_qp, int lid, int pin,
                    double* h_rhs, int* h_boundary)
{
    JFG_CHECK(cx >= 1 && cy >= 1, JFG_ERR_BAD_ARG, "empty grid");
    cudaStream_t s = c->stream;
    THGrid g{};
    g.cx = cx;
    g.cy = cy;
    g.vnx = 2 * cx + 1;
    g.vny = 2 * cy + 1;
    g.pnx = cx + 1;
    g.pny = cy + 1;
    g.nv1 = g.vnx * g.vny;
    g.nv = 2 * g.nv1;
    g.n = g.nv + g.pnx * g.pny;
    g.lid = lid;
    g.pin = pin;
    const int64_t ncell = (int64_t)cx * cy;
    const int64_t ntrip = ncell * 306;
    std::vector<double> K, B, rw;
    th_tables(1.0 / cx, 1.0 / cy, K, B, rw);
    DevBuf<double> dK, dB, drw, df, drhs;
    dK.alloc(K.size());
    dB.alloc(B.size());
    drw.alloc(rw.size());
    JFG_CUDA(cudaMemcpyAsync(dK.p, K.data(), sizeof(double) * K.size(), cudaMemcpyHostToDevice, s));
    JFG_CUDA(cudaMemcpyAsync(dB.p, B.data(), sizeof(double) * B.size(), cudaMemcpyHostToDevice, s));
    JFG_CUDA(cudaMemcpyAsync(drw.p, rw.data(), sizeof(double) * rw.size(), cudaMemcpyHostToDevice, s));
    if (h_force_qp) {
        df.alloc((size_t)2 * ncell * 25);
        JFG_CUDA(cudaMemcpyAsync(df.p, h_force_qp, sizeof(double) * 2 * ncell * 25, cudaMemcpyHostToDevice, s));
    }
    const int64_t total = ntrip + g.n;
    DevBuf<int> ri, ci, lrow, lrow2, urow;
    DevBuf<double> v, lval, lval2, usum;
    DevBuf<char> flag;
    DevBuf<int64_t> nrun;
    ri.alloc((size_t)total);
    ci.alloc((size_t)total);
    v.alloc((size_t)total);
    lrow.alloc((size_t)ntrip);
    lval.alloc((size_t)ntrip);
    flag.alloc((size_t)g.n);
    k_th_triples<<<nblk(ntrip), 256, 0, s>>>(g, dK.p, dB.p, nu, ri.p, ci.p, v.p, lrow.p, lval.p);
    JFG_CUDA(cudaGetLastError());
    k_th_fixed<<<nblk(g.n), 256, 0, s>>>(g, ntrip, ri.p, ci.p, v.p, flag.p);
    JFG_CUDA(cudaGetLastError());
    // rhs: force integrals, then the lifted boundary values per row (stable
    // sort by row keeps the triple order, the run sums are deterministic)
    drhs.alloc((size_t)g.n);
    k_th_rhs<<<nblk(g.n), 256, 0, s>>>(g, h_force_qp ? df.p : nullptr, drw.p, drhs.p);
    JFG_CUDA(cudaGetLastError());
    if (lid) {
        lrow2.alloc((size_t)ntrip);
        lval2.alloc((size_t)ntrip);
        urow.alloc((size_t)ntrip);
        usum.alloc((size_t)ntrip);
        nrun.alloc(1);
        int bits = 1;
        while (bits < 31 && (1 << bits) < g.n) bits++;
        size_t t1 = 0, t2 = 0;
        JFG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, lrow.p, lrow2.p, lval.p, lval2.p, ntrip, 0, bits, s));
        JFG_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, t2, lrow2.p, urow.p, lval2.p, usum.p, nrun.p, cub::Sum(),
                                                ntrip, s));
        DevBuf<char> tmp;
        tmp.alloc(std::max(t1, t2) + 16);
        JFG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, t1, lrow.p, lrow2.p, lval.p, lval2.p, ntrip, 0, bits, s));
        JFG_CUDA(cub::DeviceReduce::ReduceByKey(tmp.p, t2, lrow2.p, urow.p, lval2.p, usum.p, nrun.p, cub::Sum(),
                                                ntrip, s));
        k_th_lift<<<nblk(ntrip), 256, 0, s>>>(urow.p, usum.p, nrun.p, drhs.p);
        JFG_CUDA(cudaGetLastError());
        JFG_CUDA(cudaStreamSynchronize(s));
    }
    k_th_set_fixed<<<nblk(g.n), 256, 0, s>>>(g, drhs.p);
    JFG_CUDA(cudaGetLastError());
    if (h_rhs) JFG_CUDA(cudaMemcpyAsync(h_rhs, drhs.p, sizeof(double) * g.n, cudaMemcpyDeviceToHost, s));
    if (h_boundary) {
        // ascending velocity boundary dofs (the pinned pressure unknown is not listed)
        std::vector<int> bd;
        for (int comp = 0; comp < 2; comp++)
            for (int gx = 0; gx < g.vnx; gx++)
                for (int gy = 0; gy < g.vny; gy++)
                    if (gx == 0 || gx == g.vnx - 1 || gy == 0 || gy == g.vny - 1)
                        bd.push_back(comp * g.nv1 + gx * g.vny + gy);
        std::copy(bd.begin(), bd.end(), h_boundary);
    }
    JFG_CUDA(cudaStreamSynchronize(s));
    return matrix_from_device_coo(c, g.n, g.n, total, ri.p, ci.p, v.p);
}

}  // namespace jfg
