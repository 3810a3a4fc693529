// Krylov solvers on the device: shared declarations.
#pragma once
#include <functional>
#include <map>
#include <tuple>

#include "jfg_mg.cuh"

namespace jfg {

template <typename T>
struct Precond {
    int kind = JFG_PREC_NONE;
    MGImpl<T>* mg = nullptr;
    Matrix* M = nullptr;
    const T* dinv = nullptr;
    int n = 0;
    // FP64 iteration with an FP32 multigrid preconditioner: r is rounded to
    // FP32 into r32, the FP32 hierarchy computes z32, z is z32 widened.
    MGImpl<float>* mg32 = nullptr;
    float* r32 = nullptr;
    float* z32 = nullptr;
    // an external preconditioner (the multigrid + learned smoother of jfg_cnn.cu)
    void (*hook)(void* self, const T* r, T* z, const Scratch& sc, const int* done, cudaStream_t st) = nullptr;
    void* hook_self = nullptr;
    uint64_t hook_uid = 0;
    void apply(const T* r, T* z, const Scratch& sc, const int* done, cudaStream_t st) const;
};

// Runs `iter()` (which enqueues one iteration) until ctl->done is set,
// either as a CUDA graph with a conditional WHILE node, as replayed graphs of
// `chunk` iterations with a convergence poll in between, or as plain launches.
struct GraphCache {
    std::map<std::vector<uintptr_t>, cudaGraphExec_t> execs;
    std::map<std::vector<uintptr_t>, int> nodes;     // kernel nodes per body
    ~GraphCache();
};

struct SolverWork {
    Context* c = nullptr;
    DevBuf<Ctl> ctl;                // [0] outer / plain solve, [1] inner solve
    DevBuf<double> hist;
    DevBuf<double> partials;
    DevBuf<unsigned> counter;
    Scratch sc;
    DevBuf<double> v64[12];         // FP64 work vectors
    DevBuf<float> v32[8];           // FP32 work vectors
    DevBuf<double> dinv64;
    DevBuf<float> dinv32;
    // GMRES
    DevBuf<double> V, H, gam, cs, sn, fac, alpha, mdot_part;
    // GMRES2: the v and A v bases and a few device scalars
    DevBuf<double> V2, AV2, g2;
    int g2_cap = 0;
    // FGMRES: preconditioned directions and the second Gram-Schmidt pass
    DevBuf<double> Z, fac2, facsum;
    int gm_m = 0;
    GraphCache graphs;
    void ensure(int n, int max_blocks, int hist_cap);
};

int run_loop(SolverWork& w, const int* flag, const std::vector<uintptr_t>& key, const std::function<void()>& iter,
              int use_graph, int chunk);

template <typename T>
int run_cg(SolverWork& w, int ci, Matrix* A, const Precond<T>& M, const T* b, T* x, T* r, T* p, T* Ap, T* z,
            bool xzero, int use_graph, int chunk);
// unpreconditioned FP64 CG of a small system in one cluster launch (jfg_cg_small.cu)
bool cg_small_fits(const Matrix* A);
void run_cg_small(SolverWork& w, Matrix* A, const double* b, double* x);
template <typename T>
int run_bicgstab(SolverWork& w, int ci, Matrix* A, const Precond<T>& M, const T* b, T* x, T* const* v,
                  int use_graph, int chunk);
// A linear operator of the GMRES loop: a matrix, or (apply set) a
// composition of device products that writes A x into tmp -- the implicit
// Schur complement of ImplicitSchurSolver.  A gives the sizes and the
// product grid of the composition.
struct Operator {
    Matrix* A = nullptr;
    int n = 0;
    uint64_t uid = 0;
    void (*apply)(void* self, const double* x, double* y, const Scratch& sc, const int* done, cudaStream_t st) = nullptr;
    void* self = nullptr;
    double* tmp = nullptr;
};
inline Operator op_of(Matrix* A)
{
    Operator o;
    o.A = A;
    o.n = A->rows;
    o.uid = A->uid;
    return o;
}

template <class Epi>
struct VEpi {   // an SpMV epilogue applied to row sums already in s
    const double* s;
    Epi epi;
    template <int K> __device__ void operator()(int i, double (&acc)[K]) const { epi(i, s[i], acc); }
};

// y-epilogue product with the operator: one SpMV for a matrix; the
// composition into tmp, then the epilogue as a vector pass, for the rest.
template <int NR, class Epi, class Fin = NoFin>
void op_launch(cudaStream_t st, const Operator& op, const double* x, Epi epi, const Scratch& sc, const int* done,
               Fin fin = Fin())
{
    if (!op.apply) {
        spmv_launch<double, double, NR, Epi, Fin>(st, op.A, op.A->val.p, x, epi, sc, done, fin);
        return;
    }
    op.apply(op.self, x, op.tmp, sc, done, st);
    vec_launch<NR>(st, op.n, VEpi<Epi>{op.tmp, epi}, sc, done, fin);
}

int run_gmres(SolverWork& w, Matrix* A, const Precond<double>& M, const double* b, double* x, int IBR,
              int max_restarts, int use_graph, int chunk);
int run_gmres(SolverWork& w, const Operator& op, const Precond<double>& M, const double* b, double* x, int IBR,
              int max_restarts, int use_graph, int chunk);
int run_mixed_cg(SolverWork& w, Matrix* A, const Precond<float>& M, const double* b, double* x, double tol,
                 int maxit, double inner_rtol, int use_graph, int chunk, int* inner_iters, double* hist, int hist_cap);
int run_fgmres(SolverWork& w, Matrix* A, const Precond<double>& M, const double* b, double* x, int m_restart,
               int max_restarts, int use_graph, int chunk);
int run_gmres2(SolverWork& w, Matrix* A, const Precond<double>& M, const double* b, double* x, double tol,
               int maxit, int max_restarts, int basis_cap, int* iters, int* restarts, double* final_norm,
               double* hist, int hist_cap);
uint64_t next_uid();
// Fills P with the multigrid + learned-smoother hook of a jfg_mgcnn handle
// (defined with the network kernels); returns its largest grid.
int mgcnn_precond(void* handle, Precond<double>& P, int n);
// The same for a jfg_schwarz handle (AbstractSchwarz.mvMul); defined with the Schwarz kernels.
int schwarz_precond(void* handle, Precond<double>& P, int n);
// The same for a jfg_blockdiag handle (velocity multigrid + diagonal pressure block).
int blockdiag_precond(void* handle, Precond<double>& P, int n);

}  // namespace jfg
