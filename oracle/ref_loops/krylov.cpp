// The reference's Krylov solver classes (src/solvers/detail/bicgstab.inl,
// pbicgstab.inl, pcg.inl, rbicgstab.inl, merged/merged_bicgstab.inl,
// merged/merged_pbicgstab.inl, with the merged BLAS groups of
// specific/blas_merged_bicgstab.inl) compiled unchanged against the
// stand-ins of solver_base.h, one process.  Their preconditioner is the
// reference's MultiGrid class (ref_mg_apply_d), the multigrid cycle restated
// over its loops (ref_hier_apply_d) or the identity.
#include "solver_base.h"
#include "blas/detail/specific/blas_merged_bicgstab.inl"
#include "solvers/detail/bicgstab.inl"
#include "solvers/detail/pbicgstab.inl"
#include "solvers/detail/pcg.inl"
#include "solvers/detail/rbicgstab.inl"
#include "solvers/detail/merged/merged_bicgstab.inl"
#include "solvers/detail/merged/merged_pbicgstab.inl"

using namespace refloops;

namespace {

// MultiGrid::solve as a preconditioner: one cycle from the x given; without
// a hierarchy the identity (x = b)
struct Precond : XAMG::solver::base_solver_interface {
    void *hier;
    int nv;
    bool mg_class;  // hier is a MultiGrid class object (ref_mg_create), else a ref_hier_create cycle
    Precond(void *h, int nv_, bool m) : hier(h), nv(nv_), mg_class(m) {}
    void solve(vector &x, const vector &b, XAMG::mpi::token & = XAMG::mpi::null_token) override {
        // the solvers clear x by flag only (set_const without force); the
        // cycle's first smoother zeroes a flagged x (blas2.h:264-265)
        if (x.if_zero) std::memset(x.get_aligned_ptr<double>(), 0, sizeof(double) * x.size * nv);
        if (hier && mg_class) {
            ref_mg_apply_d(hier, b.get_aligned_ptr<double>(), x.get_aligned_ptr<double>());
        } else if (hier) {
            ref_hier_apply_d(hier, b.get_aligned_ptr<double>(), x.get_aligned_ptr<double>(), nv);
        } else {
            std::memcpy(x.get_aligned_ptr<double>(), b.get_aligned_ptr<double>(), sizeof(double) * b.size * nv);
        }
        x.if_initialized = true;
        x.if_zero = false;
    }
};

template <template <typename, uint16_t> class S, int NV>
int run_solver(bool with_precond, Precond &pc, XAMG::matrix::matrix &A, vector &X, vector &B, int max_iters,
               double abs_tol, double rel_tol, double *hist, int cap) {
    S<double, NV> s(A, X, B);
    s.param_list.v["max_iters"] = max_iters;
    s.stats.conv_check = true;
    s.stats.abs_tol = abs_tol;
    s.stats.rel_tol = rel_tol;
    s.stats.hist = hist;
    s.stats.cap = cap;
    if (with_precond) s.precond = &pc;
    s.run(s.nvecs);
    return s.stats.iters;
}

struct SolverRun {
    int method; void *hier; bool mg_class; int64_t n; const int *rp, *ci; const double *v, *b; double *x; int nv, max_iters;
    double abs_tol, rel_tol; double *hist; int cap;
    int iters;
    template <int NV> void run() {
        using namespace XAMG::solver;
        XAMG::matrix::matrix A;
        A.n = n; A.rp = rp; A.ci = ci; A.v = v;
        vector X = block(x, n, NV), B = block(b, n, NV);
        Precond pc(hier, NV, mg_class);
        switch (method) {
        case 0: iters = run_solver<BiCGStab, NV>(false, pc, A, X, B, max_iters, abs_tol, rel_tol, hist, cap); break;
        case 1: iters = run_solver<PBiCGStab, NV>(true, pc, A, X, B, max_iters, abs_tol, rel_tol, hist, cap); break;
        case 2: iters = run_solver<PCG, NV>(true, pc, A, X, B, max_iters, abs_tol, rel_tol, hist, cap); break;
        case 3: iters = run_solver<RBiCGStab, NV>(true, pc, A, X, B, max_iters, abs_tol, rel_tol, hist, cap); break;
        case 4: iters = run_solver<MergedBiCGStab, NV>(false, pc, A, X, B, max_iters, abs_tol, rel_tol, hist, cap); break;
        case 5: iters = run_solver<MergedPBiCGStab, NV>(true, pc, A, X, B, max_iters, abs_tol, rel_tol, hist, cap); break;
        default: iters = -1;
        }
    }
};

}  // namespace

extern "C" {
int ref_solver_d(int method, void *hier, int64_t n, const int *rp, const int *ci, const double *v,
                 const double *b, double *x, int nv, int max_iters, double abs_tol, double rel_tol,
                 double *hist, int hist_cap) {
    SolverRun f{method & 15, hier, (method & 16) != 0, n, rp, ci, v, b, x, nv, max_iters, abs_tol, rel_tol, hist,
                hist_cap, 0};
    if (dispatch_nv(nv, f)) return -1;
    return f.iters;
}
}
