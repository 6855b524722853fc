// The reference's Chebyshev smoother (src/solvers/detail/chebyshev.inl),
// the solver class compiled unchanged against stand-ins for its solver base
// class, parameter list and statistics (defined below, this file's own): its
// polynomial coefficients (Chebyshev_polynomial_coeffs) and the application
// of the polynomial in D^{-1/2} A D^{-1/2} (Chebyshev::solve).
#include <cstring>
#include <string>

#include "include_ref.h"
#include "ref_loops.h"

namespace XAMG {
namespace params {
// the two keys the smoother reads
struct param_list {
    int64_t order = 2;
    float64_t fraction = 0.3;
    int64_t get_int(const std::string &) const { return order; }
    float64_t get_float(const std::string &) const { return fraction; }
};
}  // namespace params
namespace mpi {
struct token {};
static token null_token;
}  // namespace mpi
namespace blas {
template <typename F> struct ConstVectorsCache {
    static const vector::vector &get_ones_vec(int nv) {
        static std::map<int, vector::vector> cache;
        vector::vector &v = cache[nv];
        if (!v.if_allocated) {
            F *p = v.alloc_and_get_aligned_ptr<F>(1, (uint16_t)nv);
            for (int k = 0; k < nv; ++k) p[k] = F(1);
            v.if_initialized = true;
            v.if_zero = false;
        }
        return v;
    }
};
}  // namespace blas
namespace blas2 {
// y = A x for the one-process operator (blas2.h:305-326 reduces to csr_Ax_y)
template <typename F, uint16_t NV>
void Ax_y(matrix::matrix &A, const vector::vector &x, vector::vector &y, uint16_t) {
    ref_csr_ax_y_d(A.n, A.rp, A.ci, A.v, x.get_aligned_ptr<double>(), y.get_aligned_ptr<double>(), NV);
    y.if_initialized = true;
    y.if_zero = false;
}
}  // namespace blas2
namespace solver {
struct base_solver_interface {
    virtual ~base_solver_interface() {}
};
template <typename F, uint16_t NV> struct base_solver;
// statistics of a smoother: convergence checks off (the preconditioner role)
template <typename F, uint16_t NV> struct stats_stub {
    base_solver<F, NV> *s;
    void init(vector::vector &) {}
    bool is_converged_initial(vector::vector &r) {
        s->get_residual(r);  // stats.h:208-212: the residual is formed, then no check
        return false;
    }
    bool is_converged() { return false; }
};
template <typename F, uint16_t NV> struct base_solver : base_solver_interface {
    std::string solver_role;
    params::param_list param_list;
    matrix::matrix &A;
    vector::vector *x = nullptr;
    const vector::vector *b = nullptr;
    std::vector<vector::vector> buffer;
    base_solver_interface *precond = nullptr;
    int allreduce_buffer = 0;
    uint16_t buffer_nvecs = 0, allreduce_buffer_size = 0;
    stats_stub<F, NV> stats{this};
    base_solver(matrix::matrix &a, vector::vector &x_, const vector::vector &b_) : A(a), x(&x_), b(&b_) {}
    explicit base_solver(matrix::matrix &a) : A(a) {}
    void init_base(const params::param_list &l) { param_list = l; }
    void set_buffers_zero() {
        for (auto &v : buffer) blas::set_const<F, NV>(v, 0.0, true);
    }
    // solver.h:183-190: r = b - A x
    void get_residual(vector::vector &r) {
        blas2::Ax_y<F, NV>(A, *x, r, NV);
        blas::axpby<F, NV>(1.0, *b, -1.0, r);
    }
    virtual void init(const params::param_list &, const std::string &) {}
    virtual void solve(const vector::vector &conv, mpi::token &tok) = 0;
    virtual void matrix_info() = 0;
};
}  // namespace solver
}  // namespace XAMG

// the reference's class-body macro (solver.h:256-281), restated: the names
// the solver classes take from their base, constructors, the overrides
#define DECLARE_INHERITED_FROM_BASESOLVER(CLASSNAME)                                               \
    using base = base_solver<F, NV>;                                                               \
    using base_iface = base_solver_interface;                                                      \
    using base::stats;                                                                             \
    using base::param_list;                                                                        \
    using base::buffer;                                                                            \
    using base::A;                                                                                 \
    using base::x;                                                                                 \
    using base::b;                                                                                 \
    using base::precond;                                                                           \
    using base::allreduce_buffer;                                                                  \
    CLASSNAME(matrix::matrix &_A, vector::vector &_x, const vector::vector &_b) : base(_A, _x, _b) { \
        base::buffer_nvecs = nvecs;                                                                \
        base::allreduce_buffer_size = comm_size;                                                   \
    }                                                                                              \
    virtual void solve(const vector::vector &conv, XAMG::mpi::token &tok = XAMG::mpi::null_token)  \
        override;                                                                                  \
    virtual void matrix_info() override;

#include "solvers/detail/chebyshev.inl"

using namespace refloops;

namespace {

struct ChebRun {
    int64_t n; const int *rp, *ci; const double *v, *b; double *x; int nv, order;
    double fraction, min_eig, max_eig;
    template <int NV> void run() {
        XAMG::matrix::matrix A;
        A.n = n; A.rp = rp; A.ci = ci; A.v = v;
        A.min_eig = min_eig; A.max_eig = max_eig;
        // D^{-1/2}: sqrt(1.0 / a_ii) (csr_matrix.h:377-384)
        std::vector<double> isd(n, 0.0);
        for (int64_t i = 0; i < n; ++i)
            for (int j = rp[i]; j < rp[i + 1]; ++j)
                if (ci[j] == i) isd[i] = std::sqrt(1.0 / v[j]);
        A.isd = block(isd.data(), n, 1);
        vector X = block(x, n, NV), B = block(b, n, NV);
        XAMG::solver::Chebyshev<double, NV> s(A, X, B);
        s.param_list.order = order;
        s.param_list.fraction = fraction;
        s.buffer.resize(3);
        for (auto &bv : s.buffer) bv.template alloc<double>(n, NV);
        s.set_buffers_zero();
        vector conv;
        s.solve(conv);
    }
};

}  // namespace

extern "C" {
int ref_chebyshev_d(int64_t n, const int *rp, const int *ci, const double *v, const double *b, double *x, int nv,
                    int order, double fraction, double min_eig, double max_eig) {
    if (order < 1 || order > 4) return -1;
    ChebRun f{n, rp, ci, v, b, x, nv, order, fraction, min_eig, max_eig};
    return dispatch_nv(nv, f);
}
}
