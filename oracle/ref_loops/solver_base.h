// Stand-ins for the reference's solver framework (src/solvers/solver.h,
// stats.h, convergence.h, the parameter list, the allreduce buffer and the
// constant-vector cache), so that its solver classes (bicgstab.inl,
// pbicgstab.inl, pcg.inl, rbicgstab.inl, merged/*.inl, chebyshev.inl)
// compile unchanged for one process.  The classes' step order and vector
// operations are the reference's; the convergence bookkeeping below restates
// convergence.h:200-245 (per column: res frozen once converged, converged
// when sqrt(res) <= max(abs_tol, rel_tol * sqrt(res0)), the column's iconv
// entry then 0) and records every checked residual.
#pragma once
#include <cstring>
#include <map>
#include <string>

#include "include_ref.h"
#include "ref_loops.h"

namespace XAMG {
namespace params {
struct param_list {
    std::map<std::string, double> v;
    int64_t get_int(const std::string &k) const { return (int64_t)v.at(k); }
    float64_t get_float(const std::string &k) const { return v.at(k); }
    bool get_bool(const std::string &k) const { return v.count(k) && v.at(k) != 0; }
};
// the solver tree's parameter sets: only looked up by setup code that the
// checks never run
struct global_param_list {
    param_list l;
    bool find(const std::string &) const { return false; }
    const param_list &get(const std::string &, int = -1) const { return l; }
    template <typename T>
    const param_list &get_if(const std::map<std::string, T> &, std::string &) const { return l; }
};
struct xamg_overrides_holder {
    param_list l;
    explicit xamg_overrides_holder(size_t) {}
    void fill_in(const param_list &) {}
    bool find(size_t) const { return false; }
    const param_list &get(size_t) const { return l; }
};
}  // namespace params
namespace mpi {
struct token {};
static token null_token;
}  // namespace mpi
// named time regions of the reference: not timed here
struct time_monitor_stub {
    void start(const char *) {}
    void stop(const char *) {}
};
static time_monitor_stub monitor;
namespace blas {
template <typename F> struct ConstVectorsCache {
    static const vector::vector &get(int nv, F value) {
        static std::map<std::pair<int, double>, vector::vector> cache;
        vector::vector &v = cache[std::make_pair(nv, (double)value)];
        if (!v.if_allocated) {
            F *p = v.alloc_and_get_aligned_ptr<F>(1, (uint16_t)nv);
            for (int k = 0; k < nv; ++k) p[k] = value;
            v.if_initialized = true;
            v.if_zero = (value == F(0));
        }
        return v;
    }
    static const vector::vector &get_ones_vec(int nv) { return get(nv, F(1)); }
    static const vector::vector &get_minus_ones_vec(int nv) { return get(nv, F(-1)); }
    static const vector::vector &get_zeroes_vec(int nv) { return get(nv, F(0)); }
};
}  // namespace blas
namespace blas2 {
// y = A x for the one-process operator (blas2.h:305-326 reduces to csr_Ax_y)
template <typename F, uint16_t NV>
void Ax_y(matrix::matrix &A, const vector::vector &x, vector::vector &y, uint16_t) {
    if (x.if_zero) {  // csr_matvec.inl:156-159
        blas::set_const<F, NV>(y, 0.0, true);
        return;
    }
    if (sizeof(F) == sizeof(float))
        ref_csr_ax_y_f(A.n, A.rp, A.ci, A.v32.data(), x.get_aligned_ptr<float>(), y.get_aligned_ptr<float>(), NV);
    else
        ref_csr_ax_y_d(A.n, A.rp, A.ci, A.v, x.get_aligned_ptr<double>(), y.get_aligned_ptr<double>(), NV);
    y.if_initialized = true;
    y.if_zero = false;
}
// y += A x (blas2.h:283-303 reduces to csr_Axpy)
template <typename F, uint16_t NV>
void Axpy(matrix::matrix &A, const vector::vector &x, vector::vector &y, uint16_t) {
    if (x.if_zero) return;  // csr_matvec.inl:40-42
    if (sizeof(F) == sizeof(float))
        ref_csr_axpy_f(A.n, A.rp, A.ci, A.v32.data(), x.get_aligned_ptr<float>(), y.get_aligned_ptr<float>(), NV);
    else
        ref_csr_axpy_d(A.n, A.rp, A.ci, A.v, x.get_aligned_ptr<double>(), y.get_aligned_ptr<double>(), NV);
    y.if_zero = false;
}
// blas2::SGS (blas2.h:184-281) on one process with the operator's hybrid
// blocks as its cores: ref_hsgs_* (t from the incoming x, then csr_SGS per
// block); a flagged-zero x is zeroed first, as blas2.h:264-265 does before
// the sweep (its off-block products of a zero x add nothing to t)
template <typename F, uint16_t NV>
void SGS(matrix::matrix &A, const vector::vector &b, vector::vector &x, vector::vector &, const vector::vector &relax,
         uint16_t) {
    if (x.if_zero) blas::set_const<F, NV>(x, 0.0, true);
    if (sizeof(F) == sizeof(float))
        ref_hsgs_f(A.n, A.rp, A.ci, A.v32.data(), A.invd.get_aligned_ptr<float>(), b.get_aligned_ptr<float>(),
                   x.get_aligned_ptr<float>(), relax.get_aligned_ptr<float>(), NV, A.nb, A.bp.data());
    else
        ref_hsgs_d(A.n, A.rp, A.ci, A.v, A.invd.get_aligned_ptr<double>(), b.get_aligned_ptr<double>(),
                   x.get_aligned_ptr<double>(), relax.get_aligned_ptr<double>(), NV, A.nb, A.bp.data());
    x.if_zero = false;
}
}  // namespace blas2
namespace solver {
// what a solver sees of its preconditioner and smoothers (solver.h:77-103)
struct base_solver_interface {
    virtual ~base_solver_interface() {}
    virtual void solve(vector::vector &, const vector::vector &, mpi::token & = mpi::null_token) {}
    virtual void solve(vector::vector &x, const vector::vector &b, const vector::vector &,
                       mpi::token &tok = mpi::null_token) {
        solve(x, b, tok);
    }
    virtual void matrix_info() {}
    virtual void setup(const params::global_param_list &) {}
    virtual void renew_params(const params::global_param_list &, bool = true) {}
    virtual void renew_param_list(const params::param_list &) {}
};
// the solver factory and the hypre hierarchy import, named by
// MultiGrid::setup (which the checks never run: they hand the class its
// hierarchy and solvers)
template <typename F, uint16_t NV>
std::shared_ptr<base_solver_interface> construct_basic_solver(const params::global_param_list &,
                                                              const params::param_list &, matrix::matrix &,
                                                              const std::string & = "solver") {
    return nullptr;
}
}  // namespace solver
namespace hypre {
template <typename F>
void get_full_hierarchy(matrix::matrix &, std::vector<matrix::mg_layer> &, const params::global_param_list &) {}
template <typename F>
void get_per_level_hierarchy(matrix::matrix &, std::vector<matrix::mg_layer> &,
                             const params::global_param_list &) {}
}  // namespace hypre
namespace solver {
template <typename F, uint16_t NV> struct base_solver;
// one process: the allreduce of a local value is the value itself
struct allreduce_stub {
    void push_vector(const vector::vector &) {}
    void pull_vector(vector::vector &) {}
    void init() {}
    void process_sync_action() {}
    void process_async_action() {}
    void wait() {}
    mpi::token &get_token() { return mpi::null_token; }
};
template <typename F, uint16_t NV> struct stats_stub {
    base_solver<F, NV> *s;
    explicit stats_stub(base_solver<F, NV> *s_) : s(s_) {}
    bool conv_check = false;
    double abs_tol = 0, rel_tol = 0;
    int iters = 0;
    std::vector<double> res0 = std::vector<double>(NV, 0.0), res = std::vector<double>(NV, 0.0);
    std::vector<int> status = std::vector<int>(NV, 0);
    vector::vector *p_iconv = nullptr;
    double *hist = nullptr;
    int cap = 0, cnt = 0;
    struct convergence_status_t {
        stats_stub *st;
        void set_initial_residual(const vector::vector &r) {
            for (int k = 0; k < NV; ++k) st->res0[k] = r.get_aligned_ptr<F>()[k];
        }
    } convergence_status{this};
    // stats.h:90-99: every solve starts its iteration count afresh
    void init(vector::vector &) { iters = 0; }
    void init(vector::vector &, vector::vector &iconv) {
        iters = 0;
        p_iconv = &iconv;
    }
    int increment_iters_counter() { return ++iters; }
    bool check_and_record(const vector::vector &r) {
        if (!conv_check) return false;
        for (int k = 0; k < NV; ++k)
            if (!status[k]) res[k] = r.get_aligned_ptr<F>()[k];
        if (hist && cnt < cap) std::memcpy(hist + (size_t)cnt * NV, res.data(), sizeof(double) * NV);
        cnt++;
        bool all = true;
        for (int k = 0; k < NV; ++k) {
            if (status[k]) continue;
            double tol = std::max(abs_tol, rel_tol * std::sqrt(res0[k]));
            F a = std::sqrt(res[k]);
            if (a > (F)tol) all = false;
            else status[k] = 1;
        }
        if (p_iconv)
            for (int k = 0; k < NV; ++k)
                if (status[k]) p_iconv->get_aligned_ptr<F>()[k] = 0;
        return all;
    }
    // stats.h:195-206: r0 = b - A x, r_norm = (r0, r0), the initial check
    bool is_converged_initial(vector::vector &r0, vector::vector &r_norm) {
        s->get_residual(r0);
        blas::vector_norm<F, NV>(r0, 0, r_norm);
        if (!conv_check) return false;
        convergence_status.set_initial_residual(r_norm);
        return check_and_record(r_norm);
    }
    bool is_converged_initial(vector::vector &r0) {
        s->get_residual(r0);
        if (!conv_check) return false;
        vector::vector t;
        t.alloc<F>(1, NV);
        blas::vector_norm<F, NV>(r0, 0, t);
        convergence_status.set_initial_residual(t);
        return check_and_record(t);
    }
    bool is_converged_simple(vector::vector &r_norm) { return check_and_record(r_norm); }
    // the smoothers' and the preconditioner's own checks: off in those roles
    bool is_converged_initial() { return false; }
    bool is_converged() { return false; }
    bool is_converged(vector::vector &) { return false; }
    void print_residuals_footer() {}
};
template <typename F, uint16_t NV> struct base_solver : base_solver_interface {
    std::string solver_role;
    params::param_list param_list;
    matrix::matrix &A;
    vector::vector *x = nullptr;
    const vector::vector *b = nullptr;
    std::vector<vector::vector> buffer;
    base_solver_interface *precond = nullptr;
    allreduce_stub allreduce_buffer;
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
    // buffers and a convergence vector of ones, then the class's own solve
    void run(int nvecs) {
        buffer.resize(nvecs);
        for (auto &v : buffer) v.template alloc<F>(x->size, NV);
        vector::vector conv;
        F *c = conv.alloc_and_get_aligned_ptr<F>(1, NV);
        for (int k = 0; k < NV; ++k) c[k] = F(1);
        conv.if_initialized = true;
        conv.if_zero = false;
        solve(conv);
    }
    virtual void init(const params::param_list &, const std::string &) {}
    virtual void solve(const vector::vector &conv, mpi::token &tok = mpi::null_token) = 0;
    virtual void matrix_info() = 0;
    // solver.h:227-245: point at x and b, then the class's own solve
    void solve(vector::vector &x_, const vector::vector &b_, const vector::vector &conv,
               mpi::token &tok = mpi::null_token) override {
        x = &x_;
        b = &b_;
        if (buffer.empty()) {
            buffer.resize(buffer_nvecs);
            for (auto &v : buffer) v.template alloc<F>(x_.size, NV);
        }
        solve(conv, tok);
    }
    using base_solver_interface::solve;
};
}  // namespace solver
}  // namespace XAMG

// the reference's class-body macro (solver.h:256-281), restated: the names
// the solver classes take from their base, a constructor, the overrides
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
