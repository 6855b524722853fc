// The reference's multigrid solver class (src/solvers/detail/mg.inl:
// MultiGrid::solve and MG_cycle<T1, T2>) and its smoother classes HSGS
// (hsgs.inl) and Jacobi (jacobi.inl), compiled unchanged against the
// stand-ins of solver_base.h, one process.  The hierarchy is handed in (the
// reference takes it from hypre); the coarsest level is the Direct solver's
// product with the reference's Gauss-Jordan inverse.  Compiled with the row
// loops' flags: the Jacobi update is fused as in the reference's FMA
// configuration, and the vector operations of the cycle (scalings by +-1)
// round alike either way.
#include "solver_base.h"
#include "solvers/detail/hsgs.inl"
#include "solvers/detail/jacobi.inl"
#include "solvers/detail/mg.inl"

using namespace refloops;
using XAMG::matrix::matrix;

namespace {

// Direct::solve (direct.inl:51-59): x = A^{-1} b with the Gauss-Jordan
// inverse of the coarsest operator, in the level's precision
struct Coarse : XAMG::solver::base_solver_interface {
    int64_t n;
    bool f32;
    std::vector<double> inv64;
    std::vector<float> inv32;
    int nv;
    void solve(vector &x, const vector &b, XAMG::mpi::token & = XAMG::mpi::null_token) override {
        if (f32)
            ref_dense_ax_y_f(n, n, inv32.data(), b.get_aligned_ptr<float>(), x.get_aligned_ptr<float>(), nv);
        else
            ref_dense_ax_y_d(n, n, inv64.data(), b.get_aligned_ptr<double>(), x.get_aligned_ptr<double>(), nv);
        x.if_initialized = true;
        x.if_zero = false;
    }
};

// The Chebyshev smoother class, compiled in its own unit with the BLAS
// flags (cheb.cpp: its vector updates round apart, as the oracle's), called
// as a smoother of this cycle; a flag-cleared x is zeroed first
struct ChebSmoother : XAMG::solver::base_solver_interface {
    matrix *A;
    int nv, order;
    double fraction;
    void solve(vector &x, const vector &b, XAMG::mpi::token & = XAMG::mpi::null_token) override {
        if (x.if_zero) std::memset(x.get_aligned_ptr<double>(), 0, sizeof(double) * x.size * nv);
        ref_chebyshev_d(A->n, A->rp, A->ci, A->v, b.get_aligned_ptr<double>(), x.get_aligned_ptr<double>(), nv,
                        order, fraction, A->min_eig, A->max_eig);
        x.if_initialized = true;
        x.if_zero = false;
    }
};

struct MGBase {
    virtual ~MGBase() {}
    virtual void apply(const double *b, double *x) = 0;
    virtual void set_chebyshev(int order, double fraction, const double *min_eig, const double *max_eig) = 0;
};

template <int NV> struct MGImpl : MGBase {
    vector dx, db;
    matrix A0;
    XAMG::solver::MultiGrid<double, NV> mg{A0, dx, db};
    std::vector<std::shared_ptr<XAMG::solver::base_solver_interface>> keep;
    std::vector<std::vector<double>> invd64;
    std::vector<std::vector<float>> invd32;

    MGImpl(int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci, const double *const *av,
           const int *const *prp, const int *const *pci, const double *const *pv, const int *const *rrp,
           const int *const *rci, const double *const *rv, const int *nb, const int64_t *const *bp, double relax,
           int pre_it, int post_it, int smoother, int cycle, int reduced) {
        mg.param_list.v["max_iters"] = 1;
        mg.param_list.v["mg_cycle"] = cycle;
        mg.mg_tree.resize(nlev);
        invd64.resize(nlev);
        invd32.resize(nlev);
        for (int l = 0; l < nlev; ++l) {
            XAMG::matrix::mg_layer &L = mg.mg_tree[l];
            const bool f32 = reduced && l > 0;
            const int64_t n = nrows[l];
            L.A.n = L.A.ncols = n; L.A.rp = arp[l]; L.A.ci = aci[l]; L.A.v = av[l];
            L.A.reduced_prec = f32;
            L.A.nb = nb[l];
            L.A.bp.assign(bp[l], bp[l] + nb[l] + 1);
            if (f32) L.A.v32.assign(av[l], av[l] + arp[l][n]);
            // inverse diagonal, csr_matrix.h:344-349 in the level's precision
            invd64[l].assign(n, 0.0);
            invd32[l].assign(n, 0.f);
            for (int64_t i = 0; i < n; ++i)
                for (int j = arp[l][i]; j < arp[l][i + 1]; ++j)
                    if (aci[l][j] == i) {
                        invd64[l][i] = 1.0 / av[l][j];
                        invd32[l][i] = (float)(1.0 / (double)(float)av[l][j]);
                    }
            if (f32) L.A.invd = block(invd32[l].data(), n, 1);
            else L.A.invd = block(invd64[l].data(), n, 1);
            if (l + 1 < nlev) {
                const int64_t nc = nrows[l + 1];
                const bool t32 = reduced;  // the transfers of every level are FP32 when reduced
                L.P.n = n; L.P.ncols = nc; L.P.rp = prp[l]; L.P.ci = pci[l]; L.P.v = pv[l];
                L.R.n = nc; L.R.ncols = n; L.R.rp = rrp[l]; L.R.ci = rci[l]; L.R.v = rv[l];
                L.P.reduced_prec = L.R.reduced_prec = t32;
                if (t32) {
                    L.P.v32.assign(pv[l], pv[l] + prp[l][n]);
                    L.R.v32.assign(rv[l], rv[l] + rrp[l][nc]);
                }
            }
            // mg.inl:157-183: level 0 one vector (+ an FP32 one when reduced), three below
            if (l == 0) {
                L.buffer.emplace_back();
                L.buffer.back().alloc<double>(n, NV);
                if (reduced) {
                    L.buffer.emplace_back();
                    L.buffer.back().alloc<float>(n, NV);
                }
            } else {
                for (int k = 0; k < 3; ++k) {
                    L.buffer.emplace_back();
                    if (f32) L.buffer.back().alloc<float>(n, NV);
                    else L.buffer.back().alloc<double>(n, NV);
                }
            }
        }
        // smoothers of every level but the coarsest (mg.inl:132-145)
        for (int l = 0; l + 1 < nlev; ++l) {
            matrix &A = mg.mg_tree[l].get_A();
            for (int role = 0; role < 2; ++role) {
                const int it = role ? post_it : pre_it;
                std::shared_ptr<XAMG::solver::base_solver_interface> s;
                if (A.reduced_prec) s = make_smoother<float>(A, smoother, relax, it);
                else s = make_smoother<double>(A, smoother, relax, it);
                (role ? mg.post_smooth : mg.pre_smooth).push_back(s);
            }
        }
        // the coarsest level: Direct, inverse in the level's precision
        {
            const int l = nlev - 1;
            const int64_t n = nrows[l];
            auto c = std::make_shared<Coarse>();
            c->n = n;
            c->nv = NV;
            c->f32 = reduced != 0;
            std::vector<double> d((size_t)(n * n), 0.0);
            for (int64_t i = 0; i < n; ++i)
                for (int j = arp[l][i]; j < arp[l][i + 1]; ++j) d[i * n + aci[l][j]] = av[l][j];
            // the Gauss-Jordan of inverse.inl from the unit compiled with the
            // BLAS flags (host arithmetic, products rounded apart)
            if (c->f32) {
                std::vector<float> d32(d.begin(), d.end());
                c->inv32.resize(d32.size());
                ref_dense_inverse_f(n, d32.data(), c->inv32.data());
            } else {
                c->inv64.resize(d.size());
                ref_dense_inverse_d(n, d.data(), c->inv64.data());
            }
            mg.coarse_grid_solver = c;
        }
        mg.buffer_nvecs = 1;
    }

    template <typename F>
    std::shared_ptr<XAMG::solver::base_solver_interface> make_smoother(matrix &A, int kind, double relax, int it) {
        vector *nx = nullptr;
        const vector *nb_ = nullptr;
        (void)nx; (void)nb_;
        if (kind == 1) {
            auto s = std::make_shared<XAMG::solver::Jacobi<F, NV>>(A, dx, db);
            s->param_list.v["max_iters"] = it;
            s->param_list.v["relax_factor"] = relax;
            return s;
        }
        auto s = std::make_shared<XAMG::solver::HSGS<F, NV>>(A, dx, db);
        s->param_list.v["max_iters"] = it;
        s->param_list.v["relax_factor"] = relax;
        return s;
    }

    // Chebyshev smoothers on every level but the coarsest (FP64 levels),
    // with the given spectrum bounds of D^-1/2 A D^-1/2 per level
    void set_chebyshev(int order, double fraction, const double *min_eig, const double *max_eig) override {
        const int nlev = (int)mg.mg_tree.size();
        mg.pre_smooth.clear();
        mg.post_smooth.clear();
        for (int l = 0; l + 1 < nlev; ++l) {
            matrix &A = mg.mg_tree[l].get_A();
            A.min_eig = min_eig[l];
            A.max_eig = max_eig[l];
            for (int role = 0; role < 2; ++role) {
                auto c = std::make_shared<ChebSmoother>();
                c->A = &A;
                c->nv = NV;
                c->order = order;
                c->fraction = fraction;
                (role ? mg.post_smooth : mg.pre_smooth).push_back(c);
            }
        }
    }

    void apply(const double *b, double *x) override {
        const int64_t n = mg.mg_tree[0].get_A().n;
        vector X = block(x, n, NV), B = block(b, n, NV);
        vector conv;
        double *c = conv.alloc_and_get_aligned_ptr<double>(1, NV);
        for (int k = 0; k < NV; ++k) c[k] = 1.0;
        conv.if_initialized = true;
        conv.if_zero = false;
        static_cast<XAMG::solver::base_solver_interface &>(mg).solve(X, B, conv);
    }
};

struct Make {
    int nlev; const int64_t *nrows; const int *const *arp; const int *const *aci; const double *const *av;
    const int *const *prp; const int *const *pci; const double *const *pv; const int *const *rrp;
    const int *const *rci; const double *const *rv; const int *nb; const int64_t *const *bp; double relax;
    int pre_it, post_it, smoother, cycle, reduced;
    MGBase *out;
    template <int NV> void run() {
        out = new MGImpl<NV>(nlev, nrows, arp, aci, av, prp, pci, pv, rrp, rci, rv, nb, bp, relax, pre_it, post_it,
                             smoother, cycle, reduced);
    }
};

}  // namespace

extern "C" {
void *ref_mg_create(int nv, int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                    const double *const *av, const int *const *prp, const int *const *pci, const double *const *pv,
                    const int *const *rrp, const int *const *rci, const double *const *rv, const int *nb,
                    const int64_t *const *bp, double relax, int pre_it, int post_it, int smoother) {
    if (nlev < 2) return nullptr;
    Make f{nlev, nrows, arp, aci, av, prp, pci, pv, rrp, rci, rv, nb, bp, relax, pre_it, post_it, smoother & 15,
           (smoother >> 4) & 15, (smoother >> 8) & 1, nullptr};
    if (dispatch_nv(nv, f)) return nullptr;
    return f.out;
}
int ref_mg_apply_d(void *h, const double *b, double *x) {
    ((MGBase *)h)->apply(b, x);
    return 0;
}
void ref_mg_destroy(void *h) { delete (MGBase *)h; }
void ref_mg_set_chebyshev(void *h, int order, double fraction, const double *min_eig, const double *max_eig) {
    ((MGBase *)h)->set_chebyshev(order, fraction, min_eig, max_eig);
}
}
