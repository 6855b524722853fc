// BLAS-1 loops and the dense inverse of the reference, compiled unchanged
// (with the generic release flags in the generic and contract builds), and
// the multigrid cycle of the reference's loops in its MG_cycle order, the
// preconditioner of the solver classes in krylov.cpp.
#include <algorithm>
#include <cstring>
#include <memory>

#include "include_ref.h"
#include "ref_loops.h"

using namespace refloops;
namespace blas = XAMG::blas;

namespace {

struct Blas {
    int op;
    int64_t n; int nv;
    const double *a, *x, *b, *y, *c;
    double *z;
    template <int NV> void run() {
        vector av = scalars(a, nv), bv = scalars(b, nv), cv = scalars(c, nv);
        vector xv = block(x, n, nv), yv = block(y, n, nv), zv = block((const double *)z, n, nv);
        switch (op) {
        case 0: blas::dot<double, NV>(xv, yv, zv); break;           // z[0..nv) = (x, y)
        case 1: blas::axpby<double, NV>(av, xv, bv, zv); break;      // z = a x + b z
        case 2: blas::axpby_z<double, NV>(av, xv, bv, yv, zv); break;
        case 3: blas::axpbypcz<double, NV>(av, xv, bv, yv, cv, zv); break;
        case 4: blas::xdivy_z<double, NV>(xv, yv, zv); break;
        case 5: blas::ax_y<double, NV>(av, xv, zv); break;
        case 6: blas::scal<double, NV>(av, zv); break;
        }
    }
};

int run_blas(Blas f) { return dispatch_nv(f.nv, f); }

// The AMG hierarchy of the multigrid preconditioner: per level the operator,
// its inverse diagonal (csr_matrix.h:344-349), P and R = P^T, the hybrid
// blocks; the coarsest level's inverse from the reference's own Gauss-Jordan
// routine (Direct::init, direct.inl:31-45).
struct Hier {
    int nlev;
    const int64_t *nrows;
    const int *const *arp; const int *const *aci; const double *const *av;
    const int *const *prp; const int *const *pci; const double *const *pv;
    const int *const *rrp; const int *const *rci; const double *const *rv;
    const int *nb; const int64_t *const *bp;
    double relax; int pre_it, post_it;
    int smoother;  // 0: HSGS (hsgs.inl), 1: Jacobi (jacobi.inl, no-check path)
    int mg_cycle;  // 0 V, 1 F, 2 W
    int reduced;   // mg_reduced_precision: levels >= 1, P_0 and R_0 in FP32 (HSGS only)
    std::vector<std::vector<double>> invd;
    std::vector<double> ainv;
    std::vector<std::vector<float>> av32, pv32, rv32, invd32;
    std::vector<float> ainv32;
    void init_reduced() {
        av32.resize(nlev); pv32.resize(nlev); rv32.resize(nlev); invd32.resize(nlev);
        for (int l = 0; l < nlev; ++l) {
            const int64_t n = nrows[l];
            av32[l].assign(av[l], av[l] + arp[l][n]);
            invd32[l].assign(n, 0.f);
            for (int64_t i = 0; i < n; ++i)
                for (int j = arp[l][i]; j < arp[l][i + 1]; ++j)
                    if (aci[l][j] == i) invd32[l][i] = (float)(1.0 / (double)av32[l][j]);  // csr_matrix.h:344-349, F = float
            if (l + 1 < nlev) {
                pv32[l].assign(pv[l], pv[l] + prp[l][n]);
                rv32[l].assign(rv[l], rv[l] + rrp[l][nrows[l + 1]]);
            }
        }
        // the coarsest level's Direct<float> (mg.inl:147-149): the inverse of the FP32 matrix in FP32
        int64_t nc = nrows[nlev - 1];
        std::vector<float> d((size_t)(nc * nc), 0.f);
        for (int64_t i = 0; i < nc; ++i)
            for (int j = arp[nlev - 1][i]; j < arp[nlev - 1][i + 1]; ++j)
                d[i * nc + aci[nlev - 1][j]] = av32[nlev - 1][j];
        ainv32.resize(d.size());
        XAMG::matrix::dense_matrix<float> m(XAMG::mem::CORE), mi(XAMG::mem::CORE);
        m.nrows = m.block_nrows = (uint64_t)nc;
        m.ncols = m.block_ncols = (uint64_t)nc;
        m.val = block(d.data(), nc * nc, 1);
        XAMG::matrix::inverse<float>(m, mi);
        std::memcpy(ainv32.data(), mi.val.get_aligned_ptr<float>(), sizeof(float) * d.size());
    }
    // MG_cycle<float, float> on levels >= 1 of a reduced hierarchy
    template <int NV> void cycle32(int l, float *x, const float *b, int cyc) const {
        int64_t n = nrows[l], nc = nrows[l + 1];
        std::vector<float> rl(NV, (float)relax);
        if (cyc != 1)
            for (int k = 0; k < pre_it; ++k)
                ref_hsgs_f(n, arp[l], aci[l], av32[l].data(), invd32[l].data(), b, x, rl.data(), NV, nb[l], bp[l]);
        std::vector<float> tmp((size_t)n * NV), bH((size_t)nc * NV), xH((size_t)nc * NV, 0.f);
        std::vector<float> one(NV, 1.f), mone(NV, -1.f);
        vector a1 = scalars(one.data(), NV), a_1 = scalars(mone.data(), NV);
        ref_csr_ax_y_f(n, arp[l], aci[l], av32[l].data(), x, tmp.data(), NV);
        vector B = block(b, n, NV), T = block(tmp.data(), n, NV);
        blas::axpby<float, NV>(a1, B, a_1, T);
        ref_csr_ax_y_f(nc, rrp[l], rci[l], rv32[l].data(), tmp.data(), bH.data(), NV);
        if (l + 1 == nlev - 1)
            ref_dense_ax_y_f(nc, nc, ainv32.data(), bH.data(), xH.data(), NV);
        else {
            cycle32<NV>(l + 1, xH.data(), bH.data(), cyc);
            if (cyc == 2) cycle32<NV>(l + 1, xH.data(), bH.data(), 2);
            else if (cyc == 1) cycle32<NV>(l + 1, xH.data(), bH.data(), 0);
        }
        ref_csr_axpy_f(n, prp[l], pci[l], pv32[l].data(), xH.data(), x, NV);
        for (int k = 0; k < post_it; ++k)
            ref_hsgs_f(n, arp[l], aci[l], av32[l].data(), invd32[l].data(), b, x, rl.data(), NV, nb[l], bp[l]);
    }
    // MG_cycle<double, float> on level 0 (mg.inl:186-280, 320-321)
    template <int NV> void cycle_reduced(double *x, const double *b, int cyc) const {
        int64_t n = nrows[0], nc = nrows[1];
        if (cyc != 1) smooth(0, b, x, NV, pre_it);
        std::vector<double> tmp((size_t)n * NV);
        std::vector<float> t32((size_t)n * NV), bH((size_t)nc * NV), xH((size_t)nc * NV, 0.f);
        std::vector<double> one(NV, 1.0), mone(NV, -1.0);
        vector a1 = scalars(one.data(), NV), a_1 = scalars(mone.data(), NV);
        ref_csr_ax_y_d(n, arp[0], aci[0], av[0], x, tmp.data(), NV);
        vector B = block(b, n, NV), T = block(tmp.data(), n, NV), T32 = block(t32.data(), n, NV),
               X = block(x, n, NV);
        blas::axpby<double, NV>(a1, B, a_1, T);
        XAMG::vector::convert<double, float>(T, T32);
        ref_csr_ax_y_f(nc, rrp[0], rci[0], rv32[0].data(), t32.data(), bH.data(), NV);
        if (nlev == 2)
            ref_dense_ax_y_f(nc, nc, ainv32.data(), bH.data(), xH.data(), NV);
        else {
            cycle32<NV>(1, xH.data(), bH.data(), cyc);
            if (cyc == 2) cycle32<NV>(1, xH.data(), bH.data(), 2);
            else if (cyc == 1) cycle32<NV>(1, xH.data(), bH.data(), 0);
        }
        ref_csr_ax_y_f(n, prp[0], pci[0], pv32[0].data(), xH.data(), t32.data(), NV);
        XAMG::vector::convert<float, double>(T32, T);
        blas::axpby<double, NV>(a1, T, a1, X);
        smooth(0, b, x, NV, post_it);
    }
    void init() {
        if (reduced) init_reduced();
        invd.resize(nlev);
        for (int l = 0; l < nlev; ++l) {
            invd[l].assign(nrows[l], 0.0);
            for (int64_t i = 0; i < nrows[l]; ++i)
                for (int j = arp[l][i]; j < arp[l][i + 1]; ++j)
                    if (aci[l][j] == i) invd[l][i] = 1.0 / av[l][j];
        }
        int64_t nc = nrows[nlev - 1];
        std::vector<double> d((size_t)(nc * nc), 0.0);
        for (int64_t i = 0; i < nc; ++i)
            for (int j = arp[nlev - 1][i]; j < arp[nlev - 1][i + 1]; ++j) d[i * nc + aci[nlev - 1][j]] = av[nlev - 1][j];
        ainv.resize(d.size());
        ref_dense_inverse_d(nc, d.data(), ainv.data());
    }
    // HSGS::solve (hsgs.inl:57-91) as a smoother: relax_conv = relax, then
    // `it` calls of blas2::SGS
    // or Jacobi::solve's no-check path: `it` sweeps
    void smooth(int l, const double *b, double *x, int nv, int it) const {
        std::vector<double> rl(nv, relax);
        if (smoother == 1) {
            ref_jacobi_d(nrows[l], arp[l], aci[l], av[l], invd[l].data(), b, x, rl.data(), nv, it);
            return;
        }
        for (int k = 0; k < it; ++k)
            ref_hsgs_d(nrows[l], arp[l], aci[l], av[l], invd[l].data(), b, x, rl.data(), nv, nb[l], bp[l]);
    }
    // MultiGrid::MG_cycle, mg.inl:186-280, one precision; cyc = mg_cycle
    // (0 V, 1 F: no pre-smoothing, then F and V on the coarser level, 2 W)
    template <int NV> void cycle(int l, double *x, const double *b, int cyc) const {
        int64_t n = nrows[l], nc = nrows[l + 1];
        if (cyc != 1) smooth(l, b, x, NV, pre_it);
        std::vector<double> tmp((size_t)n * NV), bH((size_t)nc * NV), xH((size_t)nc * NV, 0.0);
        std::vector<double> one(NV, 1.0), mone(NV, -1.0);
        vector a1 = scalars(one.data(), NV), a_1 = scalars(mone.data(), NV);
        ref_csr_ax_y_d(n, arp[l], aci[l], av[l], x, tmp.data(), NV);
        vector B = block(b, n, NV), T = block(tmp.data(), n, NV);
        blas::axpby<double, NV>(a1, B, a_1, T);
        ref_csr_ax_y_d(nc, rrp[l], rci[l], rv[l], tmp.data(), bH.data(), NV);
        vector XH = block(xH.data(), nc, NV);
        blas::set_const<double, NV>(XH, 0.0, true);
        if (l + 1 == nlev - 1)
            ref_dense_ax_y_d(nc, nc, ainv.data(), bH.data(), xH.data(), NV);  // Direct::solve
        else {
            cycle<NV>(l + 1, xH.data(), bH.data(), cyc);
            if (cyc == 2) cycle<NV>(l + 1, xH.data(), bH.data(), 2);
            else if (cyc == 1) cycle<NV>(l + 1, xH.data(), bH.data(), 0);
        }
        ref_csr_axpy_d(n, prp[l], pci[l], pv[l], xH.data(), x, NV);
        smooth(l, b, x, NV, post_it);
    }
};

// one cycle of a created hierarchy (ref_hier_apply_d)
struct HierApply {
    const Hier *h; const double *b; double *x;
    template <int NV> void run() {
        if (h->reduced) h->cycle_reduced<NV>(x, b, h->mg_cycle);
        else h->cycle<NV>(0, x, b, h->mg_cycle);
    }
};

}  // namespace

extern "C" {
int ref_dot_d(int64_t n, int nv, const double *x, const double *y, double *res) {
    return run_blas(Blas{0, n, nv, nullptr, x, nullptr, y, nullptr, res});
}
int ref_axpby_d(int64_t n, int nv, const double *a, const double *x, const double *b, double *y) {
    return run_blas(Blas{1, n, nv, a, x, b, nullptr, nullptr, y});
}
int ref_axpby_z_d(int64_t n, int nv, const double *a, const double *x, const double *b,
                  const double *y, double *z) {
    return run_blas(Blas{2, n, nv, a, x, b, y, nullptr, z});
}
int ref_axpbypcz_d(int64_t n, int nv, const double *a, const double *x, const double *b,
                   const double *y, const double *c, double *z) {
    return run_blas(Blas{3, n, nv, a, x, b, y, c, z});
}
int ref_xdivy_z_d(int64_t n, int nv, const double *x, const double *y, double *z) {
    return run_blas(Blas{4, n, nv, nullptr, x, nullptr, y, nullptr, z});
}
int ref_ax_y_d(int64_t n, int nv, const double *a, const double *x, double *y) {
    return run_blas(Blas{5, n, nv, a, x, nullptr, nullptr, nullptr, y});
}
int ref_scal_d(int64_t n, int nv, const double *a, double *y) {
    return run_blas(Blas{6, n, nv, a, nullptr, nullptr, nullptr, nullptr, y});
}
int ref_dense_inverse_f(int64_t n, const float *a, float *ainv) {
    XAMG::matrix::dense_matrix<float> m(XAMG::mem::CORE), mi(XAMG::mem::CORE);
    m.nrows = m.block_nrows = (uint64_t)n;
    m.ncols = m.block_ncols = (uint64_t)n;
    m.val = block(a, n * n, 1);
    XAMG::matrix::inverse<float>(m, mi);
    std::memcpy(ainv, mi.val.get_aligned_ptr<float>(), sizeof(float) * (size_t)(n * n));
    return 0;
}
int ref_dense_inverse_d(int64_t n, const double *a, double *ainv) {
    XAMG::matrix::dense_matrix<double> m(XAMG::mem::CORE), mi(XAMG::mem::CORE);
    m.nrows = m.block_nrows = (uint64_t)n;
    m.ncols = m.block_ncols = (uint64_t)n;
    m.val = block(a, n * n, 1);
    XAMG::matrix::inverse<double>(m, mi);
    std::memcpy(ainv, mi.val.get_aligned_ptr<double>(), sizeof(double) * (size_t)(n * n));
    return 0;
}
static Hier *make_hier(int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                       const double *const *av, const int *const *prp, const int *const *pci,
                       const double *const *pv, const int *const *rrp, const int *const *rci,
                       const double *const *rv, const int *nb, const int64_t *const *bp, double relax,
                       int pre_it, int post_it, int smoother) {
    if (nlev < 2) return nullptr;
    Hier *h = new Hier{nlev, nrows, arp, aci, av, prp, pci, pv, rrp, rci, rv, nb, bp, relax, pre_it, post_it,
                       smoother & 15, (smoother >> 4) & 15, (smoother >> 8) & 1, {}, {}, {}, {}, {}, {}, {}};
    h->init();
    return h;
}
void *ref_hier_create(int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                      const double *const *av, const int *const *prp, const int *const *pci,
                      const double *const *pv, const int *const *rrp, const int *const *rci,
                      const double *const *rv, const int *nb, const int64_t *const *bp, double relax, int pre_it,
                      int post_it, int smoother) {
    return make_hier(nlev, nrows, arp, aci, av, prp, pci, pv, rrp, rci, rv, nb, bp, relax, pre_it, post_it,
                     smoother);
}
void ref_hier_destroy(void *h) { delete (Hier *)h; }
int ref_hier_apply_d(void *h, const double *b, double *x, int nv) {
    HierApply f{(const Hier *)h, b, x};
    return dispatch_nv(nv, f);
}
}
