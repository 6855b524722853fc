// BLAS-1 loops of the reference, compiled unchanged with its generic release
// flags, and BiCGStab in the reference's step order over them.
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

// Convergence as convergence.h:85-130 + stats.h:195-245: squared residual
// norms per column, a column freezes once sqrt(res) <= max(abs, rel*sqrt(res0)).
struct Conv {
    std::vector<double> res0, res;
    std::vector<int> done;
    double abs_tol, rel_tol;
    double *hist; int cap, cnt, nv;
    void push() {
        if (hist && cnt < cap) std::memcpy(hist + (size_t)cnt * nv, res.data(), sizeof(double) * nv);
        cnt++;
    }
    void update(const double *r) {
        for (int k = 0; k < nv; ++k) if (!done[k]) res[k] = r[k];
        push();
    }
    bool check(double *iconv) {
        bool all = true;
        for (int k = 0; k < nv; ++k) {
            if (done[k]) continue;
            if (std::sqrt(res[k]) > std::max(abs_tol, rel_tol * std::sqrt(res0[k]))) all = false;
            else { done[k] = 1; iconv[k] = 0.0; }
        }
        return all;
    }
};

// The AMG hierarchy handed to the PBiCGStab driver: per level the operator,
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

// (P)BiCGStab in the step order of pbicgstab.inl:48-207 (bicgstab.inl:44-197
// without a preconditioner: the preconditioned vectors are p and s).
struct Bicgstab {
    int64_t n; const int *rp, *ci; const double *v, *b; double *x; int nv, max_iters;
    double abs_tol, rel_tol; double *hist; int cap;
    const Hier *mg;
    int iters;
    template <int NV> void run() {
        typedef double F;
        size_t sz = (size_t)n * NV;
        std::vector<F> r0(sz, 0.0), r(sz, 0.0), p(sz, 0.0), vv(sz, 0.0), s(sz, 0.0), t(sz, 0.0),
            p_(sz, 0.0), s_(sz, 0.0);
        vector R0 = block(r0.data(), n, NV), R = block(r.data(), n, NV), P = block(p.data(), n, NV),
               V = block(vv.data(), n, NV), S = block(s.data(), n, NV), T = block(t.data(), n, NV),
               P_ = block(p_.data(), n, NV), S_ = block(s_.data(), n, NV);
        vector X = block(x, n, NV), B = block(b, n, NV);
        std::vector<F> one(NV, 1.0), mone(NV, -1.0), ic(NV, 1.0);
        std::vector<F> rho(NV), res(NV), s1(NV), s2(NV), s3(NV), s4(NV), al(NV), be(NV), om(NV),
            alc(NV), omc(NV);
        vector a1 = scalars(one.data(), NV), a_1 = scalars(mone.data(), NV),
               iconv = scalars(ic.data(), NV), Rho = scalars(rho.data(), NV),
               Res = scalars(res.data(), NV), S1 = scalars(s1.data(), NV),
               S2 = scalars(s2.data(), NV), S3 = scalars(s3.data(), NV),
               S4 = scalars(s4.data(), NV), Al = scalars(al.data(), NV),
               Be = scalars(be.data(), NV), Om = scalars(om.data(), NV),
               Alc = scalars(alc.data(), NV), Omc = scalars(omc.data(), NV);
        auto Ax = [&](const vector &in, vector &out) {
            ref_csr_ax_y_d(n, rp, ci, v, in.get_aligned_ptr<F>(), out.get_aligned_ptr<F>(), NV);
        };
        // M^{-1}: one V-cycle from zero (MultiGrid::solve with max_iters 1)
        auto precond = [&](vector &out, const vector &in) {
            blas::set_const<F, NV>(out, 0.0, true);
            if (mg->reduced)
                mg->cycle_reduced<NV>(out.get_aligned_ptr<F>(), in.get_aligned_ptr<F>(), mg->mg_cycle);
            else
                mg->cycle<NV>(0, out.get_aligned_ptr<F>(), in.get_aligned_ptr<F>(), mg->mg_cycle);
        };
        Conv cv{std::vector<double>(NV), std::vector<double>(NV), std::vector<int>(NV, 0),
                abs_tol, rel_tol, hist, cap, 0, NV};
        // 1-2. r0 = b - A x (solver.h:183-190), rho = (r0, r0)
        Ax(X, R0);
        blas::axpby<F, NV>(1.0, B, -1.0, R0);
        blas::dot<F, NV>(R0, R0, Rho);
        for (int k = 0; k < NV; ++k) cv.res0[k] = rho[k];
        cv.update(rho.data());
        if (cv.check(ic.data())) { iters = 0; return; }
        blas::copy<F, NV>(R0, R);
        blas::copy<F, NV>(R0, P);
        vector &PP = mg ? P_ : P, &SS = mg ? S_ : S;
        int it = 0;
        for (bool last = false; !last;) {
            it++;
            if (it >= max_iters) last = true;
            if (mg) precond(P_, P);                              // 5*
            Ax(PP, V);                                            // 5
            blas::dot<F, NV>(V, R0, S1);                          // 6
            blas::xdivy_z<F, NV>(Rho, S1, Al);
            blas::scal<F, NV>(a_1, Al);                           // 7
            blas::axpby_z<F, NV>(a1, R, Al, V, S);
            blas::scal<F, NV>(a_1, Al);
            if (mg) precond(S_, S);                              // 8*
            Ax(SS, T);                                            // 8
            blas::dot<F, NV>(T, S, S2);                           // 9
            blas::dot<F, NV>(T, T, S3);
            blas::dot<F, NV>(S, S, S4);
            blas::xdivy_z<F, NV>(S2, S3, Om);
            blas::ax_y<F, NV>(iconv, Al, Alc);                    // 10
            blas::ax_y<F, NV>(iconv, Om, Omc);
            blas::axpbypcz<F, NV>(Alc, PP, Omc, SS, a1, X);
            blas::ax_y<F, NV>(Om, S2, Res);                       // 12
            blas::axpby<F, NV>(a1, S4, a_1, Res);
            cv.update(res.data());
            if (cv.check(ic.data())) break;
            blas::scal<F, NV>(a_1, Om);                           // 11
            blas::axpby_z<F, NV>(a1, S, Om, T, R);
            blas::scal<F, NV>(a_1, Om);
            blas::dot<F, NV>(R, R0, S1);                          // 15
            blas::xdivy_z<F, NV>(S1, Rho, S2);                    // 16
            blas::xdivy_z<F, NV>(Al, Om, S3);
            blas::ax_y<F, NV>(S2, S3, Be);
            blas::copy<F, NV>(S1, Rho);
            blas::ax_y<F, NV>(Om, Be, S1);                        // 17
            blas::scal<F, NV>(a_1, S1);
            blas::axpbypcz<F, NV>(a1, R, S1, V, Be, P);
        }
        iters = it;
    }
};

// Shared state of the PCG and RBiCGStab drivers: operator, optional V-cycle
// preconditioner (identity without one: M^{-1} r = r), convergence.
struct KrylovBase {
    int64_t n; const int *rp, *ci; const double *v, *b; double *x; int nv, max_iters;
    double abs_tol, rel_tol; double *hist; int cap;
    const Hier *mg;
    int iters;
    template <int NV> void Ax(const vector &in, vector &out) const {
        ref_csr_ax_y_d(n, rp, ci, v, in.get_aligned_ptr<double>(), out.get_aligned_ptr<double>(), NV);
    }
    // set_const(out, 0); precond->solve(out, in)
    template <int NV> void precond(vector &out, const vector &in) const {
        blas::set_const<double, NV>(out, 0.0, true);
        if (mg && mg->reduced)
            mg->cycle_reduced<NV>(out.get_aligned_ptr<double>(), in.get_aligned_ptr<double>(), mg->mg_cycle);
        else if (mg)
            mg->cycle<NV>(0, out.get_aligned_ptr<double>(), in.get_aligned_ptr<double>(), mg->mg_cycle);
        else
            blas::copy<double, NV>(in, out);
    }
};

// PCG in the step order of pcg.inl:48-160.
struct Pcg : KrylovBase {
    explicit Pcg(const KrylovBase &k) : KrylovBase(k) {}
    template <int NV> void run() {
        typedef double F;
        size_t sz = (size_t)n * NV;
        std::vector<F> r(sz, 0.0), z(sz, 0.0), p(sz, 0.0), ap(sz, 0.0);
        vector R = block(r.data(), n, NV), Z = block(z.data(), n, NV), P = block(p.data(), n, NV),
               AP = block(ap.data(), n, NV), X = block(x, n, NV), B = block(b, n, NV);
        std::vector<F> one(NV, 1.0), mone(NV, -1.0), ic(NV, 1.0), s1(NV), s2(NV), s3(NV), al(NV), be(NV),
            res(NV), alc(NV);
        vector a1 = scalars(one.data(), NV), a_1 = scalars(mone.data(), NV), iconv = scalars(ic.data(), NV),
               S1 = scalars(s1.data(), NV), S2 = scalars(s2.data(), NV), S3 = scalars(s3.data(), NV),
               Al = scalars(al.data(), NV), Be = scalars(be.data(), NV), Res = scalars(res.data(), NV),
               Alc = scalars(alc.data(), NV);
        Conv cv{std::vector<double>(NV), std::vector<double>(NV), std::vector<int>(NV, 0),
                abs_tol, rel_tol, hist, cap, 0, NV};
        // r = b - A x, res0 = (r, r) (stats.h:208-219)
        Ax<NV>(X, R);
        blas::axpby<F, NV>(1.0, B, -1.0, R);
        blas::dot<F, NV>(R, R, Res);
        for (int k = 0; k < NV; ++k) cv.res0[k] = res[k];
        cv.update(res.data());
        if (cv.check(ic.data())) { iters = 0; return; }
        precond<NV>(Z, R);
        blas::copy<F, NV>(Z, P);
        int it = 0;
        for (bool last = false; !last;) {
            it++;
            if (it >= max_iters) last = true;
            Ax<NV>(P, AP);
            blas::dot<F, NV>(R, Z, S1);
            blas::dot<F, NV>(P, AP, S2);
            blas::xdivy_z<F, NV>(S1, S2, Al);
            blas::ax_y<F, NV>(iconv, Al, Alc);
            blas::axpby<F, NV>(Alc, P, a1, X);
            blas::scal<F, NV>(a_1, Al);
            blas::axpby<F, NV>(Al, AP, a1, R);
            precond<NV>(Z, R);
            blas::dot<F, NV>(R, Z, S3);
            blas::xdivy_z<F, NV>(S3, S1, Be);
            blas::axpby<F, NV>(a1, Z, Be, P);
            blas::dot<F, NV>(R, R, Res);
            cv.update(res.data());
            if (cv.check(ic.data())) break;
        }
        iters = it;
    }
};

// RBiCGStab in the step order of rbicgstab.inl:48-225 (the allreduce that
// the reference overlaps with the preconditioner changes no value on one
// process).
struct Rbicgstab : KrylovBase {
    explicit Rbicgstab(const KrylovBase &k) : KrylovBase(k) {}
    template <int NV> void run() {
        typedef double F;
        size_t sz = (size_t)n * NV;
        std::vector<F> r0(sz, 0.0), r(sz, 0.0), z(sz, 0.0), v_(sz, 0.0), vv(sz, 0.0), s(sz, 0.0),
            t_(sz, 0.0), t(sz, 0.0);
        vector R0 = block(r0.data(), n, NV), R = block(r.data(), n, NV), Z = block(z.data(), n, NV),
               V_ = block(v_.data(), n, NV), V = block(vv.data(), n, NV), S = block(s.data(), n, NV),
               T_ = block(t_.data(), n, NV), T = block(t.data(), n, NV), X = block(x, n, NV),
               B = block(b, n, NV);
        std::vector<F> one(NV, 1.0), mone(NV, -1.0), ic(NV, 1.0), rho(NV), delta(NV), al(NV), om(NV),
            theta(NV), phi(NV), psi(NV), eta(NV), res(NV), alc(NV), omc(NV), be(NV), tmp(NV);
        vector a1 = scalars(one.data(), NV), a_1 = scalars(mone.data(), NV), iconv = scalars(ic.data(), NV),
               Rho = scalars(rho.data(), NV), Delta = scalars(delta.data(), NV), Al = scalars(al.data(), NV),
               Om = scalars(om.data(), NV), Theta = scalars(theta.data(), NV), Phi = scalars(phi.data(), NV),
               Psi = scalars(psi.data(), NV), Eta = scalars(eta.data(), NV), Res = scalars(res.data(), NV),
               Alc = scalars(alc.data(), NV), Omc = scalars(omc.data(), NV), Be = scalars(be.data(), NV),
               Tmp = scalars(tmp.data(), NV);
        Conv cv{std::vector<double>(NV), std::vector<double>(NV), std::vector<int>(NV, 0),
                abs_tol, rel_tol, hist, cap, 0, NV};
        Ax<NV>(X, R0);                                             // 1
        blas::axpby<F, NV>(1.0, B, -1.0, R0);
        blas::dot<F, NV>(R0, R0, Rho);                            // 2
        for (int k = 0; k < NV; ++k) cv.res0[k] = rho[k];
        cv.update(rho.data());
        if (cv.check(ic.data())) { iters = 0; return; }
        blas::copy<F, NV>(R0, R);
        precond<NV>(Z, R0);                                       // 3
        blas::copy<F, NV>(Z, V_);                                 // 4
        int it = 0;
        for (bool last = false; !last;) {
            it++;
            if (it >= max_iters) last = true;
            Ax<NV>(V_, V);                                        // 6
            blas::dot<F, NV>(V, R0, Delta);                       // 7
            precond<NV>(S, V);                                    // 8
            blas::xdivy_z<F, NV>(Rho, Delta, Al);                 // 9
            blas::scal<F, NV>(a_1, Al);                           // 10
            blas::axpby_z<F, NV>(a1, Z, Al, S, T_);
            blas::scal<F, NV>(a_1, Al);
            Ax<NV>(T_, T);                                        // 11
            blas::scal<F, NV>(a_1, Al);                           // 12
            blas::axpby<F, NV>(Al, V, a1, R);
            blas::scal<F, NV>(a_1, Al);
            blas::dot<F, NV>(T, R, Theta);                        // 13
            blas::dot<F, NV>(T, T, Phi);
            blas::dot<F, NV>(T, R0, Psi);
            blas::dot<F, NV>(R, R, Eta);
            precond<NV>(Z, T);                                    // 14
            blas::xdivy_z<F, NV>(Theta, Phi, Om);                 // 15
            blas::scal<F, NV>(a_1, Om);                           // 16
            blas::axpby<F, NV>(Om, T, a1, R);
            blas::scal<F, NV>(a_1, Om);
            blas::ax_y<F, NV>(Om, Theta, Res);                    // 17
            blas::axpby<F, NV>(a1, Eta, a_1, Res);
            blas::ax_y<F, NV>(iconv, Al, Alc);                    // 23
            blas::ax_y<F, NV>(iconv, Om, Omc);
            blas::axpbypcz<F, NV>(Alc, V_, Omc, T_, a1, X);
            cv.update(res.data());
            if (cv.check(ic.data())) break;
            blas::ax_y<F, NV>(Om, Psi, Rho);                      // 21
            blas::scal<F, NV>(a_1, Rho);
            blas::ax_y<F, NV>(Delta, Om, Tmp);                    // 22
            blas::xdivy_z<F, NV>(Rho, Tmp, Be);
            blas::scal<F, NV>(a_1, Om);                           // 24 (omega stays negated)
            blas::axpby<F, NV>(a1, T_, Om, Z);
            blas::ax_y<F, NV>(Om, Be, Delta);                     // 25
            blas::scal<F, NV>(a_1, Om);
            blas::axpbypcz<F, NV>(a1, Z, Delta, S, Be, V_);
        }
        iters = it;
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
int ref_dense_inverse_d(int64_t n, const double *a, double *ainv) {
    XAMG::matrix::dense_matrix<double> m(XAMG::mem::CORE), mi(XAMG::mem::CORE);
    m.nrows = m.block_nrows = (uint64_t)n;
    m.ncols = m.block_ncols = (uint64_t)n;
    m.val = block(a, n * n, 1);
    XAMG::matrix::inverse<double>(m, mi);
    std::memcpy(ainv, mi.val.get_aligned_ptr<double>(), sizeof(double) * (size_t)(n * n));
    return 0;
}
int ref_bicgstab_d(int64_t n, const int *rp, const int *ci, const double *v, const double *b,
                   double *x, int nv, int max_iters, double abs_tol, double rel_tol, double *hist,
                   int hist_cap) {
    Bicgstab f{n, rp, ci, v, b, x, nv, max_iters, abs_tol, rel_tol, hist, hist_cap, nullptr, 0};
    if (dispatch_nv(nv, f)) return -1;
    return f.iters;
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
int ref_krylov_d(int method, int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                 const double *const *av, const int *const *prp, const int *const *pci,
                 const double *const *pv, const int *const *rrp, const int *const *rci,
                 const double *const *rv, const int *nb, const int64_t *const *bp, double relax, int pre_it,
                 int post_it, int smoother, const double *b, double *x, int nv, int max_iters, double abs_tol,
                 double rel_tol, double *hist, int hist_cap) {
    std::unique_ptr<Hier> h(make_hier(nlev, nrows, arp, aci, av, prp, pci, pv, rrp, rci, rv, nb, bp, relax,
                                      pre_it, post_it, smoother));
    KrylovBase kb{nrows[0], arp[0], aci[0], av[0], b, x, nv, max_iters, abs_tol, rel_tol, hist, hist_cap,
                  h.get(), 0};
    if (method == 0) {
        Bicgstab f{kb.n, kb.rp, kb.ci, kb.v, b, x, nv, max_iters, abs_tol, rel_tol, hist, hist_cap, h.get(), 0};
        if (dispatch_nv(nv, f)) return -1;
        return f.iters;
    }
    if (method == 1) {
        Pcg f(kb);
        if (dispatch_nv(nv, f)) return -1;
        return f.iters;
    }
    if (method == 2) {
        Rbicgstab f(kb);
        if (dispatch_nv(nv, f)) return -1;
        return f.iters;
    }
    return -1;
}
int ref_pbicgstab_amg_d(int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                        const double *const *av, const int *const *prp, const int *const *pci,
                        const double *const *pv, const int *const *rrp, const int *const *rci,
                        const double *const *rv, const int *nb, const int64_t *const *bp, double relax,
                        int pre_it, int post_it, const double *b, double *x, int nv, int max_iters,
                        double abs_tol, double rel_tol, double *hist, int hist_cap) {
    if (nlev < 2) return -1;
    Hier h{nlev, nrows, arp, aci, av, prp, pci, pv, rrp, rci, rv, nb, bp, relax, pre_it, post_it, 0, 0, 0,
           {}, {}, {}, {}, {}, {}, {}};
    h.init();
    Bicgstab f{nrows[0], arp[0], aci[0], av[0], b, x, nv, max_iters, abs_tol, rel_tol, hist, hist_cap, &h, 0};
    if (dispatch_nv(nv, f)) return -1;
    return f.iters;
}
}
