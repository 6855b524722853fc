// BLAS-1 loops of the reference, compiled unchanged with its generic release
// flags, and BiCGStab in the reference's step order over them.
#include <algorithm>
#include <cstring>

#include "include_ref.h"
#include "ref_loops.h"

XAMG::perf_info perf;
ID id;

using namespace refloops;
namespace blas = XAMG::blas;

namespace {

// per-column scalars: a vector of one row and nv columns
template <class T> vector scalars(const T *p, int nv) { return block<T>(p, 1, nv); }

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

struct Bicgstab {
    int64_t n; const int *rp, *ci; const double *v, *b; double *x; int nv, max_iters;
    double abs_tol, rel_tol; double *hist; int cap;
    int iters;
    template <int NV> void run() {
        typedef double F;
        size_t sz = (size_t)n * NV;
        std::vector<F> r0(sz, 0.0), r(sz, 0.0), p(sz, 0.0), vv(sz, 0.0), s(sz, 0.0), t(sz, 0.0);
        vector R0 = block(r0.data(), n, NV), R = block(r.data(), n, NV), P = block(p.data(), n, NV),
               V = block(vv.data(), n, NV), S = block(s.data(), n, NV), T = block(t.data(), n, NV);
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
        int it = 0;
        for (bool last = false; !last;) {
            it++;
            if (it >= max_iters) last = true;
            Ax(P, V);                                             // 5
            blas::dot<F, NV>(V, R0, S1);                          // 6
            blas::xdivy_z<F, NV>(Rho, S1, Al);
            blas::scal<F, NV>(a_1, Al);                           // 7
            blas::axpby_z<F, NV>(a1, R, Al, V, S);
            blas::scal<F, NV>(a_1, Al);
            Ax(S, T);                                             // 8
            blas::dot<F, NV>(T, S, S2);                           // 9
            blas::dot<F, NV>(T, T, S3);
            blas::dot<F, NV>(S, S, S4);
            blas::xdivy_z<F, NV>(S2, S3, Om);
            blas::ax_y<F, NV>(iconv, Al, Alc);                    // 10
            blas::ax_y<F, NV>(iconv, Om, Omc);
            blas::axpbypcz<F, NV>(Alc, P, Omc, S, a1, X);
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
    Bicgstab f{n, rp, ci, v, b, x, nv, max_iters, abs_tol, rel_tol, hist, hist_cap, 0};
    if (dispatch_nv(nv, f)) return -1;
    return f.iters;
}
}
