// The reference's Chebyshev smoother (src/solvers/detail/chebyshev.inl),
// the solver class compiled unchanged against the stand-ins of
// solver_base.h: its polynomial coefficients (Chebyshev_polynomial_coeffs)
// and the application of the polynomial in D^{-1/2} A D^{-1/2}
// (Chebyshev::solve).
#include "solver_base.h"
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
        s.param_list.v["polynomial_order"] = order;
        s.param_list.v["spectrum_fraction"] = fraction;
        s.run(3);
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
