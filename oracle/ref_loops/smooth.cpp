// The Jacobi smoother's merged update of the reference
// (src/blas/detail/specific/blas_merged_jacobi.inl), compiled unchanged with
// the row loops' flags: like the Gauss-Seidel row update it is one product
// feeding one sum per entry, fused in the reference's FMA configuration.
#include "include_ref.h"
#include "ref_loops.h"

using namespace refloops;

namespace {

// Jacobi::solve's no-check path (jacobi.inl:91-100)
struct JacobiRun {
    int64_t n; const int *rp, *ci; const double *v, *invd, *b; double *x; const double *relax; int nv, sweeps;
    template <int NV> void run() {
        std::vector<double> r((size_t)n * NV, 0.0);
        vector X = block(x, n, NV), B = block(b, n, NV), R = block(r.data(), n, NV), D = block(invd, n, 1),
               W = scalars(relax, NV);
        for (int k = 0; k < sweeps; ++k) {
            ref_csr_ax_y_d(n, rp, ci, v, x, r.data(), NV);
            XAMG::blas::specific::merged_jacobi<double, NV>(X, B, D, R, W);
        }
    }
};

}  // namespace

extern "C" {
int ref_jacobi_d(int64_t n, const int *rp, const int *ci, const double *v, const double *invd,
                 const double *b, double *x, const double *relax, int nv, int sweeps) {
    JacobiRun f{n, rp, ci, v, invd, b, x, relax, nv, sweeps};
    return dispatch_nv(nv, f);
}
}
