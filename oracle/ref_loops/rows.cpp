// Row loops of the reference (sparse and dense products, Gauss-Seidel sweep),
// compiled unchanged.  The build compiles this file once with the reference's
// generic release flags and once with FMA contraction (the form its
// FMA-capable machine configurations compile to), see oracle/build_ref_loops.py.
#include "include_ref.h"
#include "ref_loops.h"

using namespace refloops;
using XAMG::mem::CORE;
using XAMG::mem::NUMA_NODE;

namespace {

template <class F> using Csr = XAMG::matrix::csr_matrix<F, int, int, int, int>;

// A CSR block of n rows over caller arrays (one core, all rows).
template <class F> Csr<F> csr(int64_t n, int64_t ncols, const int *rp, const int *ci, const F *v) {
    Csr<F> m;
    int64_t nnz = rp[n] - rp[0];
    m.row = block<int>(rp, n + 1, 1);
    m.col = block<int>(ci, nnz, 1);
    m.val = block<F>(v, nnz, 1);
    m.nrows = m.block_nrows = (uint64_t)n;
    m.ncols = m.block_ncols = (uint64_t)ncols;
    m.nonzeros = (uint64_t)nnz;
    m.if_empty = (n == 0);
    return m;
}

template <class F> struct AxY {
    int64_t n; const int *rp, *ci; const F *v, *x; F *y; int nv; bool acc;
    template <int NV> void run() {
        Csr<F> m = csr<F>(n, n, rp, ci, v);
        vector xv = block<F>(x, n, nv), yv = block<F>(y, n, nv);
        if (acc)
            XAMG::blas2::backend::csr_Axpy<F, int, int, int, int, NV>(m, xv, yv, nv);
        else
            XAMG::blas2::backend::csr_Ax_y<F, int, int, int, int, NV>(m, xv, yv, nv);
    }
};

// blas2::SGS with one core per block (see ref_loops.h).
template <class F> struct Hsgs {
    int64_t n; const int *rp, *ci; const F *v, *invd, *b; F *x; const F *relax; int nv, nb;
    const int64_t *bp;
    template <int NV> void run() {
        std::vector<int> blk(n);
        for (int q = 0; q < nb; ++q)
            for (int64_t i = bp[q]; i < bp[q + 1]; ++i) blk[i] = q;
        vector bv = block<F>(b, n, nv), xv = block<F>(x, n, nv), iv = block<F>(invd, n, 1),
               rv = block<F>(relax, 1, nv);
        std::vector<F> t((size_t)n * nv);
        vector tv = block<F>(t.data(), n, nv);
        // the diagonal blocks, block-local columns
        std::vector<std::vector<int>> drp(nb), dci(nb);
        std::vector<std::vector<F>> dv(nb);
        for (int q = 0; q < nb; ++q) {
            int64_t r0 = bp[q], r1 = bp[q + 1];
            drp[q].assign(1, 0);
            for (int64_t i = r0; i < r1; ++i) {
                for (int j = rp[i]; j < rp[i + 1]; ++j)
                    if (blk[ci[j]] == q) { dci[q].push_back((int)(ci[j] - r0)); dv[q].push_back(v[j]); }
                drp[q].push_back((int)dci[q].size());
            }
        }
        // t of every block from the incoming x: t = 0; t += A_offd(r) x for
        // each other block r in ascending order (global rows through the
        // block's row offset, x as the core-local received copy)
        std::vector<F> xold(x, x + (size_t)n * nv);
        vector xo = block<F>(xold.data(), n, nv);
        xo.sharing_mode = CORE;
        for (int q = 0; q < nb; ++q) {
            int64_t r0 = bp[q], r1 = bp[q + 1], nr = r1 - r0;
            vector tq = block<F>(t.data() + (size_t)r0 * nv, nr, nv);
            XAMG::blas::set_const<F, NV>(tq, 0.0, true);
            for (int r = 0; r < nb; ++r) {
                if (r == q) continue;
                std::vector<int> orp(1, 0), oci;
                std::vector<F> ov;
                for (int64_t i = r0; i < r1; ++i) {
                    for (int j = rp[i]; j < rp[i + 1]; ++j)
                        if (blk[ci[j]] == r) { oci.push_back(ci[j]); ov.push_back(v[j]); }
                    orp.push_back((int)oci.size());
                }
                if (oci.empty()) continue;
                Csr<F> m = csr<F>(nr, n, orp.data(), oci.data(), ov.data());
                m.block_row_offset = (uint64_t)r0;
                XAMG::blas2::backend::csr_Axpy<F, int, int, int, int, NV>(m, xo, tv, nv);
            }
        }
        for (int q = 0; q < nb; ++q) {
            int64_t r0 = bp[q], r1 = bp[q + 1], nr = r1 - r0;
            vector tq = block<F>(t.data() + (size_t)r0 * nv, nr, nv);
            vector bq = block<F>(b + (size_t)r0 * nv, nr, nv);
            XAMG::blas::axpby<F, NV>(1.0, bq, -1.0, tq);
        }
        for (int q = 0; q < nb; ++q) {
            int64_t r0 = bp[q], r1 = bp[q + 1];
            Csr<F> m = csr<F>(r1 - r0, r1 - r0, drp[q].data(), dci[q].data(), dv[q].data());
            m.block_row_offset = (uint64_t)r0;
            XAMG::blas2::backend::csr_SGS<F, int, int, int, int, NV>(m, iv, tv, xv, rv, nv);
        }
    }
};

template <class F> struct Dense {
    int64_t nr, nc; const F *m, *x; F *y; int nv;
    template <int NV> void run() {
        XAMG::matrix::dense_matrix<F> d;
        d.val = block<F>(m, nr * nc, 1);
        d.nrows = d.block_nrows = (uint64_t)nr;
        d.ncols = d.block_ncols = (uint64_t)nc;
        vector xv = block<F>(x, nc, nv), yv = block<F>(y, nr, nv);
        XAMG::blas2::backend::dense_Ax_y<F, NV>(d, xv, yv, nv);
    }
};

}  // namespace

extern "C" {
int ref_csr_ax_y_d(int64_t n, const int *rp, const int *ci, const double *v, const double *x,
                   double *y, int nv) {
    AxY<double> f{n, rp, ci, v, x, y, nv, false};
    return dispatch_nv(nv, f);
}
int ref_csr_ax_y_f(int64_t n, const int *rp, const int *ci, const float *v, const float *x,
                   float *y, int nv) {
    AxY<float> f{n, rp, ci, v, x, y, nv, false};
    return dispatch_nv(nv, f);
}
int ref_csr_axpy_d(int64_t n, const int *rp, const int *ci, const double *v, const double *x,
                   double *y, int nv) {
    AxY<double> f{n, rp, ci, v, x, y, nv, true};
    return dispatch_nv(nv, f);
}
int ref_csr_axpy_f(int64_t n, const int *rp, const int *ci, const float *v, const float *x,
                   float *y, int nv) {
    AxY<float> f{n, rp, ci, v, x, y, nv, true};
    return dispatch_nv(nv, f);
}
int ref_hsgs_d(int64_t n, const int *rp, const int *ci, const double *v, const double *invd,
               const double *b, double *x, const double *relax, int nv, int nb, const int64_t *bp) {
    Hsgs<double> f{n, rp, ci, v, invd, b, x, relax, nv, nb, bp};
    return dispatch_nv(nv, f);
}
int ref_hsgs_f(int64_t n, const int *rp, const int *ci, const float *v, const float *invd,
               const float *b, float *x, const float *relax, int nv, int nb, const int64_t *bp) {
    Hsgs<float> f{n, rp, ci, v, invd, b, x, relax, nv, nb, bp};
    return dispatch_nv(nv, f);
}
int ref_dense_ax_y_d(int64_t nr, int64_t nc, const double *m, const double *x, double *y, int nv) {
    Dense<double> f{nr, nc, m, x, y, nv};
    return dispatch_nv(nv, f);
}
int ref_dense_ax_y_f(int64_t nr, int64_t nc, const float *m, const float *x, float *y, int nv) {
    Dense<float> f{nr, nc, m, x, y, nv};
    return dispatch_nv(nv, f);
}
}
