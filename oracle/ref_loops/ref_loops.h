// C entry points of the reference-loop library (oracle/_ref/libxamg_ref_loops_*.so):
// each wraps one of the reference's own loop templates, compiled unchanged
// from its source files, over caller-owned arrays.  Test infrastructure only:
// the tests compare the oracle with these, never the product.
//
// Block vectors are row-major, x[i*nv + k]; nv must be one of 1, 2, 4, 8, 16,
// 32 (the template widths instantiated); entry points return 0, or -1 for an
// unsupported nv.  CSR arrays are int32 (the benchmark's index type).
#pragma once
#include <cstdint>

extern "C" {

// csr_Ax_y, src/blas2/detail/csr_matvec.inl:148-260 (y = A x)
int ref_csr_ax_y_d(int64_t n, const int *rp, const int *ci, const double *v, const double *x,
                   double *y, int nv);
int ref_csr_ax_y_f(int64_t n, const int *rp, const int *ci, const float *v, const float *x,
                   float *y, int nv);
// csr_Axpy, csr_matvec.inl:32-144 (y += A x)
int ref_csr_axpy_d(int64_t n, const int *rp, const int *ci, const double *v, const double *x,
                   double *y, int nv);
int ref_csr_axpy_f(int64_t n, const int *rp, const int *ci, const float *v, const float *x,
                   float *y, int nv);
// One hybrid symmetric Gauss-Seidel call as blas2::SGS (src/blas2/blas2.h:184-281)
// runs it with one core per row block [bp[q], bp[q+1]): t = 0, t += (entries of
// each other block, ascending) x by csr_Axpy, t = 1*b + (-1)*t, then csr_SGS
// (src/blas2/detail/csr_gs.inl:32-134) on the block's own entries.  The t of
// every block is formed from the incoming x before any block sweeps.
int ref_hsgs_d(int64_t n, const int *rp, const int *ci, const double *v, const double *invd,
               const double *b, double *x, const double *relax, int nv, int nb, const int64_t *bp);
int ref_hsgs_f(int64_t n, const int *rp, const int *ci, const float *v, const float *invd,
               const float *b, float *x, const float *relax, int nv, int nb, const int64_t *bp);
// dense_Ax_y, src/blas2/detail/dense_matvec.inl:71-121 (y = M x, M n_r x n_c row-major)
int ref_dense_ax_y_d(int64_t nr, int64_t nc, const double *m, const double *x, double *y, int nv);
int ref_dense_ax_y_f(int64_t nr, int64_t nc, const float *m, const float *x, float *y, int nv);

// The reference's channel-with-cube generator
// (examples/common/generator/channel_with_cube.inl:40-245, grid scale 1-3,
// constant or divergence right-hand sides, one process): returns the row
// count and *nnz; copies the CSR arrays (entries in the generator's own
// order) and the n x nv right-hand sides into every non-null output.
int64_t ref_channel_cube_d(int scale, int const_rhs, int nv, int64_t *nnz, int *rp, int *ci, double *v,
                           double *b);

// The reference's binary system reader (src/io/detail/reader.inl:30-180,
// read_system, one process): row count, *nnz, and into non-null outputs the
// CSR arrays and the n x nv b and x it reads.
int64_t ref_read_system_d(const char *path, int nv, int64_t *nnz, int *rp, int *ci, double *v, double *b,
                          double *x);

// The reference's cube generator (examples/common/generator/cube.inl:71-225,
// configurations 0-4, one process): row count, *nnz and, into non-null
// outputs, the CSR arrays (diagonal first, then its neighbour order).
int64_t ref_cube_d(int64_t nx, int64_t ny, int64_t nz, int config, int64_t *nnz, int *rp, int *ci,
                   double *v);

// BLAS-1 (src/blas/detail/blas.inl, blas_ext.inl) over n rows; a, b, c are
// per-column scalars (nv values).
int ref_dot_d(int64_t n, int nv, const double *x, const double *y, double *res);      // blas.inl:521-589
int ref_axpby_d(int64_t n, int nv, const double *a, const double *x, const double *b,
                double *y);                                                          // blas.inl:89-151
int ref_axpby_z_d(int64_t n, int nv, const double *a, const double *x, const double *b,
                  const double *y, double *z);                                       // blas_ext.inl:30-102
int ref_axpbypcz_d(int64_t n, int nv, const double *a, const double *x, const double *b,
                   const double *y, const double *c, double *z);                     // blas_ext.inl:106-189
int ref_xdivy_z_d(int64_t n, int nv, const double *x, const double *y, double *z);    // blas_ext.inl:193-239
int ref_ax_y_d(int64_t n, int nv, const double *a, const double *x, double *y);       // blas.inl:30-85
int ref_scal_d(int64_t n, int nv, const double *a, double *y);                        // blas.inl:155-219

// Jacobi smoother, the no-check path of Jacobi::solve (jacobi.inl:91-100):
// `sweeps` times r = A x, then blas_merged_jacobi.inl:32-90
// (x += relax_k * invd_i * (b - r)).
int ref_jacobi_d(int64_t n, const int *rp, const int *ci, const double *v, const double *invd,
                 const double *b, double *x, const double *relax, int nv, int sweeps);

// The Chebyshev smoother (src/solvers/detail/chebyshev.inl: its coefficient
// table and Chebyshev::solve, compiled unchanged) applied once to x with the
// given spectrum bounds of D^-1/2 A D^-1/2.
int ref_chebyshev_d(int64_t n, const int *rp, const int *ci, const double *v, const double *b, double *x, int nv,
                    int order, double fraction, double min_eig, double max_eig);

// Gauss-Jordan inverse of a dense n x n matrix (row-major),
// src/primitives/matrix/operations/inverse.inl:31-106 (the coarse-grid
// Direct solver's setup)
int ref_dense_inverse_d(int64_t n, const double *a, double *ainv);
int ref_dense_inverse_f(int64_t n, const float *a, float *ainv);

// The multigrid preconditioner of the solver classes: one cycle of the
// reference's loops in its MG_cycle order (mg.inl:186-280) over a hierarchy
// given per level l: nrows[l] rows, the operator (arp, aci, av), P_l
// (nrows[l] x nrows[l+1]: prp, pci, pv) and R_l = P_l^T (rrp, rci, rv), hybrid
// blocks nb[l] with offsets bp[l]; HSGS (smoother & 15 = 0, the sweep above)
// or Jacobi (1) with relax and pre_it / post_it sweeps, (smoother >> 4) & 15 =
// mg_cycle (0 V, 1 F, 2 W), bit 8 = mg_reduced_precision (FP32 below the
// first level, HSGS only); the coarsest level by the reference's Gauss-Jordan
// inverse (FP64, or FP32 when reduced) and dense product.  Applied as one
// cycle from the x given (MultiGrid::solve with max_iters 1), then destroyed.
void *ref_hier_create(int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                      const double *const *av, const int *const *prp, const int *const *pci,
                      const double *const *pv, const int *const *rrp, const int *const *rci,
                      const double *const *rv, const int *nb, const int64_t *const *bp, double relax, int pre_it,
                      int post_it, int smoother);
int ref_hier_apply_d(void *h, const double *b, double *x, int nv);
void ref_hier_destroy(void *h);

// The reference's MultiGrid class (mg.inl) with its HSGS / Jacobi smoother
// classes (hsgs.inl, jacobi.inl), compiled unchanged (mg.cpp), over a
// hierarchy given as for ref_hier_create; applied as MultiGrid::solve with
// max_iters 1 (the preconditioner role) from the x given.
void *ref_mg_create(int nv, int nlev, const int64_t *nrows, const int *const *arp, const int *const *aci,
                    const double *const *av, const int *const *prp, const int *const *pci, const double *const *pv,
                    const int *const *rrp, const int *const *rci, const double *const *rv, const int *nb,
                    const int64_t *const *bp, double relax, int pre_it, int post_it, int smoother);
int ref_mg_apply_d(void *h, const double *b, double *x);
void ref_mg_destroy(void *h);
// Chebyshev smoothing (chebyshev.inl, order and spectrum_fraction, the given
// spectrum bounds per level) in place of the object's smoothers.
void ref_mg_set_chebyshev(void *h, int order, double fraction, const double *min_eig, const double *max_eig);

// The reference's own solver classes compiled unchanged (krylov.cpp):
// method 0 BiCGStab (bicgstab.inl), 1 PBiCGStab (pbicgstab.inl), 2 PCG
// (pcg.inl), 3 RBiCGStab (rbicgstab.inl), 4 MergedBiCGStab, 5
// MergedPBiCGStab (merged/*.inl); the preconditioned ones use hier (from
// ref_hier_create, or from ref_mg_create when method has bit 4 (16) set;
// PCG and RBiCGStab the identity when hier is null), from
// x = 0, to max(abs_tol, rel_tol * initial residual) per column.  hist
// receives the (iterations + 1) x nv squared residual norms the solver
// checks; returns the iteration count (-1 on bad input).
int ref_solver_d(int method, void *hier, int64_t n, const int *rp, const int *ci, const double *v,
                 const double *b, double *x, int nv, int max_iters, double abs_tol, double rel_tol,
                 double *hist, int hist_cap);
}
