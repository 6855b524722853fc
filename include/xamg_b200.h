/* Extension and kernel-level entry points of libxamg_b200.so.
 *
 * Part 1 (XAMG_b200_*) extends the XAMG C API with what the reference exposes
 * only through its C++ classes or its test driver: runtime NV, error text,
 * residual histories, hierarchy export, generators and the binary system
 * format.  Part 2 (xamg_*) is the device-pointer interface of the individual
 * solve-phase kernels; each entry names the reference routine whose
 * arithmetic it performs.  All pointers in part 2 are device pointers unless
 * the name says host; `stream` is a cudaStream_t (NULL = the library stream).
 * Precision codes: 0 = FP64, 1 = FP32.  nv must be one of 1, 2, 4, 8, 16, 32.
 */
#ifndef XAMG_B200_H_
#define XAMG_B200_H_

#include <stdint.h>
#include <stddef.h>
#include "xamg_c_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: API extensions ------------------------------------------- */

/* Set the right-hand-side width used by the NV-checked API calls
 * (replaces the reference's compile-time XAMG_NV, xamg_c_api.cpp:56-60). */
int XAMG_b200_set_nv(int nv);
/* Text of the last error returned by any call of this library. */
const char *XAMG_b200_last_error(void);
/* Wait for all queued device work of the library. */
int XAMG_b200_synchronize(void);
/* Kernels launched by this library since it was loaded (every launcher counts). */
long long XAMG_b200_kernel_launches(void);
/* CUDA-event timing of the hot kernels inside solves (an extension; off by
 * default, it adds two event records per timed launch): on = 1 starts
 * recording every Gauss-Seidel sweep and sparse product (class 1) with its
 * algorithmic bytes, on = 0 stops and discards; returns the previous state.
 * Sweep classes: 2 cooperative grid; hybrid blocks, one CTA per block:
 * 3 x tile in shared memory, 4 slot window, 5 x gathered per level; the same
 * with one warp per block: 6, 7, 8; 0 any other sweep path. */
int XAMG_b200_kernel_timing(int on);
/* Kernel of the hybrid Gauss-Seidel sweeps in this process: 1 one warp per
 * block, 0 one 256-thread CTA per block (XAMG_GS_SWEEP=warp|cta, read once;
 * both give identical results). */
int XAMG_b200_gs_sweep_kernel(void);
/* Waits for the device, then writes per (class, operator rows) the launch
 * count, total milliseconds and total algorithmic bytes of the records so far
 * (at most cap groups) and clears them; returns the number of groups, or a
 * negative error code. */
int XAMG_b200_kernel_timing_read(int cap, int *kclass, int64_t *rows, int64_t *launches, double *ms,
                                 double *bytes);
/* Raw device pointer of a device-resident vector (FP64, size x nv). */
void *XAMG_b200_vector_device_ptr(XAMG_vector_id vid);
/* Convergence detail of the last solve: squared residual norms after each
 * check (nv per entry, entry 0 = initial); returns the entry count. */
int XAMG_b200_solver_get_residual_history(double *out, int cap, XAMG_solver_id sid);
/* Squared initial residual norms (nv values) and per-column status. */
int XAMG_b200_solver_get_res0(double *out, XAMG_solver_id sid);
/* Device time of the last solve in milliseconds (CUDA events). */
double XAMG_b200_solver_last_solve_ms(XAMG_solver_id sid);
/* Multigrid hierarchy of a solver (levels from the host AMG setup). */
int XAMG_b200_solver_num_levels(XAMG_solver_id sid);
int XAMG_b200_solver_level_info(int64_t *info /* n, nnzA, ncolsP, nnzP, nlev_fwd, nlev_bwd */,
                                int level, XAMG_solver_id sid);
int XAMG_b200_solver_export_level(int *rpA, int *ciA, double *vA, int *rpP, int *ciP,
                                  double *vP, int level, XAMG_solver_id sid);
/* Gauss-Seidel wavefront levels of one level's pre-smoother (per row). */
int XAMG_b200_solver_export_gs_levels(int *lf, int *lb, int level, XAMG_solver_id sid);
/* Dense inverse of the coarsest operator (row-major n x n). */
int XAMG_b200_solver_export_coarse_inverse(double *out, XAMG_solver_id sid);
/* Spectrum bounds {min, max} of D^-1/2 A D^-1/2 used by a level's Chebyshev
 * smoother (the reference takes them from hypre, hypre_base.inl:370-375; here
 * they come from a 10-step CG/Lanczos estimate); {0, 0} without one. */
int XAMG_b200_solver_level_eig(double *out, int level, XAMG_solver_id sid);
/* Human-readable description of the solver tree. */
int XAMG_b200_solver_info(char *buf, int cap, XAMG_solver_id sid);

/* Generators.  kind 0: reference cube (examples/common/generator/cube.inl),
 * iargs = {nx, ny, nz, config}; kind 1: 27-point anisotropic, iargs = {n},
 * dargs = {kx, ky, kz}; kind 2: 7-point from face coefficients, iargs =
 * {nx, ny, nz}, faces = kx[(nx+1)ny nz] ky[nx(ny+1)nz] kz[nx ny(nz+1)]. */
/* The reference's channel-with-cube test system
 * (examples/common/generator/channel_with_cube.inl, geometry lame.inl) at
 * grid scale 1, 2 or 3: the operator into the csr matrix id and, when b_out
 * is not NULL, nv right-hand-side columns (rows x nv, row-major): all ones
 * when const_rhs, else the discrete divergence of the reference's
 * pseudo-random face velocities.  XAMG_b200_channel_cube_rows gives the rows
 * of a scale (-1 for other scales). */
int64_t XAMG_b200_channel_cube_rows(int scale);
int XAMG_b200_generate_channel_cube(int scale, int const_rhs, int nv, double *b_out, XAMG_csr_matrix_id id);
int XAMG_b200_csr_matrix_generate(int kind, const int64_t *iargs, const double *dargs,
                                  const double *faces, XAMG_csr_matrix_id mcsrid);
int64_t XAMG_b200_csr_matrix_get_nnz(XAMG_csr_matrix_id mcsrid);
int XAMG_b200_csr_matrix_export(int *rp, int *ci, double *v, XAMG_csr_matrix_id mcsrid);
/* Binary system file (examples/test/mtx_gen.cpp:116-146): matrix, then b and
 * x if present.  b_out/x_out may be NULL (host arrays of nrows doubles). */
int XAMG_b200_csr_matrix_read_bin(const char *path, double *b_out, double *x_out,
                                  XAMG_csr_matrix_id mcsrid);
int XAMG_b200_csr_matrix_write_bin(const char *path, const double *b, const double *x,
                                   XAMG_csr_matrix_id mcsrid);

/* Host-only AMG setup (the role of hypre BoomerAMG in hypre_base.h:121-217):
 * builds the hierarchy of the MultiGrid role of pid on the host, without any
 * device work.  info = {n, nnzA, ncolsP, nnzP}. */
int XAMG_b200_amg_host_create(XAMG_csr_matrix_id cid, XAMG_param_id pid, size_t *hid);
int XAMG_b200_amg_host_num_levels(size_t hid);
int XAMG_b200_amg_host_level_info(int64_t *info, int level, size_t hid);
int XAMG_b200_amg_host_export_level(int *rpA, int *ciA, double *vA, int *rpP, int *ciP,
                                    double *vP, int level, size_t hid);
int XAMG_b200_amg_host_destroy(size_t hid);
/* Wavefront levels of the sequential (block_rows = 0) or hybrid Gauss-Seidel
 * sweeps, computed on the host; nlev[2] = {forward, backward} level counts. */
int XAMG_b200_gs_levels_host(int64_t n, const int *rp, const int *ci, int64_t block_rows,
                             int *lf, int *lb, int *nlev);

/* Batching form.  These entry points have no counterpart in the reference.
 * nsys independent systems (host CSR arrays, int32 indices, FP64 values;
 * n[q] rows, nv[q] in {1,2,4,8,16,32} right-hand sides each) are solved
 * together by PBiCGStab (FP64 vectors, inner products and recurrences, one
 * set of scalars per system and column) preconditioned by AMG in FP32.  The
 * systems with equal nv form one block-diagonal group; pid supplies the
 * solver (max_iters, tolerances) and preconditioner/smoother roles.  The
 * SpMV kernel variant of each group is autotuned at creation.  A solve is one
 * CUDA-graph launch: every group's iteration runs inside a device-controlled
 * while loop, so no host round trip happens until all systems converge. */
int XAMG_b200_batch_create(int nsys, const int64_t *n, const int *const *rp, const int *const *ci,
                           const double *const *val, const int *nv, XAMG_param_id pid, size_t *bid);
/* b, x0: host arrays of n[sys] x nv[sys] doubles (row-major); x0 NULL = 0. */
int XAMG_b200_batch_upload(size_t bid, int sys, const double *b, const double *x0);
/* use_graph 0: the same steps launched from the host, one check per iteration. */
int XAMG_b200_batch_set_graph(size_t bid, int use_graph);
int XAMG_b200_batch_solve(size_t bid);
int XAMG_b200_batch_download(size_t bid, int sys, double *x);
/* per column: iterations at convergence (-1 = not converged) and the final
 * relative residual estimate of the recurrence */
int XAMG_b200_batch_stats(size_t bid, int sys, int *iters, double *relres);
double XAMG_b200_batch_last_ms(size_t bid);
/* kernels executed by the last batch solve (graph: init + iterations x body) */
long long XAMG_b200_batch_last_kernels(size_t bid);
/* groups: {nv, systems, FP64 SpMV variant, FP32 SpMV variant} each (cap ints
 * in out); returns the group count */
int XAMG_b200_batch_groups(size_t bid, int *out, int cap);
int XAMG_b200_batch_destroy(size_t bid);

/* ---- Row partition of one system (host side of a multi-GPU solve) ------- */
/* Rank `rank` of `nranks` owns the contiguous rows of the reference's block
 * partition (part.h: equal blocks, the remainder on the last).  rp/ci are the
 * HOST arrays of the whole system.  The local matrix keeps each owned row's
 * entries in CSR order with columns renumbered: owned columns first (global
 * column - first row), then the halo slots (rows owned by other ranks, in
 * ascending global order, hence grouped by owner), so a product over
 * [owned x | halo x] gives every row exactly the single-system bits.
 * info: out[0] first row, out[1] rows, out[2] local entries, out[3] halo slots.
 * local_csr: rows + 1 row pointers, the renumbered columns and (optional) the
 * global entry index of every local entry.  halo: global row and owner of
 * every halo slot.  sends: the owned rows (global) `peer` needs, in the order
 * of the peer's halo; *count alone when rows_out is NULL. */
int XAMG_b200_rowpart_create(int64_t n, const int *rp_host, const int *ci_host, int nranks, int rank,
                             size_t *id);
int XAMG_b200_rowpart_info(size_t id, int64_t *out);
int XAMG_b200_rowpart_local_csr(size_t id, int *rp_out, int *ci_out, int64_t *src_out);
int XAMG_b200_rowpart_halo(size_t id, int64_t *rows_out, int *owner_out);
int XAMG_b200_rowpart_sends(size_t id, int peer, int64_t *rows_out, int64_t *count);
int XAMG_b200_rowpart_destroy(size_t id);

/* Row-partitioned solve of one system over several GPUs, one rank per GPU
 * (an extension: the reference distributes with MPI, part.h,
 * matvec_comm.h:117-312, shm_allreduce.h:112-163).  Every rank uses the same
 * NCCL unique id (rank 0 makes it with XAMG_b200_dist_unique_id, 128 bytes,
 * and the caller broadcasts it), builds its row partition
 * (XAMG_b200_rowpart_create) and then the solver from the GLOBAL host values
 * (CSR order of the partitioned matrix) and a parameter list whose solver
 * role is BiCGStab or PBiCGStab; the preconditioner role runs on the rank's
 * diagonal block (block Jacobi across ranks).  Before each product the halo
 * rows are exchanged by NCCL send/receive into this GPU's memory; the inner
 * products of a step are summed by one NCCL allreduce.  With one rank the
 * iterations equal the single-GPU solver's bit for bit.  Solve: b and x are
 * device arrays of the rank's rows (rows x nv, row-major, FP64); x holds the
 * initial guess on entry.  Info: {iterations, all columns converged, rows,
 * history length}; history: squared residual norms, nv per check.  NCCL
 * (libnccl.so.2) is loaded when first needed. */
int XAMG_b200_dist_unique_id(void *out /* 128 bytes */);
int XAMG_b200_dist_create(const void *unique_id, size_t rowpart_id, const double *val_global_host,
                          XAMG_param_id pid, int nv, size_t *did);
int XAMG_b200_dist_solve(size_t did, const double *b_dev, double *x_dev);
int XAMG_b200_dist_info(size_t did, int64_t *out /* [4] */);
int XAMG_b200_dist_history(size_t did, double *out, int64_t cap);
int XAMG_b200_dist_destroy(size_t did);

/* ---- Part 2: kernel-level device interface ----------------------------- */

/* csr_Ax_y / csr_Axpy (blas2/detail/csr_matvec.inl:32-260):
 * mode 0: y = A x; 1: y += A x; 2: y = b - A x. */
int xamg_csr_spmv(int prec, int nv, int64_t n, const int *rp, const int *ci, const void *val,
                  const void *x, void *y, int mode, const void *b, void *stream);
/* Kernel variant used by every CSR product of the library (same results):
 * 0, 1, 2 = one CTA per row tile with x gathers issued 4, 8 or 16 entries at
 * a time; 3, 4 = the tile's entries staged in shared memory, gathers 4 or 8 at
 * a time; 5, 6 = staged entries with a plain row loop unrolled 4 or 8 times;
 * 10 + k = staged streaming kernel walking k tiles per CTA; -1 = default (6
 * when nv * element size >= 64 bytes, else 0).  Under -1 and 7 the products
 * of operators that have a shifted-row run plan (below) use the run kernel
 * (7 elsewhere = the default).  The setting belongs to the calling host
 * thread; a batch's autotuned choices are held by its own operators and are
 * not affected by it.  Returns the previous setting. */
int xamg_spmv_set_variant(int variant);

/* Shifted-row run SpMV (no counterpart in the reference; the same results as
 * xamg_csr_spmv, bit for bit).  The plan groups the rows into chunks of up to
 * `rows` (4 or 8) consecutive rows whose column indices are the first row's
 * shifted by the row offset, ci(r0+q, e) = ci(r0, e) + q (the interior rows
 * of stencil operators), and stores the values chunk-interleaved; for a run
 * of up to 3 consecutive columns the chunk's rows gather the x rows they
 * share once (len + rows - 1 gathers instead of len * rows).  Every row lies in some chunk (irregular rows in
 * chunks of one), so a plan serves any square matrix.  rp/ci/val are HOST
 * arrays; values are kept in FP64 and, when fp32 != 0, in FP32.  Shapes with
 * nv * element size >= 64 bytes (FP64 nv 8, 16, 32; FP32 nv 16, 32).
 * Matrices constructed through the C API get a plan (rows set by
 * xamg_spmv_set_run_rows, default 8, 0 = none) when they have at least 4096
 * rows and half of their entries lie in full chunks.
 * plan_info (any output may be NULL): chunk count, fraction of the entries
 * in full chunks, segments (runs of at most 3 consecutive columns of each
 * chunk's first row, summed over the chunks) and stored value slots (entries
 * times rows per chunk, padding included). */
void *xamg_spmv_runs_plan_create(int64_t n, const int *rp_host, const int *ci_host,
                                 const double *val_host, int rows, int fp32);
int xamg_spmv_runs_plan_info(void *plan, int64_t *nchunks, double *coverage, int64_t *segments,
                             int64_t *value_slots);
/* The run detection alone, on the host (no device work): what plan_info
 * would report for a plan of these HOST arrays. */
int xamg_spmv_runs_analyze(int64_t n, const int *rp_host, const int *ci_host, int rows, int64_t *nchunks,
                           double *coverage, int64_t *segments);
int xamg_spmv_runs(void *plan, int prec, int nv, const void *x, void *y, int mode, const void *b,
                   void *stream);
int xamg_spmv_runs_plan_destroy(void *plan);
int xamg_spmv_set_run_rows(int rows);
/* Kernel form of the run products of the calling host thread: 0 (default)
 * gathers each segment's x rows into registers, 1 copies them into shared
 * memory one segment ahead (cp.async, fewer registers, two segments in
 * flight).  Same results.  Returns the previous setting. */
int xamg_spmv_set_run_form(int form);

/* Gauss-Seidel plan (wavefront schedule) for blas2::SGS / csr_SGS
 * (blas2.h:184-281, csr_gs.inl:32-134).  rp/ci are HOST arrays.  block_rows
 * = 0 gives the single-process sweep; > 0 the hybrid block semantics.
 * schedule: 0 = one launch per wavefront level; 1 = automatic (one
 * cooperative launch per sweep with a bounded grid barrier per level, or one
 * CTA per block for hybrid plans); 2 = cooperative grid sweep always. */
void *xamg_gs_plan_create(int64_t n, const int *rp_host, const int *ci_host,
                          int64_t block_rows, int schedule);
/* Give the plan the matrix values (HOST array, CSR order of rp/ci): sweeps in
 * precision prec then run over the plan's level-ordered copy of the matrix
 * with TMA-staged entries (schedules 1 and 2); the val argument of xamg_hsgs
 * is still used for the hybrid right-hand side. */
int xamg_gs_plan_set_values(void *plan, const double *val_host, int prec);
int xamg_gs_plan_levels(void *plan, int *nlev /* [2] */, int *lf, int *lb);
/* Self-test of the device-side bounded waits (an extension): makes a wait
 * run out on purpose with a limit of limit_s seconds (at most 2) and reports
 * it the way a solve does, code 3 with the message in XAMG_b200_last_error.
 * which = 0: cooperative grid of ncta (2..64) CTAs whose barrier misses one
 * arrival; 1: an mbarrier phase that nothing completes.  The device stays
 * usable afterwards. */
int XAMG_b200_wait_selftest(int which, int ncta, double limit_s);
/* Slots of the shared-memory x window of each sweep direction of a hybrid
 * plan with values (0: no window; the window is used when slots * nv * the
 * value size <= 64 KB and the block's x tile does not fit in shared memory). */
int xamg_gs_plan_slots(void *plan, int *nslots /* [2] */);
int xamg_gs_plan_error(void *plan);
void xamg_gs_plan_destroy(void *plan);
/* One HSGS call: t = b - A_offblock x (when hybrid), forward then backward
 * sweep updating x in place.  relax: nv values of the solver precision.
 * t_scratch: n*nv elements (needed only when block_rows > 0). */
int xamg_hsgs(void *plan, int prec, int nv, const int *rp, const int *ci, const void *val,
              const void *invdiag, const void *b, void *x, const void *relax, void *t_scratch,
              void *stream);

/* Jacobi sweep (merged_jacobi, blas_merged_jacobi.inl:61-81): xo = xi +
 * relax*invdiag*(b - A xi). */
int xamg_jacobi(int prec, int nv, int64_t n, const int *rp, const int *ci, const void *val,
                const void *invdiag, const void *b, const void *xi, void *xo,
                const void *relax, void *stream);

/* Inner products (blas::dot, blas.inl:521-589) of nd pairs (1..4), FP64
 * results out[d*nv + k]; part: xamg_dot_part_size(n, nd, nv) doubles of scratch. */
int64_t xamg_dot_part_size(int64_t n, int nd, int nv);
/* Inner products of the batching form (batch.cu k_segdot1/2), per segment of
 * concatenated vectors: segment s holds rows [segoff[s], segoff[s + 1]) (host
 * array of nseg + 1 offsets from 0); out (device, nd * nseg * nv doubles)
 * receives at [d * nseg * nv + s * nv + k] exactly what xamg_dot returns for
 * that segment's rows alone.  a, b: nd (1..3) device vectors each.  Allocates
 * its own scratch and returns after the device has finished. */
int xamg_seg_dot(int prec, int nv, int nseg, const int64_t *segoff, int nd, const void *const *a,
                 const void *const *b, double *out, void *stream);
int xamg_dot(int prec, int nv, int64_t n, int nd, const void *const *a, const void *const *b,
             double *part, double *out, void *stream);

/* Allocation-free inner products (nd = 1..4 pairs).  This entry point has no
 * counterpart in the reference.  It returns exactly what xamg_dot returns, for callers that
 * cannot allocate device memory when they need the result (a plug-in that is
 * handed only its input and output buffers, a latency-critical loop where
 * cudaMalloc's implicit synchronisation is not acceptable): the partial sums
 * go to an 8 MiB array that is part of the library's device image, held on
 * every GPU that loads the library until the process exits.  Limit:
 * xamg_dot_part_size(n, nd, nv) <= 1048576, else code 2 and nothing runs.
 * All calls share that array, so calls that overlap on the GPU race; calls on
 * one stream are safe.  The first call in a CUDA context looks up the array's
 * address with that context current; make it before any stream capture.
 * stream NULL means the library's own stream, as for xamg_dot. */
int xamg_dot_noalloc(int prec, int nv, int64_t n, int nd, const void *const *a,
                     const void *const *b, double *out, void *stream);

/* Block-vector BLAS-1 (blas.inl, blas_ext.inl) with FP64 per-column scalars:
 * op 0 z=a*x+b*y, 1 z=a*x+b*y+c*z, 2 z=a*x, 3 z=x, 4 z=a, 5 z=z*x,
 * 6 z[i,k] = z[i,k]*x[i] (x: n values, one per row). */
int xamg_blas(int prec, int nv, int64_t n, int op, const double *a, const void *x,
              const double *b, const void *y, const double *c, void *z, void *stream);

/* Dense coarse solve y = Ainv b (Direct, dense_matvec.inl:71-121) with the
 * inverse stored transposed (AinvT[j*n + i] = Ainv[i][j]). */
int xamg_dense_gemv(int prec, int nv, int n, const void *AinvT, const void *b, void *y,
                    void *stream);

#ifdef __cplusplus
}
#endif

#endif /* XAMG_B200_H_ */
