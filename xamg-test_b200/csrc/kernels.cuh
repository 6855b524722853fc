// Device kernels of the XAMG solve phase (sm_100a).  Host-callable launchers.
//
// Data layout (same as the reference, csr_matvec.inl:224-229):
//   block vectors are row-major N x NV: element (i, k) at x[i*NV + k];
//   CSR matrices use int32 row pointers and column indices and FP64 or FP32
//   values; per-column scalars (alpha, omega, ...) are NV doubles on device.
// Arithmetic contract (identical to the CPU oracle, bit for bit):
//   * CSR/dense row sums: acc = fma(a_ij, x_j, acc) in stored order;
//   * Gauss-Seidel: sum = fma(-a_ij, x_j, sum); x_i = fma(relax*invdiag_i, sum, x_i);
//   * BLAS-1: literal left-to-right evaluation, every product rounded;
//   * inner products: the fixed chunk/lane/slot tree (see dot kernels).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

typedef int64_t i64;

namespace xk {

enum class Prec : int { F64 = 0, F32 = 1 };

// Count of kernels this library has launched (every launcher adds its own).
void note_launch(int k = 1);
long long launch_count();

// ---- sparse matrix-vector products ---------------------------------------
// y = A x (mode 0), y += A x (mode 1), y = b - A x (mode 2, b given).
// variant >= 0 picks the kernel (see set_spmv_variant) for this call only;
// -1 uses the calling thread's setting.
void spmv(Prec p, int nv, i64 n, const int *rp, const int *ci, const void *val, const void *x,
          void *y, int mode, const void *b, cudaStream_t s, int variant = -1);
// Kernel variant for spmv(): 0, 1, 2 = one CTA per row tile with gather
// batches of 4, 8, 16 entries; 3, 4 = tile-staged entries (shared memory) with
// gather batches of 4, 8; 5, 6 = tile-staged with a plain row loop unrolled 4,
// 8 times; 10 + k = streaming kernel walking k tiles per CTA; -1 = default
// (6 when NV*sizeof(T) >= 64 bytes, else 0).  All give identical results.
// Operators with a shifted-row run plan use the run kernel under -1 and 7
// (7 elsewhere = the default).  The setting is per host thread; an operator
// can also carry its own choice (DCsr::variant), which takes precedence.
void set_spmv_variant(int v);
int get_spmv_variant();
// Rows per chunk of the run plans built when operators are uploaded (8; 0 =
// build no run plans).
void set_spmv_run_rows(int r);
int get_spmv_run_rows();

// ---- shifted-row runs (stencil-structured operators) ------------------------
// Chunks of up to 8 consecutive rows whose column indices are the first row's
// shifted by the row offset; chunks[c] = {r0, cnt, m, segments}, four chunks
// per tile (ntiles tiles; toff has ntiles + 1 entries {value offset, segment
// offset}, both multiples of 4).  Tile t's segments (runs of at most 3
// consecutive columns of each chunk's first row, c0 | len << 30) at
// sg[toff[t].y + 4s + slot], its values at vt[(toff[t].x + 4e + slot) * 8 + q].
// Same modes and the same results, bit for bit, as spmv().  FP64 nv 8, 16, 32
// and FP32 nv 16, 32.
bool spmv_runs_supported(Prec p, int nv);
// kernel form of the run product (per host thread): 0 = each segment's x rows
// gathered into registers, 1 = copied into shared memory one segment ahead
void set_spmv_run_form(int f);
int get_spmv_run_form();
void spmv_runs(Prec p, int nv, i64 nchunks, i64 ntiles, const int4 *chunks, const longlong2 *toff, const int *sg,
               const void *vt, const void *x, void *y, int mode, const void *b, cudaStream_t s);

// ---- Gauss-Seidel sweeps ----------------------------------------------------
// One wavefront level: rows[0..cnt) are independent and updated in place.
// brows > 0 restricts each row to the columns of its own hybrid block
// [ (i/brows)*brows, +brows ); brows == 0 uses the whole row.
void gs_level(Prec p, int nv, int cnt, const int *rows, const int *rp, const int *ci,
              const void *val, const void *invd, const void *t, void *x, const void *relax,
              i64 brows, cudaStream_t s);

// Whole sweep inside one cooperative persistent launch; level l covers
// perm[lptr[l] .. lptr[l+1]).  Waits between levels are bounded: on timeout
// *err is set and the kernel returns early.
cudaError_t gs_sweep_persistent(Prec p, int nv, int nlev, const int *lptr, const int *perm,
                                const int *rp, const int *ci, const void *val, const void *invd,
                                const void *t, void *x, const void *relax, i64 brows,
                                unsigned *bar, int *err, cudaStream_t s);

// Hybrid Gauss-Seidel with one CTA per block of brows rows: forward and
// backward sweeps of every block inside one launch, CTA barriers only.  Block
// b owns levels [blev[b], blev[b+1]) of lptr; level l covers perm[lptr[l]..lptr[l+1]).
void gs_blocks(Prec p, int nv, int nblocks, const int *blevf, const int *lptrf, const int *permf,
               const int *blevb, const int *lptrb, const int *permb, const int *rp, const int *ci,
               const void *val, const void *invd, const void *t, void *x, const void *relax,
               i64 brows, cudaStream_t s);

// Sweep over a level-ordered copy of the matrix (gs.cu).  mode 0: ncta CTAs
// share every level with a bounded grid barrier (cooperative launch); mode 1:
// CTA b owns hybrid block b (ncta blocks).  desc holds one int4 {r0, r1, e0,
// e1} per (level, CTA): mode 0 at [l*ncta + b], mode 1 at [blev[b] + l].
// lrow/invd are in level order (lrow = -1 marks padding rows).  xs = 1 keeps
// the block's x tile in shared memory (mode 1, brows*nv*sizeof(T) <=
// gs_lcsr_max_xs_bytes()).  Mode 0 uses the first 256 bytes of gbar
// (8-byte aligned) for the grid barrier and zeroes them before the launch;
// err must lie outside them.  emax: the most entries any CTA processes in one
// level (sizes the shared-memory gather buffer; <= 0 = unknown).
//
// Slot window of a BLOCKS sweep whose x tile does not fit (win may be null):
// lci then holds slot numbers instead of columns, lslot gives each
// level-ordered row's slot, and ld holds {row, slot} pairs: for level group g
// the range ldd[g] = {first, end} lists the rows first used kGsSlotAhead
// levels after g, ldpre[b] those first used in block b's first kGsSlotAhead
// levels (each range starts at an even index and has an even length, padded
// with {-1, -1}).  Used when nslots * nv * sizeof(T) <= gs_slot_window_bytes()
// and a row of x is a multiple of 16 bytes; otherwise the level gathers.
constexpr int kGsSlotAhead = 4;
struct GsSlotWin {
    const int *lslot;
    const int2 *ldd, *ldpre, *ld;
    int nslots;
};
// Point-to-point waits of a GRID sweep (deps may be null: a grid barrier
// after every level): CTA b publishes at prog[b * 8] the number of levels it
// has finished; before level l it waits for deps[dptr[l*ncta + b] ..
// dptr[l*ncta + b + 1]) = {cta, levels that CTA must have finished}.  prog
// holds ncta * 8 words and is zeroed by the launcher.
struct GsDeps {
    const int *dptr;
    const int2 *deps;
    unsigned *prog;
};
cudaError_t gs_sweep_lcsr(Prec p, int nv, int mode, int xs, int nlev, int ncta, const int *lev_row,
                          const int *blev, const int *lrp, const int *lci, const void *lva,
                          const int *lrow, const void *invd, const void *t, void *x,
                          const void *relax, i64 brows, i64 n, unsigned *gbar, int *err,
                          int emax, const GsSlotWin *win, const GsDeps *deps, cudaStream_t s);
// Hybrid sweep with one warp per block (gsw.cu): same arrays and results as
// gs_sweep_lcsr mode 1.  gsw_shape picks the x form (xm 1 tile, 2 slot
// window, 0 per-level gather; -1 none fits) and the record stages for the
// plan's extremes: emax entries, rmax rows (rounded out to 4) and nlmax
// window loads in one level of one block, lmax levels in one block.
struct GswShape {
    int xm = -1, ns = 0, recb = 0, xoff = 0;
    size_t smem = 0;
};
GswShape gsw_shape(int s, int nv, int nblocks, int sms, i64 brows, int nslots, int emax, int rmax, int lmax,
                   int nlmax);
cudaError_t gs_sweep_warp(Prec p, int nv, const GswShape &z, int nblocks, const int *desc, const int *blev,
                          const int *lrp, const int *lci, const void *lva, const int *lrow, const void *invd,
                          const void *t, void *x, const void *relax, i64 brows, i64 n, const GsSlotWin *win,
                          int lmax, cudaStream_t s);
// Bounded-wait self-test (which 0: grid barrier with one CTA missing; 1:
// mbarrier phase that nothing completes), limit in ns; words: 256 bytes of
// device scratch, err: one device int (0 after a wait that did not run out).
cudaError_t wait_selftest(int which, int ncta, unsigned long long limit_ns, unsigned *words, int *err,
                          cudaStream_t s);
int gs_lcsr_max_xs_bytes();
int gs_lcsr_xs_bytes_two_per_sm();
int gs_slot_window_bytes();

// Hybrid Gauss-Seidel right-hand side: t = 1*b + (-1)*(sum over the entries
// outside the row's block of a_ij x_j)   (blas2.h:226-259)
void offblock_resid(Prec p, int nv, i64 n, const int *rp, const int *ci, const void *val,
                    const void *b, const void *x, void *t, i64 brows, cudaStream_t s);

// ---- Jacobi ---------------------------------------------------------------
// xo = fma(relax_k * invd_i, b - A xi, xi)   (xi, xo distinct)
void jacobi(Prec p, int nv, i64 n, const int *rp, const int *ci, const void *val,
            const void *invd, const void *b, const void *xi, void *xo, const void *relax,
            cudaStream_t s);

// ---- dense coarse solve: y = Ainv b, AinvT stored transposed (n x n) --------
void dense_gemv(Prec p, int nv, int n, const void *AinvT, const void *b, void *y, cudaStream_t s);

// ---- inner products -------------------------------------------------------
// nd (1..4) pairs (a_d, b_d) of N x NV vectors (element type `in`), FP64
// results out[d*nv + k].  part must hold dot_part_size(n, nd, nv) doubles.
i64 dot_part_size(i64 n, int nd, int nv);
// Order of the inner products of dots / dot_partials on this host thread:
// the fixed tree (default) or the reference's single-core sequential order
// (k_dot_seq; same partial layout, so the reduction stages are unchanged).
void set_dot_sequential(bool on);
bool dot_sequential();
struct DotOrderScope {
    bool prev;
    explicit DotOrderScope(bool seq) : prev(dot_sequential()) { set_dot_sequential(seq); }
    ~DotOrderScope() { set_dot_sequential(prev); }
};
void dots(Prec in, int nv, i64 n, int nd, const void *const *a, const void *const *b,
          double *part, double *out, cudaStream_t s);

// ---- fused BiCGStab groups (one pass each, bits of the separate kernels) ---
// Per-column device scalars of one (P)BiCGStab solve (nv doubles each).
struct BicgScalars {
    double *rho, *alpha, *omega, *beta, *c1, *ac, *oc, *res, *iconv, *status, *tol;
    int check;  // 1: update status/iconv from res and tol in the omega stage
};
// first stage of dots() alone: chunk partials of nd pairs into part
void dot_partials(Prec in, int nv, i64 n, int nd, const void *const *a, const void *const *b, double *part,
                  cudaStream_t s);
// second stage for nd pairs of every column (out[d*nv + k]) followed by the
// scalar recurrence epi: 0 alpha = rho/out0; 1 omega = out0/out1, res =
// out2 - omega*out0, ac/oc = iconv*alpha/omega, convergence status and the
// next iconv; 2 beta = (out0/rho)(alpha/omega), rho = out0, c1 = -(omega*beta)
void dot_reduce_epi(int epi, i64 n, int nd, int nv, const double *part, double *out, const BicgScalars &sc,
                    cudaStream_t s);
// the same recurrences from already reduced values vals[d*nv + k] (after an
// allreduce over ranks), and the second stage alone (no recurrence)
void bicg_epi(int epi, int nv, const double *vals, const BicgScalars &sc, cudaStream_t s);
void dot_reduce(i64 n, int nd, int nv, const double *part, double *out, cudaStream_t s);
// dst row q = src row idx[q] of N x nv block vectors (halo send buffers)
void gather_rows(Prec p, int nv, i64 cnt, const int *idx, const void *src, void *dst, cudaStream_t s);
// s = r - alpha v (blas AXPBY_Z with 1 and -alpha); sz = 0 when given
void bicg_s(Prec p, int nv, i64 n, const BicgScalars &sc, const void *r, const void *v, void *s_out, void *sz,
            cudaStream_t s);
// p = r + c1 v + beta p (blas AXPBYPCZ); pz = 0 when given
void bicg_p(Prec p, int nv, i64 n, const BicgScalars &sc, const void *r, const void *v, void *pv, void *pz,
            cudaStream_t s);
// x = ac pp + oc ss + x; r = s - omega t; chunk partials of (r, r0) into part
void bicg_xr(Prec p, int nv, i64 n, const BicgScalars &sc, const void *pp, const void *ss, void *x, const void *sv,
             const void *t, void *r, const void *r0, double *part, cudaStream_t s);

// ---- BLAS-1 (element type T, FP64 per-column scalars) ---------------------
enum class Op : int {
    AXPBY_Z = 0,   // z = a*x + b*y
    AXPBYPCZ = 1,  // z = a*x + b*y + c*z
    AX_Y = 2,      // z = a*x
    COPY = 3,      // z = x
    SET = 4,       // z = a
    SCAL_XY = 5,   // z = z * x   (elementwise)
    ROW_SCAL = 6,  // z[i,k] = z[i,k] * x[i]  (x: one value per row; blas::scal, blas.inl:182-189)
};
void blas(Prec p, int nv, i64 n, Op op, const double *a, const void *x, const double *b,
          const void *y, const double *c, void *z, cudaStream_t s);

// constant fill with a host value (set_const with a scalar)
void fill(Prec p, i64 count, double v, void *z, cudaStream_t s);
// element conversion
void convert(Prec from, Prec to, i64 count, const void *x, void *y, cudaStream_t s);

// ---- BiCGStab scalar recurrences (one thread per column, FP64) -------------
// alpha = rho / s1
void bicg_alpha(int nv, const double *rho, const double *s1, double *alpha, cudaStream_t s);
// omega = s2/s3; res = 1*s4 + (-1)*(omega*s2); ac = iconv*alpha; oc = iconv*omega
void bicg_omega(int nv, const double *s2, const double *s3, const double *s4,
                const double *alpha, const double *iconv, double *omega, double *res,
                double *ac, double *oc, cudaStream_t s);
// beta = (s1/rho)*(alpha/omega); rho = s1; c1 = -(omega*beta); also -alpha, -omega
void bicg_beta(int nv, const double *s1, double *rho, const double *alpha, const double *omega,
               double *beta, double *c1, cudaStream_t s);
// PCG: alpha = s1/s2; ac = iconv*alpha; nalpha = -1*alpha
void pcg_alpha(int nv, const double *s1, const double *s2, const double *iconv, double *alpha, double *ac,
               double *nalpha, cudaStream_t s);
// RBiCGStab: alpha = rho/delta, nalpha = -1*alpha
void rbicg_alpha(int nv, const double *rho, const double *delta, double *alpha, double *nalpha,
                 cudaStream_t s);
// RBiCGStab: rho = -1*(omega*psi); beta = rho/(delta*omega); nomega = -1*omega;
// delta = nomega*beta (the coefficient of s in the v_ update)
void rbicg_beta(int nv, const double *omega, const double *psi, double *delta, double *rho,
                double *beta, double *nomega, cudaStream_t s);
// negate: out = -1 * in
void negate(int nv, const double *in, double *out, cudaStream_t s);

// ---- batched independent systems (batch.cu) ---------------------------------
// Segment s owns rows [segoff[s], segoff[s+1]) of the concatenated system;
// its scalars for column k are at [s*nv + k] (nsc = nseg*nv of them).
// Inner products per segment, identical to dots() run on each segment alone:
// cstart[s] = first chunk of segment s (256-row chunks counted per segment,
// nseg+1 entries), part: nchunks*nd*nv doubles, out[d*nsc + s*nv + k].
void seg_dots(Prec in, int nv, int nseg, const i64 *segoff, const i64 *cstart, i64 nchunks, int nd,
              const void *const *a, const void *const *b, double *part, double *out, cudaStream_t s);
// FP64 z = a*x + b*y (op 0) or z = a*x + b*y + c*z (op 1), per-segment scalars
void seg_blas(int nv, int nseg, const i64 *segoff, i64 n, int op, const double *a, const double *x,
              const double *b, const double *y, const double *c, double *z, cudaStream_t s);
// tol2 = max(abs, rel*sqrt(res0))^2; iconv = 1 where the column is not yet
// converged; conv_it = 0; ctr = {iterations = 0, active columns}
void batch_init(int nsc, const double *res0, double rel, double abs_tol, double *tol2, double *iconv,
                int *conv_it, int *ctr, cudaStream_t s);
// omega = s2/s3; res = s4 - omega*s2; ac, oc = alpha, omega on active columns
// and exactly 0 on the others (so a finished column's x never changes)
void batch_omega(int nsc, const double *s2, const double *s3, const double *s4, const double *alpha,
                 const double *iconv, double *omega, double *res, double *ac, double *oc, cudaStream_t s);
// end of an iteration: active columns with res <= tol2 stop (conv_it = the
// iteration); ctr[0] += 1, ctr[1] = active columns; under a CUDA graph the
// while-loop condition `handle` is set to (active && ctr[0] < max_iters)
void batch_check(int nsc, const double *res, const double *tol2, double *iconv, int *conv_it,
                 double *res_last, int *ctr, int max_iters, unsigned long long handle, int use_graph,
                 cudaStream_t s);

}  // namespace xk
