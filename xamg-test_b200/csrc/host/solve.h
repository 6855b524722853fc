// Device-resident matrices, vectors, multigrid hierarchy and solvers.
//
// Class map to the reference (src/solvers/*):
//   Krylov       <- BiCGStab / PBiCGStab (bicgstab.inl:44-197, pbicgstab.inl:48-207)
//                   RBiCGStab (rbicgstab.inl:48-225), PCG (pcg.inl:48-160)
//                   and their Merged* variants (same values, one code path)
//   MultiGrid    <- MultiGrid (mg.inl:117-331), levels from the host AMG setup
//   HSGS, Jacobi <- hsgs.inl:31-91, jacobi.inl:31-102
//   Direct       <- direct.inl:31-59 (+ inverse.inl Gauss-Jordan at setup)
//   IterRefine   <- IterativeRefinement (ir.inl:107-194)
// A solver of precision F32 keeps its vectors and matrix values in FP32 and
// accumulates inner products and scalar recurrences in FP64.
#pragma once
#include "common.h"
#include "params.h"

namespace xamg {

struct AmgParams;
struct AmgLevel;

struct DVec {
    i64 n = 0;
    int nv = 1;
    Prec prec = Prec::F64;
    DBuf buf;
    void alloc(i64 n_, int nv_, Prec p) {
        n = n_;
        nv = nv_;
        prec = p;
        buf.alloc((size_t)(n_ * nv_) * prec_size(p));
    }
    void *p() const { return buf.p; }
    i64 count() const { return n * nv; }
};

// Shifted-row run plan of a square operator (xk::spmv_runs): chunks of up to
// R = 8 consecutive rows whose column indices are the first row's shifted by
// the row offset, with the values reordered entry-major per chunk.
struct RunPlan {
    int R = 0;
    i64 nchunks = 0, ntiles = 0, nseg = 0;
    double coverage = 0.0;     // fraction of the entries that lie in chunks of R rows
    std::vector<int> hchunks;  // {r0, cnt, m, segments} per chunk (host)
    std::vector<i64> hvoff;    // per tile of four chunks: first value slot (host, ntiles + 1)
    DBuf chunks, toff, sg, v64, v32;
    // Detect the chunks of h; keeps the plan (FP64 and/or FP32 values) when at
    // least min_cov of the entries lie in chunks of R rows, else clears it.
    bool build(const HostCsr &h, int R_, bool f64, bool f32, double min_cov);
    void add_values(const HostCsr &h, Prec p);  // values of another precision
    bool has(Prec p) const { return nchunks > 0 && (p == Prec::F64 ? v64.p != nullptr : v32.p != nullptr); }
    void clear();
};

// Run detection alone (host only): chunk count, fraction of the entries in
// chunks of R rows, and segments (runs of at most 3 consecutive columns of
// each chunk's first row).
void run_plan_analyze(i64 n, const int *rp, const int *ci, int R, i64 *nchunks, double *coverage, i64 *nseg);

struct DCsr {
    i64 n = 0, ncols = 0, nnz = 0;
    DBuf rp, ci, v64, v32;
    RunPlan runs;
    // this operator's SpMV kernel choice per precision (see
    // xk::set_spmv_variant); -1 = the calling thread's setting.  Results are
    // identical for every choice.
    mutable int variant[2] = {-1, -1};
    void upload(const HostCsr &h, bool f64, bool f32);
    // y = A x (mode 0), y += A x (1), y = b - A x (2): the run kernel when this
    // operator has a plan in precision p and the shape suits it, else xk::spmv
    void spmv(Prec p, int nv, const void *x, void *y, int mode, const void *b, cudaStream_t s) const;
    const void *val(Prec p) const {
        if (p == Prec::F64) { XCHECK(v64.p || nnz == 0, "FP64 values not resident"); return v64.p; }
        XCHECK(v32.p || nnz == 0, "FP32 values not resident");
        return v32.p;
    }
    const int *rpp() const { return rp.as<int>(); }
    const int *cip() const { return ci.as<int>(); }
};

// Wavefront schedule of the forward and backward Gauss-Seidel sweeps of one
// matrix (optionally restricted to hybrid blocks of `brows` rows).
// Sweep schedules: LEVELS launches one kernel per wavefront level; GRID runs
// a whole sweep in one cooperative launch with a bounded grid barrier per
// level; BLOCKS (hybrid plans only) runs each block in its own CTA with CTA
// barriers, both sweeps in one launch.
enum class GsMode : int { LEVELS = 0, GRID = 1, BLOCKS = 2 };

// Synchronisation words of a plan's sweeps, each group on its own 128-byte
// line: grid-barrier words at 0 (arrival counter) and 128 (release word), the
// error flag at kSyncErrOffset.
constexpr size_t kSyncBytes = 384;
constexpr size_t kSyncErrOffset = 256;

struct GsPlan {
    i64 n = 0, brows = 0;
    int nlf = 0, nlb = 0;
    int nblocks = 1;
    GsMode mode = GsMode::GRID;
    std::vector<int> hlf, hlb;         // level pointers (host)
    std::vector<int> lf, lb;           // per-row levels (host, for export)
    DBuf permf, permb, lptrf, lptrb;   // device copies (global level order)
    DBuf bblevf, bblevb, blptrf, blptrb, bpermf, bpermb;  // per-block order (BLOCKS)
    DBuf sync;                         // barrier words + error flag (kSyncBytes)
    // level-ordered copies of the matrix per direction (GRID/BLOCKS sweeps)
    struct Lcsr {
        DBuf lrp, lci, lva, lrow, linvd, desc, blev;
        int nlev = 0;  // GRID: levels; BLOCKS: unused (per-block counts in blev)
        int ncta = 0;  // CTAs of the launch the descriptors were built for
        int emax = 0;  // most entries of one CTA in one level
        int rmax = 0;  // most rows of one CTA in one level (span rounded out to 4)
        int lmax = 0;  // BLOCKS: most levels of one block
        int nlmax = 0; // BLOCKS with a slot window: longest load list of one level
        // BLOCKS: slot-mapped x window (see build_slots): column indices
        // remapped to window slots, each level-ordered row's slot, and per
        // level the rows whose old x is loaded into their slot kSlotAhead
        // levels ahead of their first use
        DBuf lcs, lslot, ldd, ldpre, ld;
        int nslots = 0;  // 0: no window (too many rows live at once)
        // GRID: per (level, CTA) the CTAs whose earlier levels this one's rows
        // depend on, {cta, levels it must have finished} (see build_grid_deps)
        DBuf dptr, deps;
        bool has_deps = false;
    } lc[2];
    DBuf prog;  // GRID: per-CTA count of finished levels (32-byte stride)
    bool has_lcsr = false;
    i64 nnz_in = 0;  // entries inside the rows' blocks (all entries without blocks)
    Prec lprec = Prec::F64;
    // hybrid plans: the entries of A outside each row's block, in CSR order
    // (values in precision aprec), so that the right-hand side of the block
    // sweeps, t = b - A_off x, is one SpMV of this operator in mode 2
    DCsr aoff;
    Prec aprec = Prec::F64;
    void build(const HostCsr &A, i64 brows_, GsMode mode_);
    // store the level-ordered matrix copies in precision p (values from A)
    void build_lcsr(const HostCsr &A, Prec p);
    void build_offblock(const HostCsr &A, Prec p);
    // point-to-point dependencies of one sweep direction of a GRID plan
    void build_grid_deps(int d, const HostCsr &A, const std::vector<int> &lev, const std::vector<int> &order,
                         const std::vector<int> &desc, int G);
    // slot window of one sweep direction of a BLOCKS plan (called by build_lcsr)
    void build_slots(int d, const std::vector<int> &order, const std::vector<int> &groups,
                     const std::vector<int> &blev, const std::vector<int> &lrp, const std::vector<int> &lci);
    // forward (or backward) sweep; in BLOCKS mode the forward call runs both
    // sweeps and the backward call does nothing
    void sweep(Prec p, int nv, const int *rp, const int *ci, const void *val, const void *invd,
               const void *t, void *x, const void *relax, bool forward, cudaStream_t s);
    int error_flag() const;
};
GsMode gs_mode_from(const std::string &s, i64 brows, i64 n);

// Convergence bookkeeping, convergence.h:48-303 with conv_check/print flags.
struct Conv {
    int nv = 1;
    bool check_on = true, print_on = false;
    double abs_tol = 0, rel_tol = 0;
    std::vector<double> ptol;  // per-column tolerance (IR inner solver)
    // rel_tolerance applies to ||b|| instead of the initial residual
    // (extension key rel_tolerance_base = "rhs"); base holds ||b||^2
    bool rhs_base = false;
    std::vector<double> base;
    std::vector<double> res0, res;
    std::vector<int> status;
    int iters = 0, sub_iters = 0;
    std::vector<double> history;  // res after every check, nv per entry
    std::string prefix = "SOLV";
    void init(int nv_) {
        nv = nv_;
        res0.assign(nv, 0.0);
        res.assign(nv, 0.0);
        status.assign(nv, 0);
        iters = sub_iters = 0;
        history.clear();
    }
    double tol(int k) const;
    void update(const double *r);
    bool check();
    void record() { history.insert(history.end(), res.begin(), res.end()); }
};

// convergence flags and tolerances of a role's parameter list
// (convergence_details, abs_tolerance, rel_tolerance, rel_tolerance_base)
void parse_conv_settings(const ParamList &l, Conv &c);

struct Solver;

// One multigrid level on the device.
struct MGLevel {
    HostCsr hA, hP;         // host copies (setup output; exported for parity)
    DCsr A, P, R;
    DBuf invd64, invd32;
    DBuf isd64, isd32;       // sqrt(1/a_ii) (Chebyshev smoother), on demand
    double min_eig = 0.0, max_eig = 0.0;  // spectrum estimate of D^-1/2 A D^-1/2 (Chebyshev)
    GsPlan gs_pre, gs_post;  // share one plan when the block sizes agree
    Prec prec = Prec::F64;   // precision of this level's vectors/operator
    DVec tmp, tmp2, xH, bH;  // work vectors: tmp/tmp2 on this level, xH/bH on the next
    std::unique_ptr<Solver> pre, post;
};

struct SolveEnv {
    cudaStream_t s;
};

struct Solver {
    std::string role = "solver";
    std::string method;
    ParamList prm;
    int nv = 1;
    Prec prec = Prec::F64;
    Conv conv;
    virtual ~Solver() {}
    // x: initial guess on entry (the preconditioner role zeroes it itself)
    virtual void solve(DVec &x, const DVec &b) = 0;
    // the same with x known to be zero on entry (the caller has just zeroed
    // it): a solver may skip products with x whose result is then exactly
    // known; the results are identical to solve()
    virtual void solve_from_zero(DVec &x, const DVec &b) { solve(x, b); }
    virtual void renew(const GlobalParams &gp) {}
    virtual std::string info() const { return method; }
};

// Build the solver tree for `gp` over the FP64 host operator A (kept alive by
// the caller together with its device copy).
struct Matrix {
    HostCsr h;
    DCsr d;        // FP64 (and FP32 on demand)
    bool has32 = false;
    void ensure32();
};

std::unique_ptr<Solver> build_solver_tree(const GlobalParams &gp, Matrix &A, int nv);
// The solver of one role of gp (e.g. the preconditioner) in precision prec.
std::unique_ptr<Solver> make_role_solver(const GlobalParams &gp, const std::string &role, Matrix &A,
                                         int nv, Prec prec);

// Export hooks for parity tests.
struct MultiGrid;
MultiGrid *find_multigrid(Solver *s);
int mg_num_levels(MultiGrid *mg);
const HostCsr &mg_level_A(MultiGrid *mg, int l);
const HostCsr &mg_level_P(MultiGrid *mg, int l);
const GsPlan &mg_level_gs(MultiGrid *mg, int l);
const std::vector<double> &mg_coarse_inverse(MultiGrid *mg);
// give every operator of the hierarchy (A, P, R, off-block parts) this SpMV
// choice for products in precision p
void mg_set_spmv_variant(MultiGrid *mg, Prec p, int variant);
// spectrum bounds used by a level's Chebyshev smoother (0, 0 when none)
void mg_level_eig(MultiGrid *mg, int l, double *mn, double *mx);

// Kernel timing (see KTimeScope): enable/disable (returns the old state) and
// read the per-(class, rows) aggregates.
int ktime_enable(int on);
// 1 when hybrid Gauss-Seidel sweeps run one warp per block, 0 one CTA per block
int gs_warp_sweep();
int ktime_read(int cap, int *kclass, i64 *rows, i64 *launches, double *ms, double *bytes);

void dense_inverse(int n, const double *A, double *Ainv);
void csr_transpose(const HostCsr &P, HostCsr &R);

}  // namespace xamg
