// Batching form: many independent systems of uneven size, each with its own
// number of right-hand sides, solved together on one GPU.
#pragma once
#include "solve.h"
#include <memory>

namespace xamg {

// Systems with the same nv are concatenated into one block-diagonal system
// (a group).  The group's PBiCGStab runs in FP64 with per-(system, column)
// scalars and convergence flags on the device; its AMG preconditioner (set
// up on the block-diagonal operator, whose hierarchy is block-diagonal too)
// runs in FP32.  One iteration of every group is captured as the body of a
// CUDA-graph while loop whose condition a device kernel sets, so the whole
// batch runs as one graph launch with no host round trip.
struct BatchGroup {
    int nv = 1;
    std::vector<int> sys;     // system ids
    std::vector<i64> off;     // row offsets of the systems in the union (nseg + 1)
    Matrix A;                 // block-diagonal union, FP64 (+ FP32 for the hierarchy)
    std::unique_ptr<Solver> M;
    DVec x, b, r0, r, p, v, s, t, ph, sh;  // FP64
    DVec z32, w32;                          // FP32 preconditioner input / output
    DBuf segoff, cstart, part, sc, ctr, conv_it;
    i64 nch = 0;
    int nsc = 0;
    int var64 = -1, var32 = -1;             // autotuned SpMV variants (FP64 outer, FP32 hierarchy)
    unsigned long long cond = 0;            // CUDA-graph while-loop handle
    long long init_kernels = 0, body_kernels = 0;  // kernels of the init steps / one iteration
    double *S(int i) const;
};

struct Batch {
    GlobalParams gp;
    int max_iters = 100;
    double rel = 1e-8, abs_tol = 0.0;
    std::vector<i64> nrows;
    std::vector<int> nvs;
    std::vector<std::pair<int, int>> where;  // system -> (group, segment)
    std::vector<std::unique_ptr<BatchGroup>> groups;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double last_ms = 0.0;
    long long last_kernels = 0;  // kernel executions of the last solve
    bool use_graph = true;

    void create(int nsys, const i64 *n, const int *const *rp, const int *const *ci,
                const double *const *val, const int *nv, const GlobalParams &p);
    void upload(int sys, const double *b, const double *x0);
    void download(int sys, double *x) const;
    void solve();
    // iterations at convergence (0 = converged at the start, -1 = not
    // converged) and final relative residual estimate, per column
    void stats(int sys, int *iters, double *relres) const;
    ~Batch();

  private:
    void run_init(BatchGroup &G);
    void run_body(BatchGroup &G, int graph_mode);
    void autotune(BatchGroup &G);
    void build_graph();
};

}  // namespace xamg
