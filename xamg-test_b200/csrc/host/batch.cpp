// Batching form (see batch.h).  The iteration is the PBiCGStab of the
// reference (pbicgstab.inl:70-200, the same step order as the single-system
// Krylov solver) with every scalar held per (system, column).
#include "batch.h"
#include "../kernels.cuh"
#include <algorithm>
#include <cmath>
#include <map>

namespace xamg {

namespace {
enum { RHO, S1, S2, S3, S4, ALPHA, OMEGA, BETA, C1, RES, AC, OC, ICONV, ONES, NALPHA, NOMEGA, TOL2, RES0, RESL, NSC };
}

double *BatchGroup::S(int i) const { return sc.as<double>() + (size_t)i * nsc; }

void Batch::create(int nsys, const i64 *n, const int *const *rp, const int *const *ci,
                   const double *const *val, const int *nv, const GlobalParams &p) {
    XCHECK(nsys > 0, "empty batch");
    gp = p;
    XCHECK(gp.has("solver") && gp.has("preconditioner"), "batch needs solver and preconditioner roles");
    const ParamList &sl = gp.get("solver");
    XCHECK(sl.get_string("method") == "PBiCGStab", "the batched solver is PBiCGStab");
    max_iters = (int)sl.get_int("max_iters");
    rel = sl.has("rel_tolerance") ? sl.get_float("rel_tolerance") : 0.0;
    abs_tol = sl.has("abs_tolerance") ? sl.get_float("abs_tolerance") : 0.0;
    nrows.assign(n, n + nsys);
    nvs.assign(nv, nv + nsys);
    where.assign(nsys, {-1, -1});
    std::map<int, std::vector<int>> bynv;
    for (int q = 0; q < nsys; ++q) {
        XCHECK(nv[q] == 1 || nv[q] == 2 || nv[q] == 4 || nv[q] == 8 || nv[q] == 16 || nv[q] == 32,
               "nv must be 1, 2, 4, 8, 16 or 32");
        XCHECK(n[q] > 0, "empty system");
        bynv[nv[q]].push_back(q);
    }
    cudaStream_t st = ctx().stream;
    for (auto &kv : bynv) {
        auto G = std::unique_ptr<BatchGroup>(new BatchGroup());
        G->nv = kv.first;
        G->sys = kv.second;
        const int nseg = (int)G->sys.size();
        G->nsc = nseg * G->nv;
        // block-diagonal union
        HostCsr &U = G->A.h;
        G->off.assign(1, 0);
        for (int q : G->sys) G->off.push_back(G->off.back() + n[q]);
        const i64 N = G->off.back();
        U.n = U.ncols = N;
        U.rp.assign(N + 1, 0);
        i64 nnz = 0;
        for (int q : G->sys) nnz += rp[q][n[q]];
        XCHECK(nnz < (1ll << 31), "batch group too large for int32 offsets");
        U.ci.resize(nnz);
        U.v.resize(nnz);
        i64 e = 0;
        for (int k = 0; k < nseg; ++k) {
            const int q = G->sys[k];
            const i64 r0 = G->off[k];
            for (i64 i = 0; i < n[q]; ++i) {
                for (int j = rp[q][i]; j < rp[q][i + 1]; ++j) {
                    XCHECK(ci[q][j] >= 0 && ci[q][j] < n[q], "column index outside the system");
                    U.ci[e] = (int)(ci[q][j] + r0);
                    U.v[e] = val[q][j];
                    ++e;
                }
                U.rp[r0 + i + 1] = (int)e;
            }
            where[q] = {(int)groups.size(), k};
        }
        G->A.d.upload(U, true, false);
        G->M = make_role_solver(gp, "preconditioner", G->A, G->nv, Prec::F32);
        for (DVec *q : {&G->x, &G->b, &G->r0, &G->r, &G->p, &G->v, &G->s, &G->t, &G->ph, &G->sh})
            q->alloc(N, G->nv, Prec::F64);
        G->z32.alloc(N, G->nv, Prec::F32);
        G->w32.alloc(N, G->nv, Prec::F32);
        // segments and their 256-row chunks
        std::vector<i64> cs(1, 0);
        for (int k = 0; k < nseg; ++k) cs.push_back(cs.back() + (G->off[k + 1] - G->off[k] + 255) / 256);
        G->nch = cs.back();
        G->segoff.alloc(sizeof(i64) * G->off.size());
        G->cstart.alloc(sizeof(i64) * cs.size());
        XCUDA(cudaMemcpy(G->segoff.p, G->off.data(), sizeof(i64) * G->off.size(), cudaMemcpyHostToDevice));
        XCUDA(cudaMemcpy(G->cstart.p, cs.data(), sizeof(i64) * cs.size(), cudaMemcpyHostToDevice));
        G->part.alloc(sizeof(double) * std::max<i64>(G->nch * 3 * G->nv, 1));
        G->sc.alloc(sizeof(double) * NSC * G->nsc);
        std::vector<double> z((size_t)NSC * G->nsc, 0.0);
        for (int k = 0; k < G->nsc; ++k) z[(size_t)ONES * G->nsc + k] = 1.0;
        XCUDA(cudaMemcpy(G->sc.p, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice));
        G->ctr.alloc(sizeof(int) * 2);
        G->conv_it.alloc(sizeof(int) * G->nsc);
        XCUDA(cudaMemsetAsync(G->x.p(), 0, sizeof(double) * G->x.count(), st));
        XCUDA(cudaMemsetAsync(G->b.p(), 0, sizeof(double) * G->b.count(), st));
        groups.push_back(std::move(G));
    }
    XCUDA(cudaStreamSynchronize(st));
    for (auto &G : groups) autotune(*G);
}

// Pick the SpMV variant of each operator the group's iteration applies to
// the most data: the FP64 union (outer products) and its FP32 copy (the
// finest level of the hierarchy).  All variants give identical results.
void Batch::autotune(BatchGroup &G) {
    cudaStream_t st = ctx().stream;
    const DCsr &a = G.A.d;
    const int vars[] = {0, 1, 2, 3, 5, 6, 7};  // 7: shifted-row runs where the operator has a plan
    cudaEvent_t e0, e1;
    XCUDA(cudaEventCreate(&e0));
    XCUDA(cudaEventCreate(&e1));
    for (int pass = 0; pass < 2; ++pass) {
        const Prec p = pass == 0 ? Prec::F64 : Prec::F32;
        const void *xv = pass == 0 ? G.r.p() : G.z32.p();
        void *yv = pass == 0 ? G.v.p() : G.w32.p();
        float best = 1e30f;
        int bv = -1;
        for (int v : vars) {
            a.variant[pass] = v;
            a.spmv(p, G.nv, xv, yv, 0, nullptr, st);
            XCUDA(cudaEventRecord(e0, st));
            for (int q = 0; q < 5; ++q)
                a.spmv(p, G.nv, xv, yv, 0, nullptr, st);
            XCUDA(cudaEventRecord(e1, st));
            XCUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            XCUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) { best = ms; bv = v; }
        }
        (pass == 0 ? G.var64 : G.var32) = bv;
    }
    // every product of the group's FP64 iteration uses var64, every product
    // of its FP32 hierarchy var32 (choices held by the operators themselves)
    a.variant[0] = G.var64;
    a.variant[1] = -1;
    if (MultiGrid *mg = find_multigrid(G.M.get())) mg_set_spmv_variant(mg, Prec::F32, G.var32);
    XCUDA(cudaEventDestroy(e0));
    XCUDA(cudaEventDestroy(e1));
}

void Batch::run_init(BatchGroup &G) {
    cudaStream_t st = ctx().stream;
    const DCsr &a = G.A.d;
    const i64 N = G.x.n;
    const int nseg = (int)G.sys.size();
    const i64 *so = G.segoff.as<i64>(), *cs = G.cstart.as<i64>();
    double *part = G.part.as<double>();
    a.spmv(Prec::F64, G.nv, G.x.p(), G.r0.p(), 2, G.b.p(), st);
    const void *A1[1] = {G.r0.p()}, *B1[1] = {G.r0.p()};
    xk::seg_dots(Prec::F64, G.nv, nseg, so, cs, G.nch, 1, A1, B1, part, G.S(RHO), st);
    XCUDA(cudaMemcpyAsync(G.S(RES0), G.S(RHO), sizeof(double) * G.nsc, cudaMemcpyDeviceToDevice, st));
    XCUDA(cudaMemcpyAsync(G.S(RESL), G.S(RHO), sizeof(double) * G.nsc, cudaMemcpyDeviceToDevice, st));
    xk::batch_init(G.nsc, G.S(RES0), rel, abs_tol, G.S(TOL2), G.S(ICONV), G.conv_it.as<int>(), G.ctr.as<int>(), st);
    xk::blas(Prec::F64, G.nv, N, xk::Op::COPY, nullptr, G.r0.p(), nullptr, nullptr, nullptr, G.r.p(), st);
    xk::blas(Prec::F64, G.nv, N, xk::Op::COPY, nullptr, G.r0.p(), nullptr, nullptr, nullptr, G.p.p(), st);
}

void Batch::run_body(BatchGroup &G, int graph_mode) {
    cudaStream_t st = ctx().stream;
    const DCsr &a = G.A.d;
    const i64 N = G.x.n;
    const int nv = G.nv, nseg = (int)G.sys.size(), nsc = G.nsc;
    const i64 *so = G.segoff.as<i64>(), *cs = G.cstart.as<i64>();
    double *part = G.part.as<double>();
    auto precond = [&](const DVec &in, DVec &out) {
        xk::convert(Prec::F64, Prec::F32, in.count(), in.p(), G.z32.p(), st);
        xk::fill(Prec::F32, G.w32.count(), 0.0, G.w32.p(), st);
        G.M->solve_from_zero(G.w32, G.z32);
        xk::convert(Prec::F32, Prec::F64, G.w32.count(), G.w32.p(), out.p(), st);
    };
    auto spmv = [&](const DVec &x, DVec &y) {
        a.spmv(Prec::F64, nv, x.p(), y.p(), 0, nullptr, st);
    };
    auto dot1 = [&](const DVec &x, const DVec &y, double *out) {
        const void *A1[1] = {x.p()}, *B1[1] = {y.p()};
        xk::seg_dots(Prec::F64, nv, nseg, so, cs, G.nch, 1, A1, B1, part, out, st);
    };
    auto sb = [&](int op, const double *sa, const DVec &x, const double *sbv, const DVec &y,
                  const double *scv, DVec &z) {
        xk::seg_blas(nv, nseg, so, N, op, sa, (const double *)x.p(), sbv, (const double *)y.p(), scv,
                     (double *)z.p(), st);
    };
    precond(G.p, G.ph);
    spmv(G.ph, G.v);
    dot1(G.v, G.r0, G.S(S1));
    xk::bicg_alpha(nsc, G.S(RHO), G.S(S1), G.S(ALPHA), st);
    xk::negate(nsc, G.S(ALPHA), G.S(NALPHA), st);
    sb(0, G.S(ONES), G.r, G.S(NALPHA), G.v, nullptr, G.s);
    precond(G.s, G.sh);
    spmv(G.sh, G.t);
    {
        const void *A3[3] = {G.t.p(), G.t.p(), G.s.p()}, *B3[3] = {G.s.p(), G.t.p(), G.s.p()};
        xk::seg_dots(Prec::F64, nv, nseg, so, cs, G.nch, 3, A3, B3, part, G.S(S2), st);
    }
    xk::batch_omega(nsc, G.S(S2), G.S(S3), G.S(S4), G.S(ALPHA), G.S(ICONV), G.S(OMEGA), G.S(RES),
                    G.S(AC), G.S(OC), st);
    sb(1, G.S(AC), G.ph, G.S(OC), G.sh, G.S(ONES), G.x);
    xk::batch_check(nsc, G.S(RES), G.S(TOL2), G.S(ICONV), G.conv_it.as<int>(), G.S(RESL), G.ctr.as<int>(),
                    max_iters, G.cond, graph_mode, st);
    xk::negate(nsc, G.S(OMEGA), G.S(NOMEGA), st);
    sb(0, G.S(ONES), G.s, G.S(NOMEGA), G.t, nullptr, G.r);
    dot1(G.r, G.r0, G.S(S1));
    xk::bicg_beta(nsc, G.S(S1), G.S(RHO), G.S(ALPHA), G.S(OMEGA), G.S(BETA), G.S(C1), st);
    sb(1, G.S(ONES), G.r, G.S(C1), G.v, G.S(BETA), G.p);
}

void Batch::build_graph() {
    cudaStream_t st = ctx().stream;
    XCUDA(cudaGraphCreate(&graph, 0));
    for (auto &Gp : groups) {
        BatchGroup &G = *Gp;
        cudaGraphConditionalHandle h;
        XCUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
        G.cond = (unsigned long long)h;
        // initialisation: new root nodes of the graph (groups are independent)
        XCUDA(cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        long long k0 = xk::launch_count();
        run_init(G);
        G.init_kernels = xk::launch_count() - k0;
        cudaStreamCaptureStatus cst;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        XCUDA(cudaStreamGetCaptureInfo(st, &cst, nullptr, nullptr, &deps, &nd));
        std::vector<cudaGraphNode_t> last(deps, deps + nd);
        cudaGraph_t g2 = nullptr;
        XCUDA(cudaStreamEndCapture(st, &g2));
        // while (active columns and iterations left) { one iteration }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        XCUDA(cudaGraphAddNode(&cn, graph, last.data(), last.size(), &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        XCUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        k0 = xk::launch_count();
        run_body(G, 1);
        G.body_kernels = xk::launch_count() - k0;
        cudaGraph_t b2 = nullptr;
        XCUDA(cudaStreamEndCapture(st, &b2));
    }
    XCUDA(cudaGraphInstantiate(&exec, graph, 0));
}

void Batch::solve() {
    cudaStream_t st = ctx().stream;
    cudaEvent_t e0, e1;
    XCUDA(cudaEventCreate(&e0));
    XCUDA(cudaEventCreate(&e1));
    if (use_graph && !exec) {
        // one eager pass of every step first: allocations and function
        // attributes of the hierarchy happen outside the capture
        std::vector<DVec> keep(groups.size());
        for (size_t g = 0; g < groups.size(); ++g) {
            BatchGroup &G = *groups[g];
            keep[g].alloc(G.x.n, G.nv, Prec::F64);
            XCUDA(cudaMemcpyAsync(keep[g].p(), G.x.p(), sizeof(double) * G.x.count(), cudaMemcpyDeviceToDevice, st));
            run_init(G);
            run_body(G, 0);
            XCUDA(cudaMemcpyAsync(G.x.p(), keep[g].p(), sizeof(double) * G.x.count(), cudaMemcpyDeviceToDevice, st));
        }
        XCUDA(cudaStreamSynchronize(st));
        build_graph();
    }
    const long long k0 = xk::launch_count();
    XCUDA(cudaEventRecord(e0, st));
    if (use_graph) {
        XCUDA(cudaGraphLaunch(exec, st));
    } else {
        for (auto &G : groups) run_init(*G);
        std::vector<int> done(groups.size(), 0);
        for (int it = 0; it < max_iters; ++it) {
            bool any = false;
            for (size_t g = 0; g < groups.size(); ++g) {
                if (done[g]) continue;
                run_body(*groups[g], 0);
                int c[2];
                XCUDA(cudaMemcpyAsync(c, groups[g]->ctr.p, sizeof(c), cudaMemcpyDeviceToHost, st));
                XCUDA(cudaStreamSynchronize(st));
                if (c[1] == 0) done[g] = 1;
                else any = true;
            }
            if (!any) break;
        }
    }
    XCUDA(cudaEventRecord(e1, st));
    XCUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    XCUDA(cudaEventElapsedTime(&ms, e0, e1));
    last_ms = ms;
    XCUDA(cudaEventDestroy(e0));
    XCUDA(cudaEventDestroy(e1));
    if (use_graph) {
        // kernels the graph executed: every group's init plus its iterations
        last_kernels = 0;
        for (auto &G : groups) {
            int c[2];
            XCUDA(cudaMemcpy(c, G->ctr.p, sizeof(c), cudaMemcpyDeviceToHost));
            last_kernels += G->init_kernels + (long long)c[0] * G->body_kernels;
        }
    } else {
        last_kernels = xk::launch_count() - k0;
    }
}

void Batch::upload(int sys, const double *b, const double *x0) {
    XCHECK(sys >= 0 && sys < (int)where.size(), "system index out of range");
    BatchGroup &G = *groups[where[sys].first];
    const i64 r0 = G.off[where[sys].second], n = nrows[sys];
    cudaStream_t st = ctx().stream;
    const size_t bytes = sizeof(double) * n * G.nv;
    if (b) XCUDA(cudaMemcpyAsync(((double *)G.b.p()) + r0 * G.nv, b, bytes, cudaMemcpyHostToDevice, st));
    if (x0) XCUDA(cudaMemcpyAsync(((double *)G.x.p()) + r0 * G.nv, x0, bytes, cudaMemcpyHostToDevice, st));
    else XCUDA(cudaMemsetAsync(((double *)G.x.p()) + r0 * G.nv, 0, bytes, st));
    XCUDA(cudaStreamSynchronize(st));
}

void Batch::download(int sys, double *x) const {
    XCHECK(sys >= 0 && sys < (int)where.size(), "system index out of range");
    const BatchGroup &G = *groups[where[sys].first];
    const i64 r0 = G.off[where[sys].second], n = nrows[sys];
    cudaStream_t st = ctx().stream;
    XCUDA(cudaMemcpyAsync(x, ((double *)G.x.p()) + r0 * G.nv, sizeof(double) * n * G.nv, cudaMemcpyDeviceToHost, st));
    XCUDA(cudaStreamSynchronize(st));
}

void Batch::stats(int sys, int *iters, double *relres) const {
    XCHECK(sys >= 0 && sys < (int)where.size(), "system index out of range");
    const BatchGroup &G = *groups[where[sys].first];
    const int k0 = where[sys].second * G.nv;
    std::vector<int> it(G.nsc), ic(1);
    std::vector<double> sc((size_t)NSC * G.nsc);
    XCUDA(cudaMemcpy(it.data(), G.conv_it.p, sizeof(int) * G.nsc, cudaMemcpyDeviceToHost));
    XCUDA(cudaMemcpy(sc.data(), G.sc.p, sizeof(double) * sc.size(), cudaMemcpyDeviceToHost));
    for (int k = 0; k < G.nv; ++k) {
        const double r0 = sc[(size_t)RES0 * G.nsc + k0 + k], rl = sc[(size_t)RESL * G.nsc + k0 + k];
        const bool active = sc[(size_t)ICONV * G.nsc + k0 + k] != 0.0;
        iters[k] = active ? -1 : it[k0 + k];
        relres[k] = r0 > 0 ? std::sqrt(std::max(rl, 0.0) / r0) : 0.0;
    }
}

Batch::~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

}  // namespace xamg
