// Row-partitioned solve of one system over several GPUs (one rank per GPU).
//
// The reference distributes a system by contiguous row blocks (part.h), pulls
// the x values of other blocks that its rows read before every product
// (comm_p2p, matvec_comm.h:117-312) and sums the per-rank inner products of a
// BiCGStab step with one allreduce (shm_allreduce.h:112-163, called from
// pbicgstab.inl:125-186).  Here each rank holds its block of the operator with
// columns [owned | halo] (RowPart, dist.h); before a product the ranks gather
// the rows their peers need into a send buffer and exchange them with NCCL
// send/receive straight into the halo part of the multiplied vector (this
// GPU's own memory; no kernel reads a peer's memory); the inner products of a
// step are computed locally by the usual kernels and summed over the ranks
// with one NCCL allreduce of NV (or 3 NV) doubles before the scalar
// recurrence.  The preconditioner is the AMG V-cycle of the rank's diagonal
// block (block Jacobi across ranks, the reference's hybrid semantics between
// processes).  With one rank every step is the single-GPU solver's, bit for
// bit.  NCCL is loaded at run time (libnccl.so.2), so the library itself does
// not depend on it.
#include "solve.h"
#include "dist.h"
#include <dlfcn.h>
#include <nccl.h>
#include <mutex>

namespace xamg {

namespace {

struct Nccl {
    void *h = nullptr;
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

Nccl &nccl() {
    static Nccl n;
    static std::once_flag once;
    std::call_once(once, [] {
        n.h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!n.h) return;
        auto sym = [](const char *s) { return dlsym(n.h, s); };
        n.GetUniqueId = (decltype(n.GetUniqueId))sym("ncclGetUniqueId");
        n.CommInitRank = (decltype(n.CommInitRank))sym("ncclCommInitRank");
        n.CommDestroy = (decltype(n.CommDestroy))sym("ncclCommDestroy");
        n.AllReduce = (decltype(n.AllReduce))sym("ncclAllReduce");
        n.Send = (decltype(n.Send))sym("ncclSend");
        n.Recv = (decltype(n.Recv))sym("ncclRecv");
        n.GroupStart = (decltype(n.GroupStart))sym("ncclGroupStart");
        n.GroupEnd = (decltype(n.GroupEnd))sym("ncclGroupEnd");
        n.GetErrorString = (decltype(n.GetErrorString))sym("ncclGetErrorString");
    });
    XCHECK(n.h && n.GetUniqueId && n.CommInitRank && n.CommDestroy && n.AllReduce && n.Send && n.Recv &&
               n.GroupStart && n.GroupEnd,
           "NCCL (libnccl.so.2) is not available");
    return n;
}

void nccheck(ncclResult_t r, const char *what) {
    if (r != ncclSuccess)
        throw Error(std::string("NCCL ") + what + ": " + (nccl().GetErrorString ? nccl().GetErrorString(r) : "error"),
                    3);
}

// A device vector view onto the first n rows of another vector's buffer (it
// does not own the memory).
struct View {
    DVec v;
    void bind(const DVec &base, i64 n) {
        v.n = n;
        v.nv = base.nv;
        v.prec = base.prec;
        v.buf.p = base.buf.p;
        v.buf.bytes = (size_t)n * base.nv * prec_size(base.prec);
    }
    ~View() { v.buf.p = nullptr; }
};

}  // namespace

void dist_unique_id(void *out) {
    ncclUniqueId id;
    nccheck(nccl().GetUniqueId(&id), "GetUniqueId");
    std::memcpy(out, &id, sizeof(id));
}

struct DistSolver {
    RowPart part;
    int nv = 1;
    int nranks = 1, rank = 0;
    ncclComm_t comm = nullptr;
    GlobalParams gp;
    Matrix Aext;   // owned rows, columns [owned | halo]
    Matrix Adiag;  // owned rows and columns (the preconditioner's operator)
    std::unique_ptr<Solver> M;
    bool precond = false;
    i64 nl = 0, nh = 0;
    // pe / se: the vectors multiplied by A, extended by the halo rows (p_ and
    // s_ with a preconditioner, p and s without); pv / sv: their owned rows;
    // pd: the search direction p when it is preconditioned (else p is pv)
    DVec r0, r, v, s, t, pe, se, xe, pd;
    View pv, sv;
    DBuf part_, sc, sendidx, sendbuf;
    std::vector<i64> soff, scnt, roff, rcnt;  // per peer: send and receive rows
    Conv conv;
    int max_iters = 200;
    double *hres = nullptr;
    enum { RHO, S1, S2, S3, S4, ALPHA, OMEGA, BETA, C1, RES, AC, OC, ICONV, STAT, TOLS, NSC };
    double *S(int i) const { return sc.as<double>() + (size_t)i * nv; }

    ~DistSolver() {
        M.reset();
        if (comm) nccl().CommDestroy(comm);
        if (hres) cudaFreeHost(hres);
    }

    xk::BicgScalars scalars() const {
        xk::BicgScalars b;
        b.rho = S(RHO); b.alpha = S(ALPHA); b.omega = S(OMEGA); b.beta = S(BETA); b.c1 = S(C1);
        b.ac = S(AC); b.oc = S(OC); b.res = S(RES); b.iconv = S(ICONV); b.status = S(STAT);
        b.tol = S(TOLS);
        b.check = conv.check_on ? 1 : 0;
        return b;
    }

    void setup(const void *uid, const double *val_global) {
        nranks = part.nranks;
        rank = part.rank;
        nl = part.nrows();
        nh = (i64)part.halo.size();
        // the method first: nothing is set up for a method this solver does not run
        const ParamList &sl = gp.get("solver");
        const std::string m = sl.get_string("method");
        XCHECK(m == "BiCGStab" || m == "PBiCGStab" || m == "MergedBiCGStab" || m == "MergedPBiCGStab",
               "the row-partitioned solve runs (P)BiCGStab");
        cudaStream_t st = ctx().stream;
        ncclUniqueId id;
        std::memcpy(&id, uid, sizeof(id));
        nccheck(nccl().CommInitRank(&comm, nranks, id, rank), "CommInitRank");
        // local operators
        HostCsr &E = Aext.h;
        E.n = nl;
        E.ncols = nl + nh;
        E.rp = part.lrp;
        E.ci = part.lci;
        E.v.resize(part.lsrc.size());
        for (size_t q = 0; q < part.lsrc.size(); ++q) E.v[q] = val_global[part.lsrc[q]];
        Aext.d.upload(E, true, false);
        HostCsr &D = Adiag.h;
        D.n = D.ncols = nl;
        D.rp.assign((size_t)nl + 1, 0);
        for (i64 i = 0; i < nl; ++i) {
            for (int q = E.rp[i]; q < E.rp[i + 1]; ++q)
                if (E.ci[q] < nl) {
                    D.ci.push_back(E.ci[q]);
                    D.v.push_back(E.v[q]);
                }
            D.rp[i + 1] = (int)D.ci.size();
        }
        Adiag.d.upload(D, true, false);
        precond = (m == "PBiCGStab" || m == "MergedPBiCGStab") && gp.has("preconditioner");
        if (precond) M = make_role_solver(gp, "preconditioner", Adiag, nv, Prec::F64);
        max_iters = (int)sl.get_int("max_iters");
        parse_conv_settings(sl, conv);
        conv.prefix = "DIST";
        for (DVec *q : {&r0, &r, &v, &s, &t}) q->alloc(nl, nv, Prec::F64);
        for (DVec *q : {&pe, &se, &xe}) q->alloc(nl + nh, nv, Prec::F64);
        if (precond) pd.alloc(nl, nv, Prec::F64);
        pv.bind(pe, nl);
        sv.bind(se, nl);
        part_.alloc(sizeof(double) * std::max<i64>(xk::dot_part_size(nl, 3, nv), 1));
        sc.alloc(sizeof(double) * NSC * nv);
        XCUDA(cudaMallocHost(&hres, sizeof(double) * nv));
        // exchange plan: per peer the rows to send (local indices) and the
        // halo slots to receive (contiguous: the halo is grouped by owner)
        soff.assign(nranks + 1, 0);
        scnt.assign(nranks, 0);
        roff.assign(nranks, 0);
        rcnt.assign(nranks, 0);
        std::vector<int> idx;
        for (int q = 0; q < nranks; ++q) {
            soff[q] = (i64)idx.size();
            for (i64 g : part.sends[q]) idx.push_back((int)(g - part.first[rank]));
            scnt[q] = (i64)idx.size() - soff[q];
        }
        soff[nranks] = (i64)idx.size();
        for (size_t h = 0; h < part.halo.size(); ++h) {
            const int o = part.halo_owner[h];
            if (rcnt[o] == 0) roff[o] = (i64)h;
            ++rcnt[o];
        }
        sendidx.alloc(sizeof(int) * std::max<size_t>(idx.size(), 1));
        if (!idx.empty())
            XCUDA(cudaMemcpy(sendidx.p, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice));
        sendbuf.alloc(sizeof(double) * std::max<size_t>(idx.size() * nv, 1));
        std::vector<double> z(NSC * nv, 0.0);
        XCUDA(cudaMemcpyAsync(sc.p, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice, st));
        XCUDA(cudaStreamSynchronize(st));
    }

    // halo rows of an extended vector from their owners
    void exchange(DVec &e, cudaStream_t st) {
        if (nranks == 1) return;
        xk::gather_rows(Prec::F64, nv, soff[nranks], sendidx.as<int>(), e.p(), sendbuf.p, st);
        auto &N = nccl();
        nccheck(N.GroupStart(), "GroupStart");
        for (int q = 0; q < nranks; ++q) {
            if (q == rank) continue;
            if (scnt[q])
                nccheck(N.Send(sendbuf.as<double>() + soff[q] * nv, (size_t)scnt[q] * nv, ncclDouble, q, comm, st),
                        "Send");
            if (rcnt[q])
                nccheck(N.Recv((double *)e.p() + (nl + roff[q]) * nv, (size_t)rcnt[q] * nv, ncclDouble, q, comm, st),
                        "Recv");
        }
        nccheck(N.GroupEnd(), "GroupEnd");
    }

    // local inner products of nd pairs, summed over the ranks into out
    void dots(int nd, const void *const *a, const void *const *b, double *out, cudaStream_t st) {
        xk::dots(Prec::F64, nv, nl, nd, a, b, part_.as<double>(), out, st);
        nccheck(nccl().AllReduce(out, out, (size_t)nd * nv, ncclDouble, ncclSum, comm, st), "AllReduce");
    }

    void read_res(double *src, cudaStream_t st) {
        XCUDA(cudaMemcpyAsync(hres, src, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
        XCUDA(cudaStreamSynchronize(st));
    }

    // x (owned rows, in place) for b (owned rows); the step order of
    // PBiCGStab (pbicgstab.inl:108-204) with the single-GPU solver's kernels
    void solve(double *x, const double *b) {
        cudaStream_t st = ctx().stream;
        const i64 cnt = nl * nv;
        conv.init(nv);
        {
            std::vector<double> one(nv, 1.0);
            XCUDA(cudaMemcpyAsync(S(ICONV), one.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        }
        // r0 = b - A x, with x's halo
        XCUDA(cudaMemcpyAsync(xe.p(), x, sizeof(double) * cnt, cudaMemcpyDeviceToDevice, st));
        exchange(xe, st);
        Aext.d.spmv(Prec::F64, nv, xe.p(), r0.p(), 2, b, st);
        {
            const void *A1[1] = {r0.p()}, *B1[1] = {r0.p()};
            dots(1, A1, B1, S(RHO), st);
        }
        read_res(S(RHO), st);
        conv.res0.assign(hres, hres + nv);
        conv.update(hres);
        conv.record();
        if (conv.check()) return;
        {
            std::vector<double> h(3 * nv);
            for (int k = 0; k < nv; ++k) {
                h[k] = conv.status[k] ? 0.0 : 1.0;
                h[nv + k] = conv.status[k] ? 1.0 : 0.0;
                h[2 * nv + k] = conv.tol(k);
            }
            XCUDA(cudaMemcpyAsync(S(ICONV), h.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
            XCUDA(cudaMemcpyAsync(S(STAT), h.data() + nv, sizeof(double) * 2 * nv, cudaMemcpyHostToDevice, st));
            XCUDA(cudaStreamSynchronize(st));
        }
        xk::blas(Prec::F64, nv, nl, xk::Op::COPY, nullptr, r0.p(), nullptr, nullptr, nullptr, r.p(), st);
        // p: the direction (pd, preconditioned into pe's owned rows) or pe's
        // owned rows themselves; sS: s (preconditioned into se) or se's rows
        DVec &p = precond ? pd : pv.v;
        DVec &sS = precond ? s : sv.v;
        xk::blas(Prec::F64, nv, nl, xk::Op::COPY, nullptr, r0.p(), nullptr, nullptr, nullptr, p.p(), st);
        const xk::BicgScalars bs = scalars();
        for (int it = 1;; ++it) {
            conv.iters = it;
            if (precond) {
                xk::fill(Prec::F64, pv.v.count(), 0.0, pv.v.p(), st);
                M->solve_from_zero(pv.v, p);
            }
            exchange(pe, st);
            Aext.d.spmv(Prec::F64, nv, pe.p(), v.p(), 0, nullptr, st);
            {
                const void *A1[1] = {v.p()}, *B1[1] = {r0.p()};
                dots(1, A1, B1, S(S1), st);
                xk::bicg_epi(0, nv, S(S1), bs, st);
            }
            xk::bicg_s(Prec::F64, nv, nl, bs, r.p(), v.p(), sS.p(), precond ? sv.v.p() : nullptr, st);
            if (precond) M->solve_from_zero(sv.v, s);
            exchange(se, st);
            Aext.d.spmv(Prec::F64, nv, se.p(), t.p(), 0, nullptr, st);
            {
                const void *A3[3] = {t.p(), t.p(), sS.p()}, *B3[3] = {sS.p(), t.p(), sS.p()};
                dots(3, A3, B3, S(S2), st);
                xk::bicg_epi(1, nv, S(S2), bs, st);
            }
            xk::bicg_xr(Prec::F64, nv, nl, bs, pv.v.p(), sv.v.p(), x, sS.p(), t.p(), r.p(), r0.p(),
                        part_.as<double>(), st);
            read_res(S(RES), st);
            conv.update(hres);
            conv.record();
            if (conv.check()) break;
            if (it >= max_iters) break;
            xk::dot_reduce(nl, 1, nv, part_.as<double>(), S(S1), st);
            nccheck(nccl().AllReduce(S(S1), S(S1), (size_t)nv, ncclDouble, ncclSum, comm, st), "AllReduce");
            xk::bicg_epi(2, nv, S(S1), bs, st);
            xk::bicg_p(Prec::F64, nv, nl, bs, r.p(), v.p(), p.p(), nullptr, st);
        }
        XCUDA(cudaStreamSynchronize(st));
    }
};

// C-ABI glue (the entry points live in c_api.cpp, which keeps no NCCL types)
DistSolver *dist_create(const void *uid, const RowPart &part, const double *val_global, const GlobalParams &gp,
                        int nv) {
    std::unique_ptr<DistSolver> d(new DistSolver());
    d->part = part;
    d->gp = gp;
    d->nv = nv;
    d->setup(uid, val_global);
    return d.release();
}
void dist_solve(DistSolver *d, const double *b, double *x) { d->solve(x, b); }
void dist_destroy(DistSolver *d) { delete d; }
int dist_iters(const DistSolver *d) { return d->conv.iters; }
bool dist_converged(const DistSolver *d) {
    for (int s : d->conv.status)
        if (!s) return false;
    return true;
}
const std::vector<double> &dist_history(const DistSolver *d) { return d->conv.history; }
i64 dist_rows(const DistSolver *d) { return d->nl; }

}  // namespace xamg
