// XAMG C API (api/c/xamg_c_api.cpp:150-639 in the reference) over the B200
// solve phase, plus the extension and kernel-level entry points declared in
// include/xamg_b200.h.  Handles are indices into process-global lists and are
// never reused, as in the reference (xamg_c_api.cpp:66-85).
#include "solve.h"
#include "dist.h"
#include "batch.h"
#include "amg.h"
#include <chrono>
#include <cstdlib>
#include "../../../include/xamg_b200.h"

namespace xamg {
void gen_cube(i64 nx, i64 ny, i64 nz, int config, HostCsr &A);
void gen_27pt(i64 n, double kx, double ky, double kz, HostCsr &A);
void gen_channel_cube(int scale, bool const_rhs, int nv, HostCsr &A, std::vector<double> &b);
void gen_7pt_faces(i64 nx, i64 ny, i64 nz, const double *kx, const double *ky, const double *kz,
                   HostCsr &A);
bool read_bin(const std::string &path, HostCsr &A, std::vector<double> &b, std::vector<double> &x);
bool write_bin(const std::string &path, const HostCsr &A, const double *b, const double *x);
int mg_device_errors(MultiGrid *mg);
void gs_levels_host(const HostCsr &A, i64 brows, std::vector<int> &lf, std::vector<int> &lb);
}  // namespace xamg

using namespace xamg;

namespace {

std::string g_err;
int g_nv = 1;

struct ApiVec {
    int mode = XAMG_MEM_DISTRIBUTED;
    i64 size = 0;
    int nv = 1;
    i64 offset = 0;
    std::vector<double> host;
    DVec dev;
    bool on_device() const { return mode != XAMG_MEM_LOCAL; }
};
struct ApiCsr {
    HostCsr h;
    i64 row_off = 0, col_off = 0;
};
struct ApiMatrix {
    std::unique_ptr<Matrix> m;
};
struct ApiSolver {
    GlobalParams gp;
    std::unique_ptr<Solver> s;
    ApiMatrix *A = nullptr;
    ApiVec *x = nullptr, *b = nullptr;
    double last_ms = 0.0;
};
typedef std::map<std::string, std::string> Override;

std::vector<GlobalParams *> plist;
std::vector<Override *> ovlist;
std::vector<int> partlist;
std::vector<ApiVec *> vlist;
std::vector<ApiCsr *> mcsrlist;
std::vector<ApiMatrix *> mlist;
std::vector<ApiSolver *> slist;
std::vector<std::vector<AmgLevel> *> amglist;

template <class T> T *get(std::vector<T *> &l, size_t id, const char *what) {
    if (id >= l.size() || !l[id]) throw Error(std::string("invalid ") + what + " handle", 2);
    return l[id];
}
void check_nv(int nv) {
    if (nv != g_nv)
        throw Error("nv=" + std::to_string(nv) + " does not match the library setting " +
                        std::to_string(g_nv),
                    2);
}
// The conversions below mirror helper::xamg_param_add_value (xamg_c_api.cpp:115-128).
template <class F> int guard(F f) {
    try {
        f();
        return 0;
    } catch (const Error &e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}
void add_value(const char *role, const char *key, const PValue &v, size_t pid, bool must_exist) {
    GlobalParams *p = get(plist, pid, "param");
    std::string msg = GlobalParams::validate(key, v.t);
    if (!msg.empty()) throw Error(msg, 2);
    ParamList &l = p->roles[role];
    if (must_exist && !l.has(key)) throw Error(std::string("parameter not set: ") + key, 2);
    l.set(key, v);
}
PValue pv_s(const char *v) { PValue p; p.t = 'S'; p.s = v; return p; }
PValue pv_i(uint64_t v) { PValue p; p.t = 'I'; p.i = v; return p; }
PValue pv_f(double v) { PValue p; p.t = 'F'; p.f = v; return p; }
PValue pv_b(bool v) { PValue p; p.t = 'B'; p.b = v; return p; }

void solve_with(ApiSolver *S, ApiVec *x, ApiVec *b) {
    XCHECK(x && b && x->on_device() && b->on_device(), "solve needs device-resident x and b");
    XCHECK(x->size == S->A->m->h.n && b->size == S->A->m->h.n, "vector size differs from matrix");
    cudaStream_t st = ctx().stream;
    cudaEvent_t e0, e1;
    XCUDA(cudaEventCreate(&e0));
    XCUDA(cudaEventCreate(&e1));
    XCUDA(cudaEventRecord(e0, st));
    S->s->solve(x->dev, b->dev);
    XCUDA(cudaEventRecord(e1, st));
    XCUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    XCUDA(cudaEventElapsedTime(&ms, e0, e1));
    S->last_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    XCUDA(cudaGetLastError());
    if (MultiGrid *mg = find_multigrid(S->s.get()))
        if (mg_device_errors(mg))
            throw Error("a Gauss-Seidel sweep gave up waiting on the device (bounded wait expired)", 3);
}

cudaStream_t strm(void *s) { return s ? (cudaStream_t)s : ctx().stream; }

struct PlanHandle {
    GsPlan plan;
    HostCsr pattern;
};

}  // namespace

extern "C" {

int XAMG_id_get_proc() { return 0; }
int XAMG_id_get_nprocs() { return 1; }
void *XAMG_id_get_comm_ptr() { return nullptr; }

int XAMG_param_create(XAMG_param_id *pid) {
    return guard([&] {
        plist.push_back(new GlobalParams());
        *pid = plist.size() - 1;
    });
}
int XAMG_param_add_value_s(char *st, char *key, char *value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_s(value), pid, false); });
}
int XAMG_param_add_value_i(char *st, char *key, uint32_t value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_i(value), pid, false); });
}
int XAMG_param_add_value_d(char *st, char *key, double value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_f(value), pid, false); });
}
int XAMG_param_add_value_b(char *st, char *key, uint8_t value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_b(value != 0), pid, false); });
}
int XAMG_param_change_value_s(char *st, char *key, char *value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_s(value), pid, true); });
}
int XAMG_param_change_value_i(char *st, char *key, uint32_t value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_i(value), pid, true); });
}
int XAMG_param_change_value_d(char *st, char *key, double value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_f(value), pid, true); });
}
int XAMG_param_change_value_b(char *st, char *key, uint8_t value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_b(value != 0), pid, true); });
}
int XAMG_param_forced_change_value_s(char *st, char *key, char *value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_s(value), pid, false); });
}
int XAMG_param_forced_change_value_i(char *st, char *key, uint32_t value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_i(value), pid, false); });
}
int XAMG_param_forced_change_value_d(char *st, char *key, double value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_f(value), pid, false); });
}
int XAMG_param_forced_change_value_b(char *st, char *key, uint8_t value, XAMG_param_id pid) {
    return guard([&] { add_value(st, key, pv_b(value != 0), pid, false); });
}
void XAMG_param_set_default(XAMG_param_id pid) {
    guard([&] { get(plist, pid, "param")->set_defaults(); });
}
int XAMG_param_print(XAMG_param_id pid) {
    return guard([&] { get(plist, pid, "param")->print(); });
}
int XAMG_param_destroy(XAMG_param_id pid) {
    return guard([&] {
        if (pid < plist.size() && plist[pid]) { delete plist[pid]; plist[pid] = nullptr; }
    });
}
int XAMG_param_override_create(XAMG_param_override_id *ov) {
    return guard([&] {
        ovlist.push_back(new Override());
        *ov = ovlist.size() - 1;
    });
}
int XAMG_param_override_add_value(char *key, char *val, XAMG_param_override_id ov) {
    return guard([&] { get(ovlist, ov, "override")->insert({key, val}); });
}
int XAMG_param_override_apply(char *st, XAMG_param_id pid, XAMG_param_override_id ov) {
    return guard([&] {
        GlobalParams *p = get(plist, pid, "param");
        for (auto &kv : *get(ovlist, ov, "override")) p->overrides[st][kv.first] = kv.second;
    });
}
int XAMG_param_override_destroy(XAMG_param_override_id ov) {
    return guard([&] {
        if (ov < ovlist.size() && ovlist[ov]) { delete ovlist[ov]; ovlist[ov] = nullptr; }
    });
}

int XAMG_part_create(XAMG_part_id *pid) {
    return guard([&] {
        partlist.push_back(0);
        *pid = partlist.size() - 1;
    });
}
int XAMG_part_construct(int size, XAMG_part_id pid) {
    return guard([&] {
        XCHECK(pid < partlist.size(), "invalid part handle");
        partlist[pid] = size;
    });
}
int XAMG_part_get_numa_size(XAMG_part_id pid) {
    if (pid >= partlist.size()) { g_err = "invalid part handle"; return -1; }
    return partlist[pid];
}
int XAMG_part_destroy(XAMG_part_id pid) { return 0; }

int XAMG_vector_create(XAMG_vector_id *vid, vector_alloc_mode mode) {
    return guard([&] {
        ApiVec *v = new ApiVec();
        v->mode = mode;
        vlist.push_back(v);
        *vid = vlist.size() - 1;
    });
}
int XAMG_vector_set_part(XAMG_part_id, XAMG_vector_id vid) {
    return guard([&] { get(vlist, vid, "vector"); });
}
int XAMG_vector_offset(uint64_t off, XAMG_vector_id vid) {
    return guard([&] { get(vlist, vid, "vector")->offset = (i64)off; });
}
int XAMG_vector_alloc_d(int size, uint16_t nv, XAMG_vector_id vid) {
    return guard([&] {
        check_nv(nv);
        XCHECK(size >= 0, "negative vector size");
        ApiVec *v = get(vlist, vid, "vector");
        v->size = size;
        v->nv = nv;
        if (v->on_device()) {
            ctx();
            v->dev.alloc(size, nv, Prec::F64);
            XCUDA(cudaMemsetAsync(v->dev.p(), 0, sizeof(double) * (size_t)size * nv, ctx().stream));
        } else {
            v->host.assign((size_t)size * nv, 0.0);
        }
    });
}
int XAMG_vector_set_val_d(double val, XAMG_vector_id vid) {
    return guard([&] {
        ApiVec *v = get(vlist, vid, "vector");
        if (v->on_device()) xk::fill(Prec::F64, v->dev.count(), val, v->dev.p(), ctx().stream);
        else std::fill(v->host.begin(), v->host.end(), val);
    });
}
int XAMG_vector_upload_d(double *ptr, uint64_t bs, uint64_t bo, uint16_t nv, XAMG_vector_id vid) {
    return guard([&] {
        check_nv(nv);
        ApiVec *v = get(vlist, vid, "vector");
        i64 row = (i64)bo - v->offset;
        XCHECK(row >= 0 && row + (i64)bs <= v->size, "upload range outside the vector");
        size_t bytes = sizeof(double) * bs * nv;
        if (v->on_device()) {
            XCUDA(cudaMemcpyAsync((double *)v->dev.p() + row * nv, ptr, bytes, cudaMemcpyHostToDevice, ctx().stream));
            XCUDA(cudaStreamSynchronize(ctx().stream));
        } else {
            std::memcpy(v->host.data() + row * nv, ptr, bytes);
        }
    });
}
int XAMG_vector_download_d(double *ptr, uint64_t bs, uint64_t bo, uint16_t nv, XAMG_vector_id vid) {
    return guard([&] {
        check_nv(nv);
        ApiVec *v = get(vlist, vid, "vector");
        i64 row = (i64)bo - v->offset;
        XCHECK(row >= 0 && row + (i64)bs <= v->size, "download range outside the vector");
        size_t bytes = sizeof(double) * bs * nv;
        if (v->on_device()) {
            XCUDA(cudaMemcpyAsync(ptr, (double *)v->dev.p() + row * nv, bytes, cudaMemcpyDeviceToHost, ctx().stream));
            XCUDA(cudaStreamSynchronize(ctx().stream));
        } else {
            std::memcpy(ptr, v->host.data() + row * nv, bytes);
        }
    });
}
int XAMG_vector_upload_v(XAMG_vector_id in, XAMG_vector_id out) {
    return guard([&] {
        ApiVec *a = get(vlist, in, "vector"), *b = get(vlist, out, "vector");
        XCHECK(a->nv == b->nv, "vector widths differ");
        i64 row = a->offset - b->offset;
        XCHECK(row >= 0 && row + a->size <= b->size, "upload range outside the vector");
        size_t bytes = sizeof(double) * a->size * a->nv;
        double *dst = b->on_device() ? (double *)b->dev.p() : b->host.data();
        const double *src = a->on_device() ? (const double *)a->dev.p() : a->host.data();
        cudaMemcpyKind k = a->on_device() ? (b->on_device() ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost)
                                          : (b->on_device() ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost);
        XCUDA(cudaMemcpyAsync(dst + row * a->nv, src, bytes, k, ctx().stream));
        XCUDA(cudaStreamSynchronize(ctx().stream));
    });
}
int XAMG_vector_destroy(XAMG_vector_id vid) {
    return guard([&] {
        if (vid < vlist.size() && vlist[vid]) { delete vlist[vid]; vlist[vid] = nullptr; }
    });
}

int XAMG_csr_matrix_create(XAMG_csr_matrix_id *id) {
    return guard([&] {
        mcsrlist.push_back(new ApiCsr());
        *id = mcsrlist.size() - 1;
    });
}
int XAMG_csr_matrix_alloc(uint64_t nrows, uint64_t ncols, uint64_t nnz, XAMG_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        XCHECK(nnz < (1ull << 31), "nnz beyond the int32 index range");
        m->h.n = (i64)nrows;
        m->h.ncols = (i64)ncols;
        m->h.rp.assign(nrows + 1, 0);
        m->h.ci.assign(nnz, 0);
        m->h.v.assign(nnz, 0.0);
    });
}
// xamg_c_api.cpp:434-443: copies int rows/cols and double values
int XAMG_csr_matrix_fill(int *row, int *col, double *val, XAMG_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        i64 n = m->h.n, nnz = (i64)m->h.ci.size();
        std::memcpy(m->h.rp.data(), row, sizeof(int) * (n + 1));
        XCHECK(m->h.rp[0] == 0 && m->h.rp[n] == nnz, "row pointers do not match nnz");
        for (i64 i = 0; i < n; ++i) XCHECK(m->h.rp[i + 1] >= m->h.rp[i], "row pointers decrease");
        std::memcpy(m->h.ci.data(), col, sizeof(int) * nnz);
        for (i64 j = 0; j < nnz; ++j)
            XCHECK(m->h.ci[j] >= 0 && m->h.ci[j] < m->h.ncols, "column index out of range");
        std::memcpy(m->h.v.data(), val, sizeof(double) * nnz);
    });
}
int XAMG_csr_matrix_offset(int ro, int co, XAMG_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        m->row_off = ro;
        m->col_off = co;
    });
}
uint32_t XAMG_csr_matrix_get_nrows(XAMG_csr_matrix_id id) {
    if (id >= mcsrlist.size() || !mcsrlist[id]) return 0;
    return (uint32_t)mcsrlist[id]->h.n;
}
int XAMG_csr_matrix_destroy(XAMG_csr_matrix_id id) {
    return guard([&] {
        if (id < mcsrlist.size() && mcsrlist[id]) { delete mcsrlist[id]; mcsrlist[id] = nullptr; }
    });
}

int XAMG_matrix_create(XAMG_matrix_id *mid) {
    return guard([&] {
        mlist.push_back(new ApiMatrix());
        *mid = mlist.size() - 1;
    });
}
int XAMG_matrix_set_part(XAMG_part_id, XAMG_matrix_id mid) {
    return guard([&] { get(mlist, mid, "matrix"); });
}
int XAMG_matrix_construct(XAMG_csr_matrix_id cid, XAMG_matrix_id mid) {
    return guard([&] {
        ApiCsr *c = get(mcsrlist, cid, "csr matrix");
        ApiMatrix *m = get(mlist, mid, "matrix");
        XCHECK(c->h.n == c->h.ncols, "square matrices only");
        m->m.reset(new Matrix());
        m->m->h = c->h;
        m->m->d.upload(m->m->h, true, false);
    });
}
int XAMG_matrix_destroy(XAMG_matrix_id mid) {
    return guard([&] {
        if (mid < mlist.size() && mlist[mid]) { delete mlist[mid]; mlist[mid] = nullptr; }
    });
}

int XAMG_solver_create1(XAMG_matrix_id mid, XAMG_param_id pid, XAMG_solver_id *sid) {
    return guard([&] {
        ApiMatrix *m = get(mlist, mid, "matrix");
        XCHECK(m->m, "matrix not constructed");
        ApiSolver *S = new ApiSolver();
        S->gp = *get(plist, pid, "param");
        S->A = m;
        try {
            S->s = build_solver_tree(S->gp, *m->m, g_nv);
        } catch (...) {
            delete S;
            throw;
        }
        slist.push_back(S);
        *sid = slist.size() - 1;
    });
}
int XAMG_solver_create2(XAMG_matrix_id mid, XAMG_param_id pid, XAMG_vector_id xid,
                        XAMG_vector_id bid, XAMG_solver_id *sid) {
    int rc = XAMG_solver_create1(mid, pid, sid);
    if (rc) return rc;
    return guard([&] {
        ApiSolver *S = slist[*sid];
        S->x = get(vlist, xid, "vector");
        S->b = get(vlist, bid, "vector");
    });
}
int XAMG_solver_renew_params(XAMG_param_id pid, XAMG_solver_id sid) {
    return guard([&] {
        ApiSolver *S = get(slist, sid, "solver");
        GlobalParams *p = get(plist, pid, "param");
        // base_solver::renew_params (solver.h:211-225): the top solver's list
        // is overridden key by key; tolerances and iteration limits apply at
        // the next solve.
        std::string role = S->s->role;
        if (p->has(role))
            for (auto &kv : p->get(role).m) S->s->prm.set(kv.first, kv.second);
        S->s->conv.abs_tol = S->s->prm.has("abs_tolerance") ? S->s->prm.get_float("abs_tolerance") : 0.0;
        S->s->conv.rel_tol = S->s->prm.has("rel_tolerance") ? S->s->prm.get_float("rel_tolerance") : 0.0;
    });
}
int XAMG_solver_solve1(uint16_t nv, XAMG_solver_id sid) {
    return guard([&] {
        check_nv(nv);
        ApiSolver *S = get(slist, sid, "solver");
        XCHECK(S->x && S->b, "solver was created without x and b; use XAMG_solver_solve2");
        solve_with(S, S->x, S->b);
    });
}
int XAMG_solver_solve2(uint16_t nv, XAMG_vector_id xid, XAMG_vector_id bid, XAMG_solver_id sid) {
    return guard([&] {
        check_nv(nv);
        ApiSolver *S = get(slist, sid, "solver");
        solve_with(S, get(vlist, xid, "vector"), get(vlist, bid, "vector"));
    });
}
int XAMG_solver_print_info(XAMG_solver_id sid) {
    return guard([&] { printf("%s\n", get(slist, sid, "solver")->s->info().c_str()); });
}
int XAMG_solver_get_convergence_info(int *ci, uint16_t nv, XAMG_solver_id sid) {
    return guard([&] {
        check_nv(nv);
        Solver *s = get(slist, sid, "solver")->s.get();
        for (int k = 0; k < nv; ++k) ci[k] = k < (int)s->conv.status.size() ? s->conv.status[k] : 0;
    });
}
int XAMG_solver_get_iter_info(int *it, XAMG_solver_id sid) {
    return guard([&] {
        Solver *s = get(slist, sid, "solver")->s.get();
        it[0] = s->conv.iters;
        it[1] = s->conv.sub_iters;
    });
}
int XAMG_solver_destroy(XAMG_solver_id sid) {
    return guard([&] {
        if (sid < slist.size() && slist[sid]) { delete slist[sid]; slist[sid] = nullptr; }
    });
}

int XAMG_barrier() {
    return guard([&] { XCUDA(cudaStreamSynchronize(ctx().stream)); });
}
double XAMG_timer() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
int XAMG_get_nv() { return g_nv; }
int XAMG_init(int argc, char **argv, char *conf) {
    return guard([&] {
        const char *e = std::getenv("XAMG_NV");
        if (e) g_nv = std::atoi(e);
        ctx();
    });
}
int XAMG_finalize() {
    return guard([&] {
        for (auto &s : slist) { delete s; s = nullptr; }
        for (auto &m : mlist) { delete m; m = nullptr; }
        for (auto &c : mcsrlist) { delete c; c = nullptr; }
        for (auto &v : vlist) { delete v; v = nullptr; }
        for (auto &p : plist) { delete p; p = nullptr; }
        for (auto &o : ovlist) { delete o; o = nullptr; }
        if (ctx().stream) cudaStreamSynchronize(ctx().stream);
    });
}

// ---------------------------------------------------------------- extensions
int XAMG_b200_set_nv(int nv) {
    return guard([&] {
        XCHECK(nv == 1 || nv == 2 || nv == 4 || nv == 8 || nv == 16 || nv == 32,
               "nv must be one of 1, 2, 4, 8, 16, 32");
        g_nv = nv;
    });
}
const char *XAMG_b200_last_error(void) { return g_err.c_str(); }
int XAMG_b200_synchronize(void) {
    return guard([&] { XCUDA(cudaStreamSynchronize(ctx().stream)); });
}
void *XAMG_b200_vector_device_ptr(XAMG_vector_id vid) {
    if (vid >= vlist.size() || !vlist[vid] || !vlist[vid]->on_device()) return nullptr;
    return vlist[vid]->dev.p();
}
int XAMG_b200_solver_get_residual_history(double *out, int cap, XAMG_solver_id sid) {
    if (sid >= slist.size() || !slist[sid]) return -2;
    Solver *s = slist[sid]->s.get();
    int nv = s->conv.nv;
    int cnt = (int)(s->conv.history.size() / std::max(nv, 1));
    for (int q = 0; q < std::min(cnt, cap); ++q)
        std::memcpy(out + (size_t)q * nv, s->conv.history.data() + (size_t)q * nv, sizeof(double) * nv);
    return cnt;
}
int XAMG_b200_solver_get_res0(double *out, XAMG_solver_id sid) {
    return guard([&] {
        Solver *s = get(slist, sid, "solver")->s.get();
        for (int k = 0; k < s->conv.nv; ++k) out[k] = s->conv.res0[k];
    });
}
double XAMG_b200_solver_last_solve_ms(XAMG_solver_id sid) {
    if (sid >= slist.size() || !slist[sid]) return -1.0;
    return slist[sid]->last_ms;
}
int XAMG_b200_solver_num_levels(XAMG_solver_id sid) {
    if (sid >= slist.size() || !slist[sid]) return -2;
    MultiGrid *mg = find_multigrid(slist[sid]->s.get());
    return mg ? mg_num_levels(mg) : 0;
}
int XAMG_b200_solver_level_info(int64_t *info, int level, XAMG_solver_id sid) {
    return guard([&] {
        MultiGrid *mg = find_multigrid(get(slist, sid, "solver")->s.get());
        XCHECK(mg && level >= 0 && level < mg_num_levels(mg), "no such multigrid level");
        const HostCsr &A = mg_level_A(mg, level), &P = mg_level_P(mg, level);
        const GsPlan &g = mg_level_gs(mg, level);
        info[0] = A.n;
        info[1] = A.nnz();
        info[2] = P.n ? P.ncols : 0;
        info[3] = P.n ? P.nnz() : 0;
        info[4] = g.nlf;
        info[5] = g.nlb;
    });
}
int XAMG_b200_solver_export_level(int *rpA, int *ciA, double *vA, int *rpP, int *ciP, double *vP,
                                  int level, XAMG_solver_id sid) {
    return guard([&] {
        MultiGrid *mg = find_multigrid(get(slist, sid, "solver")->s.get());
        XCHECK(mg && level >= 0 && level < mg_num_levels(mg), "no such multigrid level");
        const HostCsr &A = mg_level_A(mg, level), &P = mg_level_P(mg, level);
        std::memcpy(rpA, A.rp.data(), sizeof(int) * (A.n + 1));
        std::memcpy(ciA, A.ci.data(), sizeof(int) * A.nnz());
        std::memcpy(vA, A.v.data(), sizeof(double) * A.nnz());
        if (P.n && rpP) {
            std::memcpy(rpP, P.rp.data(), sizeof(int) * (P.n + 1));
            std::memcpy(ciP, P.ci.data(), sizeof(int) * P.nnz());
            std::memcpy(vP, P.v.data(), sizeof(double) * P.nnz());
        }
    });
}
int XAMG_b200_solver_export_gs_levels(int *lf, int *lb, int level, XAMG_solver_id sid) {
    return guard([&] {
        MultiGrid *mg = find_multigrid(get(slist, sid, "solver")->s.get());
        XCHECK(mg && level >= 0 && level < mg_num_levels(mg), "no such multigrid level");
        const GsPlan &g = mg_level_gs(mg, level);
        XCHECK(g.n > 0, "level has no Gauss-Seidel plan");
        std::memcpy(lf, g.lf.data(), sizeof(int) * g.n);
        std::memcpy(lb, g.lb.data(), sizeof(int) * g.n);
    });
}
int XAMG_b200_solver_export_coarse_inverse(double *out, XAMG_solver_id sid) {
    return guard([&] {
        MultiGrid *mg = find_multigrid(get(slist, sid, "solver")->s.get());
        XCHECK(mg, "solver has no multigrid");
        const std::vector<double> &ci = mg_coarse_inverse(mg);
        std::memcpy(out, ci.data(), sizeof(double) * ci.size());
    });
}
int XAMG_b200_solver_level_eig(double *out, int level, XAMG_solver_id sid) {
    return guard([&] {
        MultiGrid *mg = find_multigrid(get(slist, sid, "solver")->s.get());
        XCHECK(mg, "solver has no multigrid");
        mg_level_eig(mg, level, out, out + 1);
    });
}
int XAMG_b200_solver_info(char *buf, int cap, XAMG_solver_id sid) {
    return guard([&] {
        std::string s = get(slist, sid, "solver")->s->info();
        snprintf(buf, cap, "%s", s.c_str());
    });
}

int XAMG_b200_csr_matrix_generate(int kind, const int64_t *ia, const double *da,
                                  const double *faces, XAMG_csr_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        if (kind == 0) gen_cube(ia[0], ia[1], ia[2], (int)ia[3], m->h);
        else if (kind == 1) gen_27pt(ia[0], da[0], da[1], da[2], m->h);
        else if (kind == 2) {
            i64 nx = ia[0], ny = ia[1], nz = ia[2];
            const double *kx = faces, *ky = kx + (nx + 1) * ny * nz, *kz = ky + nx * (ny + 1) * nz;
            gen_7pt_faces(nx, ny, nz, kx, ky, kz, m->h);
        } else throw Error("unknown generator kind", 2);
    });
}
int64_t XAMG_b200_channel_cube_rows(int scale) {
    if (scale == 1) return (int64_t)144 * 112 * 144;
    if (scale == 2) return (int64_t)240 * 168 * 240;
    if (scale == 3) return (int64_t)360 * 252 * 360;
    return -1;
}
int XAMG_b200_generate_channel_cube(int scale, int const_rhs, int nv, double *b_out, XAMG_csr_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        XCHECK(nv >= 1 && nv <= 64, "nv must be 1..64");
        std::vector<double> b;
        gen_channel_cube(scale, const_rhs != 0, nv, m->h, b);
        if (b_out) std::memcpy(b_out, b.data(), sizeof(double) * b.size());
    });
}
int64_t XAMG_b200_csr_matrix_get_nnz(XAMG_csr_matrix_id id) {
    if (id >= mcsrlist.size() || !mcsrlist[id]) return -1;
    return mcsrlist[id]->h.nnz();
}
int XAMG_b200_csr_matrix_export(int *rp, int *ci, double *v, XAMG_csr_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        std::memcpy(rp, m->h.rp.data(), sizeof(int) * (m->h.n + 1));
        std::memcpy(ci, m->h.ci.data(), sizeof(int) * m->h.nnz());
        std::memcpy(v, m->h.v.data(), sizeof(double) * m->h.nnz());
    });
}
int XAMG_b200_csr_matrix_read_bin(const char *path, double *b_out, double *x_out,
                                  XAMG_csr_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        std::vector<double> b, x;
        XCHECK(read_bin(path, m->h, b, x), std::string("cannot read ") + path);
        if (b_out && !b.empty()) std::memcpy(b_out, b.data(), sizeof(double) * b.size());
        if (x_out && !x.empty()) std::memcpy(x_out, x.data(), sizeof(double) * x.size());
    });
}
int XAMG_b200_csr_matrix_write_bin(const char *path, const double *b, const double *x,
                                   XAMG_csr_matrix_id id) {
    return guard([&] {
        ApiCsr *m = get(mcsrlist, id, "csr matrix");
        XCHECK(write_bin(path, m->h, b, x), std::string("cannot write ") + path);
    });
}

// ---------------------------------------------------------------- host setup
// The AMG hierarchy of the MultiGrid role in pid, built on the host only.
int XAMG_b200_amg_host_create(XAMG_csr_matrix_id cid, XAMG_param_id pid, size_t *hid) {
    return guard([&] {
        ApiCsr *c = get(mcsrlist, cid, "csr matrix");
        GlobalParams *p = get(plist, pid, "param");
        const char *role = nullptr;
        for (const char *r : {"preconditioner", "solver"})
            if (p->has(r) && p->get(r).has("method") && p->get(r).get_string("method") == "MultiGrid")
                role = r;
        XCHECK(role, "no MultiGrid role in the parameter list");
        std::vector<AmgParams> ap = amg_params_for(*p, role);
        auto *h = new std::vector<AmgLevel>();
        amg_setup(c->h, ap, *h);
        amglist.push_back(h);
        *hid = amglist.size() - 1;
    });
}
int XAMG_b200_amg_host_num_levels(size_t hid) {
    if (hid >= amglist.size() || !amglist[hid]) return -2;
    return (int)amglist[hid]->size();
}
int XAMG_b200_amg_host_level_info(int64_t *info, int l, size_t hid) {
    return guard([&] {
        auto *h = get(amglist, hid, "hierarchy");
        XCHECK(l >= 0 && l < (int)h->size(), "no such level");
        const AmgLevel &L = (*h)[l];
        info[0] = L.A.n;
        info[1] = L.A.nnz();
        info[2] = L.P.n ? L.P.ncols : 0;
        info[3] = L.P.n ? L.P.nnz() : 0;
    });
}
int XAMG_b200_amg_host_export_level(int *rpA, int *ciA, double *vA, int *rpP, int *ciP,
                                    double *vP, int l, size_t hid) {
    return guard([&] {
        auto *h = get(amglist, hid, "hierarchy");
        XCHECK(l >= 0 && l < (int)h->size(), "no such level");
        const AmgLevel &L = (*h)[l];
        std::memcpy(rpA, L.A.rp.data(), sizeof(int) * (L.A.n + 1));
        std::memcpy(ciA, L.A.ci.data(), sizeof(int) * L.A.nnz());
        std::memcpy(vA, L.A.v.data(), sizeof(double) * L.A.nnz());
        if (L.P.n && rpP) {
            std::memcpy(rpP, L.P.rp.data(), sizeof(int) * (L.P.n + 1));
            std::memcpy(ciP, L.P.ci.data(), sizeof(int) * L.P.nnz());
            std::memcpy(vP, L.P.v.data(), sizeof(double) * L.P.nnz());
        }
    });
}
int XAMG_b200_amg_host_destroy(size_t hid) {
    return guard([&] {
        if (hid < amglist.size() && amglist[hid]) { delete amglist[hid]; amglist[hid] = nullptr; }
    });
}
// Wavefront levels of the forward/backward Gauss-Seidel sweeps (host arrays).
int XAMG_b200_gs_levels_host(int64_t n, const int *rp, const int *ci, int64_t block_rows,
                             int *lf, int *lb, int *nlev) {
    return guard([&] {
        HostCsr A;
        A.n = A.ncols = n;
        A.rp.assign(rp, rp + n + 1);
        A.ci.assign(ci, ci + rp[n]);
        std::vector<int> f, b;
        gs_levels_host(A, block_rows, f, b);
        std::memcpy(lf, f.data(), sizeof(int) * n);
        std::memcpy(lb, b.data(), sizeof(int) * n);
        int mf = 0, mb = 0;
        for (int v : f) mf = std::max(mf, v + 1);
        for (int v : b) mb = std::max(mb, v + 1);
        nlev[0] = mf;
        nlev[1] = mb;
    });
}

// ---------------------------------------------------------------- kernels
int xamg_csr_spmv(int prec, int nv, int64_t n, const int *rp, const int *ci, const void *val,
                  const void *x, void *y, int mode, const void *b, void *stream) {
    return guard([&] {
        XCHECK(mode >= 0 && mode <= 2, "mode must be 0, 1 or 2");
        XCHECK(mode != 2 || b, "mode 2 needs b");
        xk::spmv((Prec)prec, nv, n, rp, ci, val, x, y, mode, b, strm(stream));
        XCUDA(cudaGetLastError());
    });
}
int xamg_spmv_set_variant(int variant) {
    int old = xk::get_spmv_variant();
    xk::set_spmv_variant(variant);
    return old;
}
int xamg_spmv_set_run_form(int form) {
    int old = xk::get_spmv_run_form();
    xk::set_spmv_run_form(form);
    return old;
}
int xamg_spmv_set_run_rows(int rows) {
    int old = xk::get_spmv_run_rows();
    xk::set_spmv_run_rows(rows);
    return old;
}
void *xamg_spmv_runs_plan_create(int64_t n, const int *rp, const int *ci, const double *val, int rows, int fp32) {
    RunPlan *h = nullptr;
    int rc = guard([&] {
        XCHECK(n > 0 && rp && ci && val, "bad CSR arrays");
        XCHECK(rows == 8, "rows must be 8");
        ctx();
        HostCsr A;
        A.n = A.ncols = n;
        A.rp.assign(rp, rp + n + 1);
        A.ci.assign(ci, ci + rp[n]);
        A.v.assign(val, val + rp[n]);
        h = new RunPlan();
        XCHECK(h->build(A, rows, true, fp32 != 0, 0.0), "run plan not built");
    });
    if (rc) { delete h; return nullptr; }
    return h;
}
int xamg_spmv_runs_analyze(int64_t n, const int *rp, const int *ci, int rows, int64_t *nchunks, double *coverage,
                           int64_t *segments) {
    return guard([&] {
        XCHECK(n >= 0 && rp && (n == 0 || ci) && nchunks && coverage && segments, "bad arguments");
        XCHECK(rows == 8, "rows must be 8");
        i64 nc = 0, ns = 0;
        run_plan_analyze(n, rp, ci, rows, &nc, coverage, &ns);
        *nchunks = nc;
        *segments = ns;
    });
}
int xamg_spmv_runs_plan_info(void *plan, int64_t *nchunks, double *coverage, int64_t *segments,
                             int64_t *value_slots) {
    return guard([&] {
        XCHECK(plan, "null plan");
        RunPlan *h = (RunPlan *)plan;
        if (coverage) *coverage = h->coverage;
        if (nchunks) {  // chunks holding rows (the padding excluded)
            int64_t k = 0;
            for (i64 c = 0; c < h->nchunks; ++c) k += h->hchunks[(size_t)c * 4 + 1] > 0;
            *nchunks = k;
        }
        if (segments) {
            int64_t s = 0;
            for (i64 c = 0; c < h->nchunks; ++c) s += h->hchunks[(size_t)c * 4 + 3];
            *segments = s;
        }
        if (value_slots) *value_slots = h->hvoff.empty() ? 0 : h->hvoff.back() * h->R;
    });
}
int xamg_spmv_runs(void *plan, int prec, int nv, const void *x, void *y, int mode, const void *b, void *stream) {
    return guard([&] {
        XCHECK(plan, "null plan");
        RunPlan *h = (RunPlan *)plan;
        XCHECK(prec == 0 || prec == 1, "prec must be 0 or 1");
        XCHECK(mode >= 0 && mode <= 2, "mode must be 0, 1 or 2");
        XCHECK(mode != 2 || b, "mode 2 needs b");
        XCHECK(xk::spmv_runs_supported((Prec)prec, nv), "shape not supported (FP64 nv 8, 16, 32; FP32 nv 16, 32)");
        XCHECK(h->has((Prec)prec), "plan has no values in this precision");
        xk::spmv_runs((Prec)prec, nv, h->nchunks, h->ntiles, h->chunks.as<int4>(), h->toff.as<longlong2>(),
                      h->sg.as<int>(), prec == 0 ? h->v64.p : h->v32.p, x, y, mode, b, strm(stream));
        XCUDA(cudaGetLastError());
    });
}
int xamg_spmv_runs_plan_destroy(void *plan) {
    return guard([&] { delete (RunPlan *)plan; });
}
void *xamg_gs_plan_create(int64_t n, const int *rp, const int *ci, int64_t block_rows,
                          int schedule) {
    PlanHandle *h = nullptr;
    int rc = guard([&] {
        ctx();
        HostCsr A;
        A.n = A.ncols = n;
        A.rp.assign(rp, rp + n + 1);
        A.ci.assign(ci, ci + rp[n]);
        h = new PlanHandle();
        GsMode md = schedule == 0 ? GsMode::LEVELS : (schedule == 2 ? GsMode::GRID : gs_mode_from("auto", block_rows, n));
        h->plan.build(A, block_rows, md);
        h->pattern = std::move(A);
    });
    if (rc) { delete h; return nullptr; }
    return h;
}
int xamg_gs_plan_set_values(void *plan, const double *val_host, int prec) {
    return guard([&] {
        XCHECK(plan, "null plan");
        PlanHandle *h = (PlanHandle *)plan;
        h->pattern.v.assign(val_host, val_host + h->pattern.nnz());
        h->plan.build_lcsr(h->pattern, (Prec)prec);
    });
}
int xamg_gs_plan_levels(void *plan, int *nlev, int *lf, int *lb) {
    return guard([&] {
        XCHECK(plan, "null plan");
        GsPlan &g = ((PlanHandle *)plan)->plan;
        nlev[0] = g.nlf;
        nlev[1] = g.nlb;
        if (lf) std::memcpy(lf, g.lf.data(), sizeof(int) * g.n);
        if (lb) std::memcpy(lb, g.lb.data(), sizeof(int) * g.n);
    });
}
int xamg_gs_plan_slots(void *plan, int *nslots) {
    return guard([&] {
        XCHECK(plan, "null plan");
        GsPlan &g = ((PlanHandle *)plan)->plan;
        nslots[0] = g.has_lcsr ? g.lc[0].nslots : 0;
        nslots[1] = g.has_lcsr ? g.lc[1].nslots : 0;
    });
}
int XAMG_b200_wait_selftest(int which, int ncta, double limit_s) {
    return guard([&] {
        XCHECK(which == 0 || which == 1, "which must be 0 (grid barrier) or 1 (mbarrier)");
        XCHECK(ncta >= 2 && ncta <= 64, "ncta must be 2..64");
        XCHECK(limit_s > 0.0 && limit_s <= 2.0, "limit must be in (0, 2] seconds");
        cudaStream_t s = ctx().stream;
        DBuf words(256), err(sizeof(int));
        XCUDA(xk::wait_selftest(which, ncta, (unsigned long long)(limit_s * 1e9), words.as<unsigned>(),
                                err.as<int>(), s));
        XCUDA(cudaStreamSynchronize(s));
        int h = 0;
        XCUDA(cudaMemcpy(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) throw Error(std::string(which == 0 ? "grid barrier" : "mbarrier") +
                               ": bounded wait expired on the device (error word " + std::to_string(h) + ")",
                           3);
    });
}
int xamg_gs_plan_error(void *plan) {
    if (!plan) return -1;
    return ((PlanHandle *)plan)->plan.error_flag();
}
void xamg_gs_plan_destroy(void *plan) { delete (PlanHandle *)plan; }
int xamg_hsgs(void *plan, int prec, int nv, const int *rp, const int *ci, const void *val,
              const void *invd, const void *b, void *x, const void *relax, void *t, void *stream) {
    return guard([&] {
        XCHECK(plan, "null plan");
        GsPlan &g = ((PlanHandle *)plan)->plan;
        cudaStream_t s = strm(stream);
        const void *tp = b;
        if (g.brows > 0 && g.brows < g.n) {
            XCHECK(t, "hybrid plans need t_scratch");
            xk::offblock_resid((Prec)prec, nv, g.n, rp, ci, val, b, x, t, g.brows, s);
            tp = t;
        }
        g.sweep((Prec)prec, nv, rp, ci, val, invd, tp, x, relax, true, s);
        g.sweep((Prec)prec, nv, rp, ci, val, invd, tp, x, relax, false, s);
        XCUDA(cudaGetLastError());
    });
}
int xamg_jacobi(int prec, int nv, int64_t n, const int *rp, const int *ci, const void *val,
                const void *invd, const void *b, const void *xi, void *xo, const void *relax,
                void *stream) {
    return guard([&] {
        xk::jacobi((Prec)prec, nv, n, rp, ci, val, invd, b, xi, xo, relax, strm(stream));
        XCUDA(cudaGetLastError());
    });
}
int64_t xamg_dot_part_size(int64_t n, int nd, int nv) { return xk::dot_part_size(n, nd, nv); }
int xamg_dot(int prec, int nv, int64_t n, int nd, const void *const *a, const void *const *b,
             double *part, double *out, void *stream) {
    return guard([&] {
        XCHECK(nd >= 1 && nd <= 4, "nd must be 1..4");
        xk::dots((Prec)prec, nv, n, nd, a, b, part, out, strm(stream));
        XCUDA(cudaGetLastError());
    });
}
int xamg_seg_dot(int prec, int nv, int nseg, const int64_t *segoff, int nd, const void *const *a,
                 const void *const *b, double *out, void *stream) {
    return guard([&] {
        XCHECK(nd >= 1 && nd <= 3, "nd must be 1..3");
        XCHECK(nseg >= 1 && segoff && segoff[0] == 0, "segoff must start at 0 and hold nseg + 1 offsets");
        XCHECK(nv == 1 || nv == 2 || nv == 4 || nv == 8 || nv == 16 || nv == 32, "nv must be 1, 2, 4, 8, 16 or 32");
        std::vector<i64> off(segoff, segoff + nseg + 1), cs(1, 0);
        for (int k = 0; k < nseg; ++k) {
            XCHECK(off[k + 1] >= off[k], "segoff must not decrease");
            cs.push_back(cs.back() + (off[k + 1] - off[k] + 255) / 256);
        }
        cudaStream_t s = strm(stream);
        DBuf so(sizeof(i64) * off.size()), cst(sizeof(i64) * cs.size()),
            part(sizeof(double) * std::max<i64>(cs.back() * nd * nv, 1));
        XCUDA(cudaMemcpyAsync(so.p, off.data(), sizeof(i64) * off.size(), cudaMemcpyHostToDevice, s));
        XCUDA(cudaMemcpyAsync(cst.p, cs.data(), sizeof(i64) * cs.size(), cudaMemcpyHostToDevice, s));
        xk::seg_dots((Prec)prec, nv, nseg, so.as<i64>(), cst.as<i64>(), cs.back(), nd, a, b, part.as<double>(), out,
                     s);
        XCUDA(cudaGetLastError());
        XCUDA(cudaStreamSynchronize(s));  // the scratch is released on return
    });
}
int xamg_blas(int prec, int nv, int64_t n, int op, const double *a, const void *x, const double *b,
              const void *y, const double *c, void *z, void *stream) {
    return guard([&] {
        XCHECK(op >= 0 && op <= 6, "op must be 0..6");
        xk::blas((Prec)prec, nv, n, (xk::Op)op, a, x, b, y, c, z, strm(stream));
        XCUDA(cudaGetLastError());
    });
}
int xamg_dense_gemv(int prec, int nv, int n, const void *AinvT, const void *b, void *y,
                    void *stream) {
    return guard([&] {
        xk::dense_gemv((Prec)prec, nv, n, AinvT, b, y, strm(stream));
        XCUDA(cudaGetLastError());
    });
}

}  // extern "C"

namespace xamg {
// Record the text returned by XAMG_b200_last_error() (used by entry points
// that live outside this file).
void set_last_error(const std::string &msg) { g_err = msg; }
// The stream that a NULL stream argument means for every kernel-level entry
// point: the library's own non-blocking stream (created on first use; a
// stream holds no device allocation of this library).
cudaStream_t library_stream() { return ctx().stream; }
}  // namespace xamg

// ---- batching form (no counterpart in the reference) -----------------------
static std::vector<Batch *> blist;

extern "C" {
int XAMG_b200_batch_create(int nsys, const int64_t *n, const int *const *rp, const int *const *ci,
                           const double *const *val, const int *nv, XAMG_param_id pid, size_t *bid) {
    return guard([&] {
        XCHECK(n && rp && ci && val && nv && bid, "null argument");
        std::unique_ptr<Batch> B(new Batch());
        std::vector<i64> nn(n, n + nsys);
        B->create(nsys, nn.data(), rp, ci, val, nv, *get(plist, pid, "param"));
        blist.push_back(B.release());
        *bid = blist.size() - 1;
    });
}
int XAMG_b200_batch_upload(size_t bid, int sys, const double *b, const double *x0) {
    return guard([&] { get(blist, bid, "batch")->upload(sys, b, x0); });
}
int XAMG_b200_batch_set_graph(size_t bid, int use_graph) {
    return guard([&] { get(blist, bid, "batch")->use_graph = use_graph != 0; });
}
int XAMG_b200_batch_solve(size_t bid) {
    return guard([&] { get(blist, bid, "batch")->solve(); });
}
int XAMG_b200_batch_download(size_t bid, int sys, double *x) {
    return guard([&] { get(blist, bid, "batch")->download(sys, x); });
}
int XAMG_b200_batch_stats(size_t bid, int sys, int *iters, double *relres) {
    return guard([&] { get(blist, bid, "batch")->stats(sys, iters, relres); });
}
double XAMG_b200_batch_last_ms(size_t bid) {
    if (bid >= blist.size() || !blist[bid]) return -1.0;
    return blist[bid]->last_ms;
}
long long XAMG_b200_batch_last_kernels(size_t bid) {
    if (bid >= blist.size() || !blist[bid]) return -1;
    return blist[bid]->last_kernels;
}
long long XAMG_b200_kernel_launches(void) { return xk::launch_count(); }
int XAMG_b200_kernel_timing(int on) { return ktime_enable(on); }
int XAMG_b200_gs_sweep_kernel(void) { return gs_warp_sweep(); }
int XAMG_b200_kernel_timing_read(int cap, int *kclass, int64_t *rows, int64_t *launches, double *ms,
                                 double *bytes) {
    int g = -1;
    int rc = guard([&] { g = ktime_read(cap, kclass, rows, launches, ms, bytes); });
    return rc ? -rc : g;
}
int XAMG_b200_batch_groups(size_t bid, int *out, int cap) {
    if (bid >= blist.size() || !blist[bid]) return -2;
    const Batch *B = blist[bid];
    int g = 0;
    for (auto &G : B->groups) {
        if (out && 4 * g + 3 < cap) {
            out[4 * g] = G->nv;
            out[4 * g + 1] = (int)G->sys.size();
            out[4 * g + 2] = G->var64;
            out[4 * g + 3] = G->var32;
        }
        ++g;
    }
    return g;
}
int XAMG_b200_batch_destroy(size_t bid) {
    return guard([&] {
        Batch *B = get(blist, bid, "batch");
        delete B;
        blist[bid] = nullptr;
    });
}

// ---------------------------------------------------------------- row partition
static std::vector<RowPart *> rplist;
int XAMG_b200_rowpart_create(int64_t n, const int *rp, const int *ci, int nranks, int rank, size_t *id) {
    return guard([&] {
        XCHECK(rp && ci && id && n > 0, "bad arguments");
        std::unique_ptr<RowPart> P(new RowPart());
        P->build(n, rp, ci, nranks, rank);
        rplist.push_back(P.release());
        *id = rplist.size() - 1;
    });
}
int XAMG_b200_rowpart_info(size_t id, int64_t *out) {
    return guard([&] {
        RowPart *P = get(rplist, id, "row partition");
        out[0] = P->first[P->rank];
        out[1] = P->nrows();
        out[2] = (int64_t)P->lci.size();
        out[3] = (int64_t)P->halo.size();
    });
}
int XAMG_b200_rowpart_local_csr(size_t id, int *rp_out, int *ci_out, int64_t *src_out) {
    return guard([&] {
        RowPart *P = get(rplist, id, "row partition");
        std::memcpy(rp_out, P->lrp.data(), sizeof(int) * P->lrp.size());
        if (!P->lci.empty()) std::memcpy(ci_out, P->lci.data(), sizeof(int) * P->lci.size());
        if (src_out && !P->lsrc.empty()) std::memcpy(src_out, P->lsrc.data(), sizeof(int64_t) * P->lsrc.size());
    });
}
int XAMG_b200_rowpart_halo(size_t id, int64_t *rows_out, int *owner_out) {
    return guard([&] {
        RowPart *P = get(rplist, id, "row partition");
        for (size_t h = 0; h < P->halo.size(); ++h) {
            if (rows_out) rows_out[h] = P->halo[h];
            if (owner_out) owner_out[h] = P->halo_owner[h];
        }
    });
}
int XAMG_b200_rowpart_sends(size_t id, int peer, int64_t *rows_out, int64_t *count) {
    return guard([&] {
        RowPart *P = get(rplist, id, "row partition");
        XCHECK(peer >= 0 && peer < P->nranks, "bad peer");
        const std::vector<i64> &v = P->sends[peer];
        *count = (int64_t)v.size();
        if (rows_out)
            for (size_t k = 0; k < v.size(); ++k) rows_out[k] = v[k];
    });
}
int XAMG_b200_rowpart_destroy(size_t id) {
    return guard([&] {
        RowPart *P = get(rplist, id, "row partition");
        delete P;
        rplist[id] = nullptr;
    });
}
}  // extern "C"

// ---- row-partitioned multi-GPU solve (an extension; the reference's
// MPI-distributed solve) ------------------------------------------------------
namespace xamg {
struct DistSolver;
void dist_unique_id(void *out);
DistSolver *dist_create(const void *uid, const RowPart &part, const double *val_global, const GlobalParams &gp,
                        int nv);
void dist_solve(DistSolver *d, const double *b, double *x);
void dist_destroy(DistSolver *d);
int dist_iters(const DistSolver *d);
bool dist_converged(const DistSolver *d);
const std::vector<double> &dist_history(const DistSolver *d);
i64 dist_rows(const DistSolver *d);
}  // namespace xamg
static std::vector<DistSolver *> dlist;

extern "C" {
int XAMG_b200_dist_unique_id(void *out) {
    return guard([&] {
        XCHECK(out, "null argument");
        dist_unique_id(out);
    });
}
int XAMG_b200_dist_create(const void *uid, size_t rowpart_id, const double *val_global, XAMG_param_id pid, int nv,
                          size_t *did) {
    return guard([&] {
        RowPart *P = get(rplist, rowpart_id, "row partition");
        GlobalParams *gp = get(plist, pid, "param");
        XCHECK(uid && val_global && did, "null argument");
        XCHECK(nv == 1 || nv == 2 || nv == 4 || nv == 8 || nv == 16 || nv == 32, "nv must be 1, 2, 4, 8, 16 or 32");
        dlist.push_back(dist_create(uid, *P, val_global, *gp, nv));
        *did = dlist.size() - 1;
    });
}
int XAMG_b200_dist_solve(size_t did, const double *b_dev, double *x_dev) {
    return guard([&] {
        DistSolver *d = get(dlist, did, "distributed solver");
        XCHECK(b_dev && x_dev, "null argument");
        dist_solve(d, b_dev, x_dev);
    });
}
int XAMG_b200_dist_info(size_t did, int64_t *out) {
    return guard([&] {
        DistSolver *d = get(dlist, did, "distributed solver");
        out[0] = dist_iters(d);
        out[1] = dist_converged(d) ? 1 : 0;
        out[2] = dist_rows(d);
        out[3] = (int64_t)dist_history(d).size();
    });
}
int XAMG_b200_dist_history(size_t did, double *out, int64_t cap) {
    return guard([&] {
        DistSolver *d = get(dlist, did, "distributed solver");
        const auto &h = dist_history(d);
        for (size_t k = 0; k < h.size() && (int64_t)k < cap; ++k) out[k] = h[k];
    });
}
int XAMG_b200_dist_destroy(size_t did) {
    return guard([&] {
        DistSolver *d = get(dlist, did, "distributed solver");
        dist_destroy(d);
        dlist[did] = nullptr;
    });
}
}  // extern "C"
