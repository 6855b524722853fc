// Device objects and solver drivers of the XAMG B200 solve phase.
#include "solve.h"
#include "amg.h"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <set>
#include <tuple>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace xamg {


Context &ctx() {
    static Context c;
    c.init();
    return c;
}

static bool quiet() { return std::getenv("XAMG_QUIET") != nullptr; }

// ------------------------------------------------------------ kernel timing
namespace {
struct KRec {
    int kclass;
    i64 rows;
    double bytes;
    cudaEvent_t e0, e1;
};
bool g_ktime = false;
std::vector<KRec> g_krecs;
std::vector<cudaEvent_t> g_kpool;
cudaEvent_t kevent() {
    if (!g_kpool.empty()) {
        cudaEvent_t e = g_kpool.back();
        g_kpool.pop_back();
        return e;
    }
    cudaEvent_t e;
    XCUDA(cudaEventCreate(&e));
    return e;
}
void kclear() {
    for (KRec &r : g_krecs) {
        g_kpool.push_back(r.e0);
        g_kpool.push_back(r.e1);
    }
    g_krecs.clear();
}
}  // namespace

bool ktime_on() { return g_ktime; }

KTimeScope::KTimeScope(KClass k, i64 rows, double bytes, cudaStream_t st) : on(g_ktime), s(st) {
    if (!on) return;
    KRec r{(int)k, rows, bytes, kevent(), kevent()};
    XCUDA(cudaEventRecord(r.e0, s));
    slot = (int)g_krecs.size();
    g_krecs.push_back(r);
}
KTimeScope::~KTimeScope() {
    if (on && slot >= 0) cudaEventRecord(g_krecs[slot].e1, s);
}

int ktime_enable(int on) {
    int old = g_ktime;
    if (!on) kclear();
    g_ktime = on != 0;
    return old;
}

// Aggregate the records by (class, rows) after the device has finished them;
// clears the records.  Returns the number of groups written (at most cap).
int ktime_read(int cap, int *kclass, i64 *rows, i64 *launches, double *ms, double *bytes) {
    XCUDA(cudaDeviceSynchronize());
    std::map<std::pair<int, i64>, std::tuple<i64, double, double>> agg;
    for (KRec &r : g_krecs) {
        float t = 0.f;
        XCUDA(cudaEventElapsedTime(&t, r.e0, r.e1));
        auto &a = agg[{r.kclass, r.rows}];
        std::get<0>(a) += 1;
        std::get<1>(a) += t;
        std::get<2>(a) += r.bytes;
    }
    kclear();
    int g = 0;
    for (auto &kv : agg) {
        if (g >= cap) break;
        kclass[g] = kv.first.first;
        rows[g] = kv.first.second;
        launches[g] = std::get<0>(kv.second);
        ms[g] = std::get<1>(kv.second);
        bytes[g] = std::get<2>(kv.second);
        ++g;
    }
    return g;
}

static int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        XCUDA(cudaGetDevice(&dev));
        XCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (sms <= 0) sms = 148;
    }
    return sms;
}

// ------------------------------------------------------------------ DCsr
void DCsr::upload(const HostCsr &h, bool f64, bool f32) {
    cudaStream_t s = ctx().stream;
    n = h.n;
    ncols = h.ncols;
    nnz = h.nnz();
    rp.alloc(sizeof(int) * (n + 1));
    ci.alloc(sizeof(int) * std::max<i64>(nnz, 1));
    XCUDA(cudaMemcpyAsync(rp.p, h.rp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    if (nnz) XCUDA(cudaMemcpyAsync(ci.p, h.ci.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    if (f64) {
        v64.alloc(sizeof(double) * std::max<i64>(nnz, 1));
        if (nnz) XCUDA(cudaMemcpyAsync(v64.p, h.v.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    if (f32) {
        std::vector<float> f(h.v.begin(), h.v.end());
        v32.alloc(sizeof(float) * std::max<i64>(nnz, 1));
        if (nnz) XCUDA(cudaMemcpyAsync(v32.p, f.data(), sizeof(float) * nnz, cudaMemcpyHostToDevice, s));
        XCUDA(cudaStreamSynchronize(s));
    }
    XCUDA(cudaStreamSynchronize(s));
    // shifted-row run plan for large square operators whose rows mostly form
    // runs (stencil operators); irregular operators keep only the CSR arrays
    runs.clear();
    const int R = xk::get_spmv_run_rows();
    if (R > 0 && n >= 4096) runs.build(h, R, f64, f32, 0.5);
}

void Matrix::ensure32() {
    if (has32) return;
    std::vector<float> f(h.v.begin(), h.v.end());
    d.v32.alloc(sizeof(float) * std::max<i64>(d.nnz, 1));
    if (d.nnz)
        XCUDA(cudaMemcpy(d.v32.p, f.data(), sizeof(float) * d.nnz, cudaMemcpyHostToDevice));
    d.runs.add_values(h, Prec::F32);
    has32 = true;
}

// inverse diagonal, csr_matrix.h:344-349 (last diagonal entry wins; the FP32
// copy is 1.0/(double)(float)a_ii rounded to float)
static void make_invd(const HostCsr &A, bool f64, bool f32, DBuf &d64, DBuf &d32) {
    std::vector<double> i64v(A.n, 0.0);
    std::vector<float> i32v(A.n, 0.f);
    for (i64 i = 0; i < A.n; ++i)
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j)
            if (A.ci[j] == i) {
                i64v[i] = 1.0 / A.v[j];
                i32v[i] = (float)(1.0 / (double)(float)A.v[j]);
            }
    if (f64) {
        d64.alloc(sizeof(double) * std::max<i64>(A.n, 1));
        XCUDA(cudaMemcpy(d64.p, i64v.data(), sizeof(double) * A.n, cudaMemcpyHostToDevice));
    }
    if (f32) {
        d32.alloc(sizeof(float) * std::max<i64>(A.n, 1));
        XCUDA(cudaMemcpy(d32.p, i32v.data(), sizeof(float) * A.n, cudaMemcpyHostToDevice));
    }
}

// ------------------------------------------------------------------ GsPlan
// Wavefront levels (one pass over the CSR, O(nnz)): row i's forward level is
// one more than the largest level of any j < i that row i reads or that reads
// row i; rows of equal level are independent and all their dependencies are
// resolved in the sequential order.  The backward schedule mirrors it.
void gs_levels_host(const HostCsr &A, i64 brows, std::vector<int> &lf, std::vector<int> &lb) {
    i64 n = A.n;
    auto inblk = [&](i64 i, i64 c) { return brows <= 0 || (c / brows) == (i / brows); };
    lf.assign(n, 0);
    lb.assign(n, 0);
    std::vector<int> pend(n, 0);
    for (i64 i = 0; i < n; ++i) {
        int L = pend[i];
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            i64 c = A.ci[j];
            if (c < i && inblk(i, c)) L = std::max(L, lf[c] + 1);
        }
        lf[i] = L;
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            i64 c = A.ci[j];
            if (c > i && inblk(i, c)) pend[c] = std::max(pend[c], L + 1);
        }
    }
    std::fill(pend.begin(), pend.end(), 0);
    for (i64 i = n - 1; i >= 0; --i) {
        int L = pend[i];
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            i64 c = A.ci[j];
            if (c > i && inblk(i, c)) L = std::max(L, lb[c] + 1);
        }
        lb[i] = L;
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            i64 c = A.ci[j];
            if (c < i && inblk(i, c)) pend[c] = std::max(pend[c], L + 1);
        }
    }
}

GsMode gs_mode_from(const std::string &s, i64 brows, i64 n) {
    bool hybrid = brows > 0 && brows < n;
    if (s == "levels") return GsMode::LEVELS;
    if (s == "grid" || s == "persistent") return GsMode::GRID;
    if (s == "blocks") return hybrid ? GsMode::BLOCKS : GsMode::GRID;
    return hybrid ? GsMode::BLOCKS : GsMode::GRID;  // auto
}

static void upload_ints(DBuf &d, const std::vector<int> &h) {
    d.alloc(sizeof(int) * std::max<size_t>(h.size(), 1));
    if (!h.empty()) XCUDA(cudaMemcpy(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
}

void GsPlan::build(const HostCsr &A, i64 brows_, GsMode mode_) {
    n = A.n;
    brows = brows_ > 0 && brows_ < A.n ? brows_ : 0;
    mode = mode_;
    if (mode == GsMode::BLOCKS && brows == 0) mode = GsMode::GRID;
    gs_levels_host(A, brows, lf, lb);
    if (mode == GsMode::BLOCKS) {
        // rows of each block in (level, row) order; levels of block b are the
        // consecutive entries [blev[b], blev[b+1]) of lptr
        nblocks = (int)((n + brows - 1) / brows);
        auto bsched = [&](const std::vector<int> &lev, DBuf &dblev, DBuf &dlptr, DBuf &dperm) {
            std::vector<int> blev(nblocks + 1, 0), lptr, perm(n);
            lptr.push_back(0);
            for (int b = 0; b < nblocks; ++b) {
                i64 r0 = (i64)b * brows, r1 = std::min<i64>(n, r0 + brows);
                int nl = 0;
                for (i64 i = r0; i < r1; ++i) nl = std::max(nl, lev[i] + 1);
                std::vector<int> cnt(nl + 1, 0);
                for (i64 i = r0; i < r1; ++i) cnt[lev[i] + 1]++;
                for (int l = 0; l < nl; ++l) cnt[l + 1] += cnt[l];
                std::vector<int> pos(cnt.begin(), cnt.end() - 1);
                for (i64 i = r0; i < r1; ++i) perm[r0 + pos[lev[i]]++] = (int)i;
                for (int l = 0; l < nl; ++l) lptr.push_back((int)(r0 + cnt[l + 1]));
                blev[b + 1] = blev[b] + nl;
            }
            upload_ints(dblev, blev);
            upload_ints(dlptr, lptr);
            upload_ints(dperm, perm);
        };
        bsched(lf, bblevf, blptrf, bpermf);
        bsched(lb, bblevb, blptrb, bpermb);
    }
    auto sched = [&](const std::vector<int> &lev, std::vector<int> &lptr, DBuf &dperm, DBuf &dlptr) {
        int nl = 0;
        for (i64 i = 0; i < n; ++i) nl = std::max(nl, lev[i] + 1);
        lptr.assign(nl + 1, 0);
        for (i64 i = 0; i < n; ++i) lptr[lev[i] + 1]++;
        for (int l = 0; l < nl; ++l) lptr[l + 1] += lptr[l];
        std::vector<int> pos(lptr.begin(), lptr.end() - 1), perm(std::max<i64>(n, 1));
        for (i64 i = 0; i < n; ++i) perm[pos[lev[i]]++] = (int)i;
        dperm.alloc(sizeof(int) * perm.size());
        XCUDA(cudaMemcpy(dperm.p, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice));
        dlptr.alloc(sizeof(int) * lptr.size());
        XCUDA(cudaMemcpy(dlptr.p, lptr.data(), sizeof(int) * lptr.size(), cudaMemcpyHostToDevice));
        return nl;
    };
    nlf = sched(lf, hlf, permf, lptrf);
    nlb = sched(lb, hlb, permb, lptrb);
    sync.alloc(kSyncBytes);
    XCUDA(cudaMemset(sync.p, 0, kSyncBytes));
}

// Level-ordered matrix copy of one sweep direction.  Rows are stored in
// schedule order ((block,) level, row); every level group is padded with
// empty rows (row id -1) to a multiple of 4 rows and every row's in-block
// entries (CSR order) are padded with column -1 to a multiple of 4, so all row
// and entry ranges handed to one CTA start on 16-byte boundaries and span
// multiples of 16 bytes (the TMA bulk-copy rule).  One descriptor {r0, r1, e0,
// e1} per (level, CTA) tells each CTA what to stage.
void GsPlan::build_offblock(const HostCsr &A, Prec p) {
    if (brows == 0) return;
    HostCsr off;
    off.n = A.n;
    off.ncols = A.ncols;
    off.rp.assign((size_t)A.n + 1, 0);
    for (i64 i = 0; i < A.n; ++i) {
        const i64 blk = i / brows;
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j)
            if (A.ci[j] / brows != blk) {
                off.ci.push_back(A.ci[j]);
                off.v.push_back(A.v[j]);
            }
        off.rp[i + 1] = (int)off.ci.size();
    }
    aprec = p;
    aoff.upload(off, p == Prec::F64, p == Prec::F32);
}

// Slot-mapped x window of hybrid blocks whose x tile does not fit in shared
// memory.  Within one block the sweep reads, at each level, the x rows of that
// level's entries: rows of earlier levels (written by this CTA) and rows of
// later ones (old values).  Every row of the block is given a shared-memory
// slot for its live range: from kSlotAhead levels before its first use (when
// its old value is loaded from global memory) to its last use; slots are
// reused by interval colouring.  The sweep then reads every x value from
// shared memory and loads only first-use rows, ahead of time, off the
// level's critical path.  No window is kept when a block needs more than
// kMaxSlots slots at once.
constexpr int kSlotAhead = xk::kGsSlotAhead;
constexpr int kMaxSlots = 4096;

void GsPlan::build_slots(int d, const std::vector<int> &order, const std::vector<int> &groups,
                         const std::vector<int> &blev, const std::vector<int> &lrp, const std::vector<int> &lci) {
    Lcsr &L = lc[d];
    L.nslots = 0;
    const i64 nr = (i64)order.size();
    const int ngroups = (int)groups.size() - 1;
    std::vector<int> slot(n, -1), first(n, INT32_MAX), last(n, -1);
    // {row, slot} pairs; ldd per level group and ldpre per block are {first, end}
    std::vector<int> ld, ldd(2 * (size_t)std::max(ngroups, 1), 0), ldpre(2 * (size_t)nblocks, 0);
    auto put_list = [&](std::vector<int> &rows, int *range) {
        std::sort(rows.begin(), rows.end());
        range[0] = (int)(ld.size() / 2);
        for (int c : rows) { ld.push_back(c); ld.push_back(slot[c]); }
        if (rows.size() & 1) { ld.push_back(-1); ld.push_back(-1); }  // even length: 16-byte ranges
        range[1] = (int)(ld.size() / 2);
    };
    int smax = 0;
    for (int b = 0; b < nblocks; ++b) {
        const int g0 = blev[b], g1 = blev[b + 1];
        std::vector<int> rows;
        for (int g = g0; g < g1; ++g)
            for (int r = groups[g]; r < groups[g + 1]; ++r) {
                const int i = order[r];
                if (i < 0) continue;
                const int lv = g - g0;
                auto use = [&](int c) {
                    if (first[c] == INT32_MAX) rows.push_back(c);
                    first[c] = std::min(first[c], lv);
                    last[c] = std::max(last[c], lv);
                };
                use(i);
                for (int q = lrp[r]; q < lrp[r + 1]; ++q)
                    if (lci[q] >= 0) use(lci[q]);
            }
        // live interval [first - ahead (or -1: loaded before the sweep), last]
        std::vector<std::pair<int, int>> iv;  // (start, row)
        iv.reserve(rows.size());
        for (int c : rows) iv.push_back({std::max(first[c] - kSlotAhead, -1), c});
        std::sort(iv.begin(), iv.end());
        std::priority_queue<std::pair<int, int>, std::vector<std::pair<int, int>>, std::greater<>> active;
        std::priority_queue<int, std::vector<int>, std::greater<>> freed;
        int used = 0;
        for (auto &e : iv) {
            while (!active.empty() && active.top().first < e.first) {
                freed.push(active.top().second);
                active.pop();
            }
            int sl;
            if (!freed.empty()) { sl = freed.top(); freed.pop(); }
            else sl = used++;
            slot[e.second] = sl;
            active.push({last[e.second], sl});
        }
        smax = std::max(smax, used);
        if (smax > kMaxSlots) return;
        // loads: before the first level the rows first used in levels
        // [0, ahead); with level group g those first used `ahead` levels later
        const int nl = g1 - g0;
        std::vector<std::vector<int>> per(nl);
        for (int c : rows) per[first[c]].push_back(c);
        std::vector<int> pre;
        for (int lv = 0; lv < std::min(nl, kSlotAhead); ++lv) pre.insert(pre.end(), per[lv].begin(), per[lv].end());
        put_list(pre, &ldpre[2 * (size_t)b]);
        for (int g = g0; g < g1; ++g) {
            std::vector<int> none;
            const int lv = g - g0 + kSlotAhead;
            put_list(lv < nl ? per[lv] : none, &ldd[2 * (size_t)g]);
        }
        for (int c : rows) { first[c] = INT32_MAX; last[c] = -1; }
    }
    std::vector<int> lcs(lci.size(), -1), lslot(std::max<i64>(nr, 4), -1);
    for (size_t q = 0; q < lci.size(); ++q)
        if (lci[q] >= 0) lcs[q] = slot[lci[q]];
    for (i64 r = 0; r < nr; ++r)
        if (order[r] >= 0) lslot[r] = slot[order[r]];
    if (ld.empty()) ld.assign(4, -1);
    // Replay the sweep's data flow on the host over exactly the arrays the
    // kernel receives: a slot is taken by a row when its load is issued (its
    // list's level) and every read at a level (the row's own slot, the slots
    // of its entries) must find that row in it.  Any mismatch drops the
    // window (the gather form then runs), so the kernel never reads a slot
    // that holds another row's value.
    {
        std::vector<int> occ(std::max(smax, 1), -1);
        bool good = true;
        auto take = [&](int a, int z) {
            if ((a & 1) || ((z - a) & 1) || a < 0 || z > (int)(ld.size() / 2)) { good = false; return; }
            for (int k = a; k < z; ++k) {
                const int row = ld[2 * (size_t)k], sl = ld[2 * (size_t)k + 1];
                if (row < 0) continue;
                if (row >= n || sl < 0 || sl >= smax) { good = false; return; }
                occ[sl] = row;
            }
        };
        for (int b = 0; good && b < nblocks; ++b) {
            std::fill(occ.begin(), occ.end(), -1);
            take(ldpre[2 * (size_t)b], ldpre[2 * (size_t)b + 1]);
            for (int g = blev[b]; good && g < blev[b + 1]; ++g) {
                take(ldd[2 * (size_t)g], ldd[2 * (size_t)g + 1]);
                for (int r = groups[g]; good && r < groups[g + 1]; ++r) {
                    if (order[r] < 0) continue;
                    const int sl = lslot[r];
                    good = sl >= 0 && sl < smax && occ[sl] == order[r];
                    for (int q = lrp[r]; good && q < lrp[r + 1]; ++q)
                        if (lci[q] >= 0) good = lcs[q] >= 0 && lcs[q] < smax && occ[lcs[q]] == lci[q];
                }
            }
        }
        if (!good) return;
    }
    upload_ints(L.lcs, lcs);
    upload_ints(L.lslot, lslot);
    upload_ints(L.ldd, ldd);
    upload_ints(L.ldpre, ldpre);
    upload_ints(L.ld, ld);
    L.nslots = std::max(smax, 1);
    L.nlmax = 0;
    for (int g = 0; g < ngroups; ++g) L.nlmax = std::max(L.nlmax, ldd[2 * (size_t)g + 1] - ldd[2 * (size_t)g]);
}

// Point-to-point waits of the cooperative (GRID) sweep.  Instead of a grid
// barrier after every level, CTA b publishes the number of levels it has
// finished, and before level l it waits only for the CTAs that own rows its
// level-l rows depend on: every row c of the symmetrised pattern of row j
// (j's own entries and the rows that read j) with a lower level.  Those are
// the values j reads after their update (c < j) and the rows that must have
// read j's old value before j changes it (rows c whose entries include j).
// Per (level, CTA) the list holds each other owner once with the most
// levels it must have finished.
void GsPlan::build_grid_deps(int d, const HostCsr &A, const std::vector<int> &lev, const std::vector<int> &order,
                             const std::vector<int> &desc, int G) {
    Lcsr &L = lc[d];
    const int ngroups = (int)(desc.size() / 4 / G);
    std::vector<int> own(n, -1);
    for (int l = 0; l < ngroups; ++l)
        for (int b = 0; b < G; ++b) {
            const int *dd = &desc[((size_t)l * G + b) * 4];
            for (int r = dd[0]; r < dd[1]; ++r)
                if (order[r] >= 0) own[order[r]] = b;
        }
    // transpose pattern: the rows whose entries include j
    std::vector<int> trp(n + 1, 0), tci(A.nnz());
    for (i64 q = 0; q < A.nnz(); ++q) trp[A.ci[q] + 1]++;
    for (i64 i = 0; i < n; ++i) trp[i + 1] += trp[i];
    {
        std::vector<int> at(trp.begin(), trp.end() - 1);
        for (i64 i = 0; i < n; ++i)
            for (int q = A.rp[i]; q < A.rp[i + 1]; ++q) tci[at[A.ci[q]]++] = (int)i;
    }
    std::vector<int> dptr((size_t)ngroups * G + 1, 0), deps;
    std::vector<int> need(G, 0), touched;
    for (int l = 0; l < ngroups; ++l)
        for (int b = 0; b < G; ++b) {
            const int *dd = &desc[((size_t)l * G + b) * 4];
            touched.clear();
            auto dep = [&](int c, int lj) {
                if (c < 0 || c >= n || lev[c] >= lj) return;
                const int o = own[c];
                if (o == b || o < 0) return;
                if (need[o] == 0) touched.push_back(o);
                need[o] = std::max(need[o], lev[c] + 1);
            };
            for (int r = dd[0]; r < dd[1]; ++r) {
                const int j = order[r];
                if (j < 0) continue;
                for (int q = A.rp[j]; q < A.rp[j + 1]; ++q) dep(A.ci[q], lev[j]);
                for (int q = trp[j]; q < trp[j + 1]; ++q) dep(tci[q], lev[j]);
            }
            std::sort(touched.begin(), touched.end());
            for (int o : touched) {
                deps.push_back(o);
                deps.push_back(need[o]);
                need[o] = 0;
            }
            dptr[(size_t)l * G + b + 1] = (int)(deps.size() / 2);
        }
    if (deps.empty()) deps.assign(2, 0);
    upload_ints(L.dptr, dptr);
    upload_ints(L.deps, deps);
    L.has_deps = true;
    if (prog.bytes < (size_t)G * 32) {
        prog.alloc((size_t)G * 32);
        XCUDA(cudaMemset(prog.p, 0, prog.bytes));
    }
}

void GsPlan::build_lcsr(const HostCsr &A, Prec p) {
    if (mode == GsMode::LEVELS) return;
    lprec = p;
    int G = 0;
    if (mode == GsMode::GRID) {
        int dev = 0;
        XCUDA(cudaGetDevice(&dev));
        XCUDA(cudaDeviceGetAttribute(&G, cudaDevAttrMultiProcessorCount, dev));
        if (G <= 0) G = 148;
    }
    std::vector<double> dinv(n, 0.0);
    for (i64 i = 0; i < n; ++i)
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j)
            if (A.ci[j] == i) dinv[i] = p == Prec::F64 ? 1.0 / A.v[j] : (double)(float)(1.0 / (double)(float)A.v[j]);
    auto inblk = [&](i64 i, i64 c) { return brows <= 0 || (c / brows) == (i / brows); };
    nnz_in = 0;
    for (i64 i = 0; i < n; ++i)
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) nnz_in += inblk(i, A.ci[j]);
    for (int d = 0; d < 2; ++d) {
        const std::vector<int> &lev = d == 0 ? lf : lb;
        std::vector<int> order;        // row id per level-ordered row (-1 = padding)
        std::vector<int> groups(1, 0); // level-group boundaries in `order`
        std::vector<int> blev(1, 0);
        order.reserve(n + n / 2);
        auto emit = [&](i64 r0, i64 r1) {
            int nl = 0;
            for (i64 i = r0; i < r1; ++i) nl = std::max(nl, lev[i] + 1);
            std::vector<int> cnt(nl + 1, 0);
            for (i64 i = r0; i < r1; ++i) cnt[lev[i] + 1]++;
            for (int l = 0; l < nl; ++l) cnt[l + 1] += cnt[l];
            std::vector<int> pos(cnt.begin(), cnt.end() - 1), seg(r1 - r0);
            for (i64 i = r0; i < r1; ++i) seg[pos[lev[i]]++] = (int)i;
            for (int l = 0; l < nl; ++l) {
                for (int q = cnt[l]; q < cnt[l + 1]; ++q) order.push_back(seg[q]);
                while (order.size() % 4) order.push_back(-1);
                groups.push_back((int)order.size());
            }
            return nl;
        };
        if (mode == GsMode::BLOCKS) {
            for (int b = 0; b < nblocks; ++b) {
                i64 r0 = (i64)b * brows, r1 = std::min<i64>(n, r0 + brows);
                blev.push_back(blev.back() + emit(r0, r1));
            }
        } else {
            emit(0, n);
        }
        const i64 nr = (i64)order.size();
        std::vector<int> lrp(nr + 5, 0);
        for (i64 r = 0; r < nr; ++r) {
            int i = order[r], k = 0;
            if (i >= 0)
                for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) k += inblk(i, A.ci[j]);
            lrp[r + 1] = lrp[r] + ((k + 3) & ~3);
        }
        for (int q = 1; q <= 4; ++q) lrp[nr + q] = lrp[nr];
        XCHECK(lrp[nr] >= 0 && (i64)lrp[nr] < (1ll << 31) - 8, "level-ordered matrix too large");
        std::vector<int> lci(std::max(lrp[nr], 4), -1);
        std::vector<double> lv(std::max(lrp[nr], 4), 0.0), li(std::max<i64>(nr, 4), 0.0);
        for (i64 r = 0; r < nr; ++r) {
            int i = order[r], q = lrp[r];
            if (i < 0) continue;
            li[r] = dinv[i];
            for (int j = A.rp[i]; j < A.rp[i + 1]; ++j)
                if (inblk(i, A.ci[j])) {
                    lci[q] = A.ci[j];
                    lv[q] = A.v[j];
                    ++q;
                }
        }
        // descriptors
        std::vector<int> desc;
        const int ngroups = (int)groups.size() - 1;
        if (mode == GsMode::GRID) {
            desc.resize((size_t)ngroups * G * 4);
            // contiguous row ranges of about equal cost (entries + 4 per row),
            // any row granularity: a level of a few long rows spreads over as
            // many CTAs as it has rows
            for (int l = 0; l < ngroups; ++l) {
                const int a = groups[l], z = groups[l + 1];
                auto cost = [&](int r) { return (i64)(lrp[r] - lrp[a]) + 4 * (i64)(r - a); };
                const i64 tot = cost(z);
                int r = a;
                for (int b = 0; b < G; ++b) {
                    const int r0 = r;
                    if (b == G - 1) {
                        r = z;
                    } else {
                        const i64 goal = tot * (b + 1) / G;
                        while (r < z && cost(r + 1) <= goal) ++r;
                    }
                    int *dd = &desc[((size_t)l * G + b) * 4];
                    dd[0] = r0; dd[1] = r; dd[2] = lrp[r0]; dd[3] = lrp[r];
                }
            }
        } else {
            desc.resize((size_t)std::max(ngroups, 1) * 4);
            for (int l = 0; l < ngroups; ++l) {
                int *dd = &desc[(size_t)l * 4];
                dd[0] = groups[l]; dd[1] = groups[l + 1]; dd[2] = lrp[groups[l]]; dd[3] = lrp[groups[l + 1]];
            }
        }
        if (order.empty()) order.push_back(-1);
        Lcsr &L = lc[d];
        L.nlev = ngroups;
        L.ncta = mode == GsMode::GRID ? G : nblocks;
        L.emax = 0;
        L.rmax = 0;
        for (size_t q = 0; q + 3 < desc.size(); q += 4) {
            L.emax = std::max(L.emax, desc[q + 3] - desc[q + 2]);
            L.rmax = std::max(L.rmax, ((desc[q + 1] + 3) & ~3) - (desc[q] & ~3));
        }
        L.lmax = 0;
        if (mode == GsMode::BLOCKS)
            for (size_t b = 0; b + 1 < blev.size(); ++b) L.lmax = std::max(L.lmax, blev[b + 1] - blev[b]);
        upload_ints(L.lrp, lrp);
        upload_ints(L.lci, lci);
        upload_ints(L.lrow, order);
        upload_ints(L.desc, desc);
        upload_ints(L.blev, blev);
        if (mode == GsMode::BLOCKS) build_slots(d, order, groups, blev, lrp, lci);
        if (mode == GsMode::GRID) build_grid_deps(d, A, lev, order, desc, G);
        if (p == Prec::F64) {
            L.lva.alloc(sizeof(double) * lv.size());
            XCUDA(cudaMemcpy(L.lva.p, lv.data(), sizeof(double) * lv.size(), cudaMemcpyHostToDevice));
            L.linvd.alloc(sizeof(double) * li.size());
            XCUDA(cudaMemcpy(L.linvd.p, li.data(), sizeof(double) * li.size(), cudaMemcpyHostToDevice));
        } else {
            std::vector<float> f(lv.begin(), lv.end()), g(li.begin(), li.end());
            L.lva.alloc(sizeof(float) * f.size());
            XCUDA(cudaMemcpy(L.lva.p, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice));
            L.linvd.alloc(sizeof(float) * g.size());
            XCUDA(cudaMemcpy(L.linvd.p, g.data(), sizeof(float) * g.size(), cudaMemcpyHostToDevice));
        }
    }
    has_lcsr = true;
}

// The slot window can be switched off (XAMG_GS_NO_SLOT_WINDOW set) to run
// the per-level gather form of the same sweeps, whose results are identical.
// Likewise the point-to-point waits of the cooperative sweep
// (XAMG_GS_GRID_BARRIER set: a grid barrier after every level instead).
static bool grid_deps_on() {
    static const bool on = std::getenv("XAMG_GS_GRID_BARRIER") == nullptr;
    return on;
}
static bool slot_window_on() {
    static const bool on = std::getenv("XAMG_GS_NO_SLOT_WINDOW") == nullptr;
    return on;
}
// Hybrid sweeps: one 256-thread CTA per block, or one warp per block
// (XAMG_GS_SWEEP=warp; XAMG_GS_SWEEP=cta selects the CTA kernel explicitly).
// Results are identical.
constexpr bool kWarpSweepDefault = false;
static bool warp_sweep_on() {
    static const bool on = [] {
        const char *e = std::getenv("XAMG_GS_SWEEP");
        if (e && std::strcmp(e, "warp") == 0) return true;
        if (e && std::strcmp(e, "cta") == 0) return false;
        return kWarpSweepDefault;
    }();
    return on;
}

int gs_warp_sweep() { return warp_sweep_on() ? 1 : 0; }

void GsPlan::sweep(Prec p, int nv, const int *rp, const int *ci, const void *val,
                   const void *invd, const void *t, void *x, const void *relax, bool forward,
                   cudaStream_t s) {
    int nl = forward ? nlf : nlb;
    const std::vector<int> &hl = forward ? hlf : hlb;
    const int *perm = (forward ? permf : permb).as<int>();
    if (nl == 0) return;
    if (has_lcsr && p == lprec && (mode == GsMode::GRID || mode == GsMode::BLOCKS)) {
        const Lcsr &L = lc[forward ? 0 : 1];
        unsigned *bar = sync.as<unsigned>();
        int *err = (int *)(sync.as<char>() + kSyncErrOffset);
        int md = mode == GsMode::BLOCKS ? 1 : 0;
        // the block's x tile in shared memory when it fits; a tile that allows
        // only one CTA per SM only when the blocks fit in one wave anyway
        // (otherwise the gather form, two CTAs per SM, finishes sooner)
        const i64 tile = (i64)brows * nv * (i64)prec_size(p);
        int xs = md == 1 && (tile <= xk::gs_lcsr_xs_bytes_two_per_sm() ||
                             (tile <= xk::gs_lcsr_max_xs_bytes() && nblocks <= sm_count()));
        // one sweep: in-block entries (column + value), per row its id, offset
        // and inverse diagonal, and t read, x read, x written
        const double sv = (double)prec_size(p);
        xk::GsSlotWin win{L.lslot.as<int>(), L.ldd.as<int2>(), L.ldpre.as<int2>(), L.ld.as<int2>(), L.nslots};
        xk::GsDeps gd{nullptr, nullptr, nullptr};
        if (md == 0 && L.has_deps && grid_deps_on()) gd = {L.dptr.as<int>(), L.deps.as<int2>(), prog.as<unsigned>()};
        const bool slots = md == 1 && !xs && L.nslots > 0 && slot_window_on() &&
                           (size_t)L.nslots * nv * prec_size(p) <= (size_t)xk::gs_slot_window_bytes() &&
                           nv * prec_size(p) >= 16;
        const double gbytes = (double)nnz_in * (4 + sv) + (double)n * (8 + sv) + 3.0 * n * nv * sv;
        if (md == 1 && warp_sweep_on()) {
            const int wslots = L.nslots > 0 && slot_window_on() ? L.nslots : 0;
            const xk::GswShape z = xk::gsw_shape(prec_size(p), nv, L.ncta, sm_count(), brows, wslots, L.emax,
                                                 L.rmax, L.lmax, L.nlmax);
            if (z.xm >= 0) {
                const KClass kw = z.xm == 1 ? KClass::GSW_TILE : z.xm == 2 ? KClass::GSW_WINDOW : KClass::GSW_GATHER;
                KTimeScope kt(kw, n, gbytes, s);
                XCUDA(xk::gs_sweep_warp(p, nv, z, L.ncta, L.desc.as<int>(), L.blev.as<int>(), L.lrp.as<int>(),
                                        z.xm == 2 ? L.lcs.as<int>() : L.lci.as<int>(), L.lva.p, L.lrow.as<int>(),
                                        L.linvd.p, t, x, relax, brows, n, z.xm == 2 ? &win : nullptr, L.lmax, s));
                return;
            }
        }
        const KClass kc = md == 0 ? KClass::GS_GRID : xs ? KClass::GS_TILE : slots ? KClass::GS_WINDOW : KClass::GS_GATHER;
        KTimeScope kt(kc, n, gbytes, s);
        XCUDA(xk::gs_sweep_lcsr(p, nv, md, xs, L.nlev, L.ncta, L.desc.as<int>(), L.blev.as<int>(),
                                L.lrp.as<int>(), slots ? L.lcs.as<int>() : L.lci.as<int>(), L.lva.p,
                                L.lrow.as<int>(), L.linvd.p, t, x, relax, brows, n, bar, err, L.emax,
                                slots ? &win : nullptr, gd.dptr ? &gd : nullptr, s));
        return;
    }
    if (mode == GsMode::BLOCKS) {
        if (forward)
            xk::gs_blocks(p, nv, nblocks, bblevf.as<int>(), blptrf.as<int>(), bpermf.as<int>(),
                          bblevb.as<int>(), blptrb.as<int>(), bpermb.as<int>(), rp, ci, val, invd, t,
                          x, relax, brows, s);
        return;
    }
    if (mode == GsMode::GRID && nl > 2) {
        unsigned *bar = sync.as<unsigned>();
        int *err = (int *)(sync.as<char>() + kSyncErrOffset);
        // {count, generation} start from zero (the level-ordered sweep leaves
        // its own arrival counter in the same words)
        XCUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
        XCUDA(xk::gs_sweep_persistent(p, nv, nl, (forward ? lptrf : lptrb).as<int>(), perm,
                                      rp, ci, val, invd, t, x, relax, brows, bar, err, s));
        return;
    }
    for (int l = 0; l < nl; ++l)
        xk::gs_level(p, nv, hl[l + 1] - hl[l], perm + hl[l], rp, ci, val, invd, t, x, relax,
                     brows, s);
}

int GsPlan::error_flag() const {
    if (!sync.p) return 0;
    int h = 0;
    XCUDA(cudaMemcpy(&h, sync.as<char>() + kSyncErrOffset, sizeof(int), cudaMemcpyDeviceToHost));
    return h;
}

// ------------------------------------------------------------------ Conv
double Conv::tol(int k) const {
    if (!ptol.empty()) return ptol[k];
    const double b2 = rhs_base && (int)base.size() == nv ? base[k] : res0[k];
    return std::max(abs_tol, rel_tol * std::sqrt(b2));
}
void Conv::update(const double *r) {
    for (int k = 0; k < nv; ++k)
        if (!status[k]) res[k] = r[k];
}
bool Conv::check() {
    if (!check_on) return false;
    bool all = true;
    for (int k = 0; k < nv; ++k) {
        if (status[k]) continue;
        double a = std::sqrt(res[k]);
        if (a > tol(k)) all = false;
        else status[k] = 1;
    }
    if (print_on && !quiet()) {
        printf("%s %4d", prefix.c_str(), iters);
        for (int k = 0; k < nv; ++k) printf(" %.3e", res0[k] > 0 ? std::sqrt(res[k] / res0[k]) : 0.0);
        printf("\n");
    }
    return all;
}

// Rows per hybrid Gauss-Seidel block of an n-row level: hybrid_blocks = P
// splits every level into P equal blocks (the reference's semantics on P
// cores, whose partition divides each level's rows among the processes);
// otherwise hybrid_block_rows, 0 meaning the single-process sweep.
static i64 hsgs_block_rows(const ParamList &pl, i64 n) {
    if (pl.has("hybrid_blocks") && pl.get_int("hybrid_blocks") > 0) {
        const i64 P = pl.get_int("hybrid_blocks");
        return P >= 2 ? (n + P - 1) / P : 0;
    }
    return pl.has("hybrid_block_rows") ? (i64)pl.get_int("hybrid_block_rows") : 0;
}

static void parse_conv(const ParamList &l, Conv &c) {
    std::set<std::string> cd;
    std::string s = l.has("convergence_details") ? l.get_string("convergence_details") : "nocheck,noprint";
    std::string cur;
    for (char ch : s + ",") {
        if (ch == ',') { if (!cur.empty()) cd.insert(cur); cur.clear(); }
        else cur += ch;
    }
    c.print_on = cd.count("noprint") == 0;
    c.check_on = cd.count("nocheck") == 0;
    if (l.has("abs_tolerance")) c.abs_tol = l.get_float("abs_tolerance");
    if (l.has("rel_tolerance")) c.rel_tol = l.get_float("rel_tolerance");
    if (l.has("rel_tolerance_base")) {
        const std::string b = l.get_string("rel_tolerance_base");
        if (b != "rhs" && b != "initial") throw Error("rel_tolerance_base must be \"initial\" or \"rhs\"", 4);
        c.rhs_base = b == "rhs";
    }
}

void parse_conv_settings(const ParamList &l, Conv &c) { parse_conv(l, c); }

// ------------------------------------------------------------------ helpers
static void dot1(const DVec &a, const DVec &b, DBuf &part, double *out, cudaStream_t s) {
    const void *A[1] = {a.p()}, *B[1] = {b.p()};
    xk::dots(a.prec, a.nv, a.n, 1, A, B, part.as<double>(), out, s);
}
// dot_order = "tree" (default: the fixed reduction tree the kernels share)
// or "sequential" (the reference's single-core order, blas.inl:561-576;
// one dependent chain per column, for results bit-identical to a
// one-process run of the reference)
static bool dot_order_sequential(const ParamList &l) {
    if (!l.has("dot_order")) return false;
    const std::string o = l.get_string("dot_order");
    if (o != "tree" && o != "sequential") throw Error("dot_order must be \"tree\" or \"sequential\"", 4);
    return o == "sequential";
}
static void ensure_part(DBuf &part, i64 n, int nd, int nv) {
    size_t need = sizeof(double) * std::max<i64>(xk::dot_part_size(n, nd, nv), 1);
    if (part.bytes < need) part.alloc(need);
}

// ||b||^2 per column as the base of the relative tolerance (rel_tolerance_base = rhs)
static void set_rhs_base(Conv &c, const DVec &b, DBuf &part) {
    if (!c.rhs_base) return;
    cudaStream_t s = ctx().stream;
    ensure_part(part, b.n, 1, b.nv);
    DBuf out(sizeof(double) * b.nv);
    dot1(b, b, part, out.as<double>(), s);
    c.base.assign(b.nv, 0.0);
    XCUDA(cudaMemcpyAsync(c.base.data(), out.p, sizeof(double) * b.nv, cudaMemcpyDeviceToHost, s));
    XCUDA(cudaStreamSynchronize(s));
}

struct Pinned {
    double *h = nullptr;
    size_t cnt = 0;
    void alloc(size_t c) {
        if (h) cudaFreeHost(h);
        XCUDA(cudaMallocHost(&h, sizeof(double) * std::max<size_t>(c, 1)));
        cnt = c;
    }
    ~Pinned() { if (h) cudaFreeHost(h); }
};

// ------------------------------------------------------------------ solvers
struct Identity : Solver {
    void solve(DVec &x, const DVec &b) override {
        xk::blas(prec, nv, x.n, xk::Op::COPY, nullptr, b.p(), nullptr, nullptr, nullptr, x.p(), ctx().stream);
    }
};

// Direct coarse solve: x = A^{-1} b with a dense inverse built at setup.
struct Direct : Solver {
    int n = 0;
    DBuf AT;
    void setup(const HostCsr &A, Prec p, std::vector<double> &inv_out) {
        n = (int)A.n;
        std::vector<double> D((size_t)n * n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) D[(size_t)i * n + A.ci[j]] = A.v[j];
        inv_out.resize((size_t)n * n);
        dense_inverse(n, D.data(), inv_out.data());
        prec = p;
        if (p == Prec::F64) {
            std::vector<double> T((size_t)n * n);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) T[(size_t)j * n + i] = inv_out[(size_t)i * n + j];
            AT.alloc(sizeof(double) * std::max<size_t>(T.size(), 1));
            XCUDA(cudaMemcpy(AT.p, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice));
        } else {
            std::vector<float> T((size_t)n * n);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) T[(size_t)j * n + i] = (float)inv_out[(size_t)i * n + j];
            AT.alloc(sizeof(float) * std::max<size_t>(T.size(), 1));
            XCUDA(cudaMemcpy(AT.p, T.data(), sizeof(float) * T.size(), cudaMemcpyHostToDevice));
        }
    }
    void solve(DVec &x, const DVec &b) override {
        xk::dense_gemv(prec, nv, n, AT.p, b.p(), x.p(), ctx().stream);
    }
};

// Smoothers operate on one level operator (device CSR + inverse diagonal).
struct LevelOp {
    const DCsr *A = nullptr;
    const void *invd = nullptr;
    GsPlan *gs = nullptr;
};

struct HSGS : Solver {
    LevelOp op;
    DVec t, r;
    DBuf relax, ones, part;
    Pinned hres;
    void init(const LevelOp &o, i64 n) {
        op = o;
        parse_conv(prm, conv);
        conv.init(nv);
        std::vector<double> rl(nv, prm.get_float("relax_factor"));
        relax.alloc(sizeof(double) * nv);
        if (prec == Prec::F64) XCUDA(cudaMemcpy(relax.p, rl.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
        else {
            std::vector<float> rf(rl.begin(), rl.end());
            XCUDA(cudaMemcpy(relax.p, rf.data(), sizeof(float) * nv, cudaMemcpyHostToDevice));
        }
        if (op.gs->brows > 0 && op.gs->brows < n) t.alloc(n, nv, prec);
        if (conv.check_on) {
            r.alloc(n, nv, prec);
            ensure_part(part, n, 1, nv);
            hres.alloc(nv);
        }
    }
    // one blas2::SGS call (blas2.h:184-281).  With x zero the off-block
    // product is +0 in every entry, so t = 1*b + (-1)*(+0) is b itself, bit
    // for bit, and is not formed
    void sgs(DVec &x, const DVec &b, bool xzero = false) {
        cudaStream_t s = ctx().stream;
        const void *tp = b.p();
        if (t.n && !xzero) {
            // t = 1*b + (-1)*(A_off x), the chain over the off-block entries in CSR order
            if (op.gs->aoff.n == x.n && op.gs->aprec == prec)
                op.gs->aoff.spmv(prec, nv, x.p(), t.p(), 2, b.p(), s);
            else
                xk::offblock_resid(prec, nv, x.n, op.A->rpp(), op.A->cip(), op.A->val(prec), b.p(), x.p(), t.p(),
                                   op.gs->brows, s);
            tp = t.p();
        }
        const DCsr &A = *op.A;
        op.gs->sweep(prec, nv, A.rpp(), A.cip(), A.val(prec), op.invd, tp, x.p(), relax.p, true, s);
        op.gs->sweep(prec, nv, A.rpp(), A.cip(), A.val(prec), op.invd, tp, x.p(), relax.p, false, s);
    }
    bool residual_check(DVec &x, const DVec &b, bool initial) {
        cudaStream_t s = ctx().stream;
        op.A->spmv(prec, nv, x.p(), r.p(), 2, b.p(), s);
        DBuf out(sizeof(double) * nv);
        dot1(r, r, part, out.as<double>(), s);
        XCUDA(cudaMemcpyAsync(hres.h, out.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, s));
        XCUDA(cudaStreamSynchronize(s));
        if (initial) conv.res0.assign(hres.h, hres.h + nv);
        conv.update(hres.h);
        conv.record();
        return conv.check();
    }
    void run(DVec &x, const DVec &b, bool xzero) {
        int iters = (int)prm.get_int("max_iters");
        conv.init(nv);
        set_rhs_base(conv, b, part);
        if (conv.check_on && residual_check(x, b, true)) return;
        for (int it = 1; it <= iters; ++it) {
            conv.iters = it;
            sgs(x, b, xzero && it == 1);
            if (conv.check_on && residual_check(x, b, false)) return;
        }
    }
    void solve(DVec &x, const DVec &b) override { run(x, b, false); }
    void solve_from_zero(DVec &x, const DVec &b) override { run(x, b, true); }
};

// Spectrum bounds of D^-1/2 A D^-1/2 for the Chebyshev smoother.  The
// reference takes them from hypre's BoomerAMG setup (hypre_base.inl:370-375,
// CG-based estimates); hypre is not available here, so the same kind of
// estimate is made: `iters` CG steps on the scaled operator from a fixed
// pseudo-random start give the Lanczos tridiagonal matrix
// (T_kk = 1/alpha_k + beta_{k-1}/alpha_{k-1}, T_k,k+1 = sqrt(beta_k)/alpha_k)
// whose extreme eigenvalues (cyclic Jacobi rotations) are the bounds.
void eig_estimate(const HostCsr &A, int iters, double &mn, double &mx) {
    const i64 n = A.n;
    std::vector<double> d(n, 0.0), r(n), p(n), w(n);
    for (i64 i = 0; i < n; ++i)
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j)
            if (A.ci[j] == i) d[i] = 1.0 / std::sqrt(std::fabs(A.v[j]));
    unsigned long long st = 0x9E3779B97F4A7C15ull;
    for (i64 i = 0; i < n; ++i) {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        r[i] = (double)(st >> 11) / 9007199254740992.0 - 0.5;
    }
    auto dot = [&](const std::vector<double> &a, const std::vector<double> &b) {
        double s = 0.0;
        for (i64 i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    };
    p = r;
    double rr = dot(r, r);
    std::vector<double> al, be;
    const int k = (int)std::min<i64>(iters, n);
    for (int it = 0; it < k && rr > 0; ++it) {
        for (i64 i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) s += A.v[j] * d[A.ci[j]] * p[A.ci[j]];
            w[i] = d[i] * s;
        }
        const double pw = dot(p, w);
        if (!(pw > 0)) break;
        const double a = rr / pw;
        for (i64 i = 0; i < n; ++i) r[i] -= a * w[i];
        const double rr2 = dot(r, r);
        al.push_back(a);
        be.push_back(rr2 / rr);
        rr = rr2;
        for (i64 i = 0; i < n; ++i) p[i] = r[i] + be.back() * p[i];
    }
    const int m = (int)al.size();
    if (m == 0) { mn = mx = 1.0; return; }
    std::vector<double> T((size_t)m * m, 0.0);
    for (int q = 0; q < m; ++q) {
        T[(size_t)q * m + q] = 1.0 / al[q] + (q > 0 ? be[q - 1] / al[q - 1] : 0.0);
        if (q + 1 < m) T[(size_t)q * m + q + 1] = T[(size_t)(q + 1) * m + q] = std::sqrt(be[q]) / al[q];
    }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < m; ++i)
            for (int j = i + 1; j < m; ++j) off += T[(size_t)i * m + j] * T[(size_t)i * m + j];
        if (off < 1e-30) break;
        for (int i = 0; i < m; ++i)
            for (int j = i + 1; j < m; ++j) {
                const double aij = T[(size_t)i * m + j];
                if (std::fabs(aij) < 1e-300) continue;
                const double th = (T[(size_t)j * m + j] - T[(size_t)i * m + i]) / (2.0 * aij);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int q = 0; q < m; ++q) {
                    const double tqi = T[(size_t)q * m + i], tqj = T[(size_t)q * m + j];
                    T[(size_t)q * m + i] = c * tqi - s * tqj;
                    T[(size_t)q * m + j] = s * tqi + c * tqj;
                }
                for (int q = 0; q < m; ++q) {
                    const double tiq = T[(size_t)i * m + q], tjq = T[(size_t)j * m + q];
                    T[(size_t)i * m + q] = c * tiq - s * tjq;
                    T[(size_t)j * m + q] = s * tiq + c * tjq;
                }
            }
    }
    mn = mx = T[0];
    for (int q = 1; q < m; ++q) {
        mn = std::min(mn, T[(size_t)q * m + q]);
        mx = std::max(mx, T[(size_t)q * m + q]);
    }
}

// Chebyshev polynomial coefficients (chebyshev.inl:51-128), orders 1..4.
std::vector<double> cheby_coeffs(double min_eig, double max_eig, int order, double fraction) {
    const double upper = max_eig * 1.1;
    const double lower = (upper - min_eig) * fraction + min_eig;
    const double th = (upper + lower) / 2., de = (upper - lower) / 2.;
    std::vector<double> c;
    double den;
    switch (order) {
    case 1: c = {1. / th}; break;
    case 2:
        den = de * de - 2 * th * th;
        c = {-4 * th / den, 2 / den};
        break;
    case 3:
        den = 3 * (de * de) * th - 4 * (th * th * th);
        c = {(3 * de * de - 12 * th * th) / den, 12 * th / den, -4 / den};
        break;
    case 4:
        den = std::pow(de, 4) - 8 * de * de * th * th + 8 * std::pow(th, 4);
        c = {(32 * std::pow(th, 3) - 16 * de * de * th) / den, (8 * de * de - 48 * th * th) / den,
             32 * th / den, -8 / den};
        break;
    default: throw Error("polynomial_order must be 1..4", 2);
    }
    return c;
}

// Chebyshev smoother (chebyshev.inl:142-183): r = D^-1/2 (b - A x);
// t1 = c_{p-1} r; for i = p-2..0: t1 = c_i r + D^-1/2 A D^-1/2 t1;
// x += D^-1/2 t1.  Coefficients in the level's precision (the reference
// stores them as F).
struct Chebyshev : Solver {
    const DCsr *A = nullptr;
    const void *isd = nullptr;
    DVec r, t1, t2;
    DBuf coef, ones;  // coef: order x nv per-column copies
    int order = 2;
    void init(const DCsr *a, const void *isd_, i64 n, double min_eig, double max_eig) {
        A = a;
        isd = isd_;
        parse_conv(prm, conv);
        conv.init(nv);
        order = (int)prm.get_int("polynomial_order");
        std::vector<double> c = cheby_coeffs(min_eig, max_eig, order, prm.get_float("spectrum_fraction"));
        std::vector<double> cv((size_t)order * nv);
        for (int i = 0; i < order; ++i)
            for (int k = 0; k < nv; ++k) cv[(size_t)i * nv + k] = prec == Prec::F32 ? (double)(float)c[i] : c[i];
        coef.alloc(sizeof(double) * cv.size());
        XCUDA(cudaMemcpy(coef.p, cv.data(), sizeof(double) * cv.size(), cudaMemcpyHostToDevice));
        std::vector<double> o(nv, 1.0);
        ones.alloc(sizeof(double) * nv);
        XCUDA(cudaMemcpy(ones.p, o.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
        r.alloc(n, nv, prec);
        t1.alloc(n, nv, prec);
        t2.alloc(n, nv, prec);
    }
    void solve(DVec &x, const DVec &b) override {
        cudaStream_t s = ctx().stream;
        const i64 n = x.n;
        const double *C = coef.as<double>();
        const double *one = ones.as<double>();
        A->spmv(prec, nv, x.p(), r.p(), 2, b.p(), s);
        xk::blas(prec, nv, n, xk::Op::ROW_SCAL, nullptr, isd, nullptr, nullptr, nullptr, r.p(), s);
        xk::blas(prec, nv, n, xk::Op::AX_Y, C + (size_t)(order - 1) * nv, r.p(), nullptr, nullptr, nullptr, t1.p(), s);
        for (int i = order - 2; i >= 0; --i) {
            xk::blas(prec, nv, n, xk::Op::ROW_SCAL, nullptr, isd, nullptr, nullptr, nullptr, t1.p(), s);
            A->spmv(prec, nv, t1.p(), t2.p(), 0, nullptr, s);
            xk::blas(prec, nv, n, xk::Op::ROW_SCAL, nullptr, isd, nullptr, nullptr, nullptr, t2.p(), s);
            xk::blas(prec, nv, n, xk::Op::AXPBY_Z, C + (size_t)i * nv, r.p(), one, t2.p(), nullptr, t1.p(), s);
        }
        xk::blas(prec, nv, n, xk::Op::ROW_SCAL, nullptr, isd, nullptr, nullptr, nullptr, t1.p(), s);
        xk::blas(prec, nv, n, xk::Op::AXPBY_Z, one, t1.p(), one, x.p(), nullptr, x.p(), s);
    }
};

struct Jacobi : Solver {
    LevelOp op;
    DVec tmp, r;
    DBuf relax, part;
    Pinned hres;
    void init(const LevelOp &o, i64 n) {
        op = o;
        parse_conv(prm, conv);
        conv.init(nv);
        std::vector<double> rl(nv, prm.get_float("relax_factor"));
        relax.alloc(sizeof(double) * nv);
        if (prec == Prec::F64) XCUDA(cudaMemcpy(relax.p, rl.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
        else {
            std::vector<float> rf(rl.begin(), rl.end());
            XCUDA(cudaMemcpy(relax.p, rf.data(), sizeof(float) * nv, cudaMemcpyHostToDevice));
        }
        tmp.alloc(n, nv, prec);
        if (conv.check_on) {
            r.alloc(n, nv, prec);
            ensure_part(part, n, 1, nv);
            hres.alloc(nv);
        }
    }
    void solve(DVec &x, const DVec &b) override {
        cudaStream_t s = ctx().stream;
        int iters = (int)prm.get_int("max_iters");
        conv.init(nv);
        set_rhs_base(conv, b, part);
        if (!conv.check_on) {
            // nocheck path (jacobi.inl:91-100): x_{k+1} = x_k + relax*D^-1 (b - A x_k),
            // ping-ponging between x and tmp
            DVec *cur = &x, *nxt = &tmp;
            for (int it = 1; it <= iters; ++it) {
                xk::jacobi(prec, nv, x.n, op.A->rpp(), op.A->cip(), op.A->val(prec), op.invd, b.p(), cur->p(), nxt->p(), relax.p, s);
                std::swap(cur, nxt);
            }
            if (cur != &x)
                xk::blas(prec, nv, x.n, xk::Op::COPY, nullptr, cur->p(), nullptr, nullptr, nullptr, x.p(), s);
            return;
        }
        // check path (jacobi.inl:76-89): r = b - A x; r *= invdiag; x = relax*r + 1*x
        throw Error("Jacobi with convergence checks is not supported on the device path", 4);
    }
};

// ------------------------------------------------------------------ MultiGrid
struct MultiGrid : Solver {
    std::vector<MGLevel> lv;
    std::unique_ptr<Direct> coarse;
    std::vector<double> coarse_inv;
    Matrix *Afine = nullptr;
    int cycle = 0;
    DVec r;
    DBuf part, ones;
    Pinned hres;
    bool reduced = false;

    Prec lvprec(int l) const { return l == 0 ? prec : (reduced ? Prec::F32 : prec); }

    void setup(const GlobalParams &gp, Matrix &A) {
        Afine = &A;
        parse_conv(prm, conv);
        conv.init(nv);
        conv.prefix = role == "preconditioner" ? "PREC" : "SOLV";
        cycle = (int)prm.get_int("mg_cycle");
        reduced = prec == Prec::F64 && prm.get_bool("mg_reduced_precision");
        std::vector<AmgLevel> al;
        amg_setup(A.h, amg_params_for(gp, role), al);
        int L = (int)al.size();
        lv.resize(L);
        for (int l = 0; l < L; ++l) {
            MGLevel &m = lv[l];
            m.prec = lvprec(l);
            if (l > 0) m.hA = std::move(al[l].A);
            m.hP = std::move(al[l].P);
            const HostCsr &hA = l == 0 ? A.h : m.hA;
            bool w64 = m.prec == Prec::F64, w32 = m.prec == Prec::F32;
            if (l == 0) {
                if (w32) A.ensure32();
            } else {
                m.A.upload(hA, w64, w32);
            }
            if (l + 1 < L) {
                Prec cp = lvprec(l + 1);
                HostCsr R;
                csr_transpose(m.hP, R);
                m.P.upload(m.hP, cp == Prec::F64, cp == Prec::F32);
                m.R.upload(R, cp == Prec::F64, cp == Prec::F32);
                m.tmp.alloc(hA.n, nv, m.prec);
                if (cp != m.prec) m.tmp2.alloc(hA.n, nv, cp);
                m.xH.alloc(m.hP.ncols, nv, cp);
                m.bH.alloc(m.hP.ncols, nv, cp);
                make_invd(hA, w64, w32, m.invd64, m.invd32);
            }
        }
        // smoothers
        for (int l = 0; l + 1 < L; ++l) {
            MGLevel &m = lv[l];
            const HostCsr &hA = l == 0 ? A.h : m.hA;
            const DCsr &dA = l == 0 ? A.d : m.A;
            ParamList pre = gp.get_level("pre_smoother", l), post = gp.get_level("post_smoother", l);
            m.pre = make_smoother(pre, "pre_smoother", m, hA, dA, true);
            m.post = make_smoother(post, "post_smoother", m, hA, dA, false);
        }
        // coarse-grid solver
        ParamList cl = gp.get("coarse_grid_solver");
        XCHECK(cl.get_string("method") == "Direct", "only the Direct coarse-grid solver is supported");
        coarse.reset(new Direct());
        coarse->nv = nv;
        coarse->method = "Direct";
        coarse->setup(L == 1 ? A.h : lv[L - 1].hA, lvprec(L - 1), coarse_inv);
        if (conv.check_on) {
            r.alloc(A.h.n, nv, prec);
            ensure_part(part, A.h.n, 1, nv);
            hres.alloc(nv);
        }
    }

    std::unique_ptr<Solver> make_smoother(const ParamList &pl, const std::string &rl, MGLevel &m,
                                          const HostCsr &hA, const DCsr &dA, bool pre) {
        std::string meth = pl.get_string("method");
        LevelOp op;
        op.A = &dA;
        op.invd = m.prec == Prec::F64 ? m.invd64.p : m.invd32.p;
        if (meth == "HSGS") {
            i64 br = hsgs_block_rows(pl, hA.n);
            GsMode md = gs_mode_from(pl.has("gs_schedule") ? pl.get_string("gs_schedule") : "auto", br, hA.n);
            GsPlan &g = pre ? m.gs_pre : m.gs_post;
            i64 brn = br > 0 && br < hA.n ? br : 0;
            if (!pre && m.gs_pre.n == hA.n && m.gs_pre.brows == brn && m.gs_pre.mode == md) {
                op.gs = &m.gs_pre;
            } else {
                g.build(hA, br, md);
                g.build_lcsr(hA, m.prec);
                g.build_offblock(hA, m.prec);
                op.gs = &g;
            }
            auto h = std::unique_ptr<HSGS>(new HSGS());
            h->role = rl; h->method = meth; h->prm = pl; h->nv = nv; h->prec = m.prec;
            h->init(op, hA.n);
            return h;
        }
        if (meth == "Chebyshev") {
            // sqrt(1/a_ii) as csr_matrix.h:357-389 computes it (last diagonal
            // entry wins; the FP32 copy from the FP32 value)
            DBuf &isd = m.prec == Prec::F64 ? m.isd64 : m.isd32;
            if (!isd.p) {
                std::vector<double> d(hA.n, 0.0);
                std::vector<float> f(hA.n, 0.f);
                for (i64 i = 0; i < hA.n; ++i)
                    for (int j = hA.rp[i]; j < hA.rp[i + 1]; ++j)
                        if (hA.ci[j] == i) {
                            d[i] = std::sqrt(1.0 / hA.v[j]);
                            f[i] = (float)std::sqrt(1.0 / (double)(float)hA.v[j]);
                        }
                const size_t es = m.prec == Prec::F64 ? sizeof(double) : sizeof(float);
                isd.alloc(es * std::max<i64>(hA.n, 1));
                XCUDA(cudaMemcpy(isd.p, m.prec == Prec::F64 ? (const void *)d.data() : (const void *)f.data(),
                                 es * hA.n, cudaMemcpyHostToDevice));
                eig_estimate(hA, 10, m.min_eig, m.max_eig);
            }
            auto c = std::unique_ptr<Chebyshev>(new Chebyshev());
            c->role = rl; c->method = meth; c->prm = pl; c->nv = nv; c->prec = m.prec;
            c->init(&dA, isd.p, hA.n, m.min_eig, m.max_eig);
            return c;
        }
        if (meth == "Jacobi") {
            auto j = std::unique_ptr<Jacobi>(new Jacobi());
            j->role = rl; j->method = meth; j->prm = pl; j->nv = nv; j->prec = m.prec;
            j->init(op, hA.n);
            return j;
        }
        throw Error("unsupported smoother method: " + meth, 4);
    }

    const DCsr &levA(int l) const { return l == 0 ? Afine->d : lv[l].A; }

    // MG_cycle mg.inl:186-280
    void mg_cycle(int l, DVec &x, const DVec &b, int cyc, bool xzero = false) {
        cudaStream_t s = ctx().stream;
        MGLevel &m = lv[l];
        Prec p = m.prec, cp = lvprec(l + 1);
        const DCsr &A = levA(l);
        if (cyc != 1) {
            if (xzero) m.pre->solve_from_zero(x, b);
            else m.pre->solve(x, b);
        }
        // temp = b - A x
        A.spmv(p, nv, x.p(), m.tmp.p(), 2, b.p(), s);
        // restriction (convert first when the next level is in FP32)
        if (cp != p) {
            xk::convert(p, cp, m.tmp.count(), m.tmp.p(), m.tmp2.p(), s);
            m.R.spmv(cp, nv, m.tmp2.p(), m.bH.p(), 0, nullptr, s);
        } else {
            m.R.spmv(cp, nv, m.tmp.p(), m.bH.p(), 0, nullptr, s);
        }
        xk::fill(cp, m.xH.count(), 0.0, m.xH.p(), s);
        if (l + 1 == (int)lv.size() - 1) {
            coarse->solve(m.xH, m.bH);
        } else {
            mg_cycle(l + 1, m.xH, m.bH, cyc, true);  // x_H was just zeroed
            if (cyc == 2) mg_cycle(l + 1, m.xH, m.bH, 2);
            else if (cyc == 1) mg_cycle(l + 1, m.xH, m.bH, 0);
        }
        // prolongation
        if (cp != p) {
            m.P.spmv(cp, nv, m.xH.p(), m.tmp2.p(), 0, nullptr, s);
            xk::convert(cp, p, m.tmp2.count(), m.tmp2.p(), m.tmp.p(), s);
            if (!ones.p) {
                std::vector<double> o(nv, 1.0);
                ones.alloc(sizeof(double) * nv);
                XCUDA(cudaMemcpy(ones.p, o.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
            }
            xk::blas(p, nv, x.n, xk::Op::AXPBY_Z, ones.as<double>(), m.tmp.p(), ones.as<double>(), x.p(), nullptr, x.p(), s);
        } else {
            m.P.spmv(p, nv, m.xH.p(), x.p(), 1, nullptr, s);
        }
        m.post->solve(x, b);
    }

    bool residual_check(DVec &x, const DVec &b, bool initial) {
        cudaStream_t s = ctx().stream;
        const DCsr &A = levA(0);
        A.spmv(prec, nv, x.p(), r.p(), 2, b.p(), s);
        DBuf out(sizeof(double) * nv);
        dot1(r, r, part, out.as<double>(), s);
        XCUDA(cudaMemcpyAsync(hres.h, out.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, s));
        XCUDA(cudaStreamSynchronize(s));
        if (initial) conv.res0.assign(hres.h, hres.h + nv);
        conv.update(hres.h);
        conv.record();
        return conv.check();
    }

    void run(DVec &x, const DVec &b, bool xzero) {
        int iters = (int)prm.get_int("max_iters");
        conv.init(nv);
        set_rhs_base(conv, b, part);
        if (conv.check_on && residual_check(x, b, true)) return;
        for (int it = 1; it <= iters; ++it) {
            conv.iters = it;
            if (lv.size() == 1) coarse->solve(x, b);
            else mg_cycle(0, x, b, cycle, xzero && it == 1);
            if (conv.check_on && residual_check(x, b, false)) return;
        }
    }
    void solve(DVec &x, const DVec &b) override { run(x, b, false); }
    void solve_from_zero(DVec &x, const DVec &b) override { run(x, b, true); }

    std::string info() const override {
        std::string s = "MultiGrid levels:";
        for (size_t l = 0; l < lv.size(); ++l) {
            const HostCsr &A = l == 0 ? Afine->h : lv[l].hA;
            s += " " + std::to_string(A.n) + "/" + std::to_string(A.nnz());
        }
        return s;
    }
};

MultiGrid *find_multigrid(Solver *s);

// ------------------------------------------------------------------ Krylov
// (P)BiCGStab and RBiCGStab.  Scalars live on the device; the host reads the
// NV residuals once per iteration for the convergence check.
struct Krylov : Solver {
    Matrix *A = nullptr;
    std::unique_ptr<Solver> M;
    bool precond = false;
    bool reordered = false;  // RBiCGStab
    bool cg = false;         // PCG
    bool seq_dot = false;    // dot_order = sequential
    DVec r0, r, p, v, s, t, p_, s_;
    DBuf part, sc;
    Pinned hres;
    enum { RHO, S1, S2, S3, S4, ALPHA, OMEGA, BETA, C1, RES, AC, OC, ICONV, ONES, NALPHA, NOMEGA,
           THETA, PHI, PSI, ETA, DELTA, STAT, TOLS, NSC };
    Pinned hres_async;
    cudaEvent_t res_ready = nullptr;
    ~Krylov() override {
        if (res_ready) cudaEventDestroy(res_ready);
    }
    xk::BicgScalars scalars() const {
        xk::BicgScalars b;
        b.rho = S(RHO); b.alpha = S(ALPHA); b.omega = S(OMEGA); b.beta = S(BETA); b.c1 = S(C1);
        b.ac = S(AC); b.oc = S(OC); b.res = S(RES); b.iconv = S(ICONV); b.status = S(STAT);
        b.tol = S(TOLS);
        b.check = conv.check_on ? 1 : 0;
        return b;
    }
    double *S(int i) const { return sc.as<double>() + (size_t)i * nv; }

    void setup(i64 n) {
        parse_conv(prm, conv);
        seq_dot = dot_order_sequential(prm);
        conv.init(nv);
        conv.prefix = role == "meta_solver" ? "META" : "SOLV";
        for (DVec *q : {&r0, &r, &p, &v, &s, &t}) q->alloc(n, nv, prec);
        if (precond || reordered || cg) { p_.alloc(n, nv, prec); s_.alloc(n, nv, prec); }
        ensure_part(part, n, reordered ? 4 : 3, nv);
        sc.alloc(sizeof(double) * NSC * nv);
        std::vector<double> z(NSC * nv, 0.0);
        for (int k = 0; k < nv; ++k) { z[ONES * nv + k] = 1.0; z[ICONV * nv + k] = 1.0; }
        XCUDA(cudaMemcpy(sc.p, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice));
        hres.alloc(nv);
        hres_async.alloc(nv);
        XCUDA(cudaEventCreateWithFlags(&res_ready, cudaEventDisableTiming));
    }

    const DCsr &dA() const { return A->d; }

    // per-column tolerances and convergence status after the initial check,
    // and the matching masks, for the device-side convergence bookkeeping of
    // the fused iteration
    void set_conv_state(cudaStream_t st) {
        std::vector<double> h(3 * nv);
        for (int k = 0; k < nv; ++k) {
            h[k] = conv.status[k] ? 0.0 : 1.0;        // ICONV
            h[nv + k] = conv.status[k] ? 1.0 : 0.0;   // STAT
            h[2 * nv + k] = conv.tol(k);              // TOLS
        }
        XCUDA(cudaMemcpyAsync(S(ICONV), h.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        XCUDA(cudaMemcpyAsync(S(STAT), h.data() + nv, sizeof(double) * 2 * nv, cudaMemcpyHostToDevice, st));
        XCUDA(cudaStreamSynchronize(st));
    }

    void read_res(int which, cudaStream_t st) {
        XCUDA(cudaMemcpyAsync(hres.h, S(which), sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
        XCUDA(cudaStreamSynchronize(st));
    }

    void set_iconv(cudaStream_t st) {
        std::vector<double> ic(nv);
        for (int k = 0; k < nv; ++k) ic[k] = conv.status[k] ? 0.0 : 1.0;
        XCUDA(cudaMemcpyAsync(S(ICONV), ic.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        XCUDA(cudaStreamSynchronize(st));
    }

    void spmv(const DVec &x, DVec &y, cudaStream_t st) {
        const DCsr &a = dA();
        a.spmv(prec, nv, x.p(), y.p(), 0, nullptr, st);
    }

    void solve(DVec &x, const DVec &b) override {
        seq_dot = dot_order_sequential(prm);  // renewed parameters apply at the next solve
        xk::DotOrderScope order(seq_dot);
        if (reordered) { solve_reordered(x, b); return; }
        if (cg) { solve_cg(x, b); return; }
        cudaStream_t st = ctx().stream;
        int max_iters = (int)prm.get_int("max_iters");
        i64 n = x.n;
        const DCsr &a = dA();
        conv.init(nv);
        set_rhs_base(conv, b, part);
        {
            std::vector<double> one(nv, 1.0);
            XCUDA(cudaMemcpyAsync(S(ICONV), one.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        }
        // r0 = b - A x; rho = (r0, r0)
        a.spmv(prec, nv, x.p(), r0.p(), 2, b.p(), st);
        dot1(r0, r0, part, S(RHO), st);
        read_res(RHO, st);
        conv.res0.assign(hres.h, hres.h + nv);
        conv.update(hres.h);
        conv.record();
        if (conv.check()) return;
        set_conv_state(st);
        xk::blas(prec, nv, n, xk::Op::COPY, nullptr, r0.p(), nullptr, nullptr, nullptr, r.p(), st);
        xk::blas(prec, nv, n, xk::Op::COPY, nullptr, r0.p(), nullptr, nullptr, nullptr, p.p(), st);
        if (precond) xk::fill(prec, p_.count(), 0.0, p_.p(), st);
        // One iteration in the reference's step order (pbicgstab.inl:108-204)
        // as the merged groups of MergedPBiCGStab: the scalar recurrences run
        // in the reduction stage of their inner products, s = r - alpha v
        // zeroes s_ for the preconditioner in the same pass, x, r and the
        // partial sums of (r, r0) are one pass, and p's update zeroes p_.
        // The convergence masks are kept on the device; the host reads the
        // NV residuals once per iteration while the last two kernels run.
        const xk::BicgScalars sc = scalars();
        for (int it = 1;; ++it) {
            conv.iters = it;
            DVec *pp = &p, *ss = &s;
            if (precond) {
                M->solve_from_zero(p_, p);
                pp = &p_;
            }
            spmv(*pp, v, st);
            {
                const void *Aa[1] = {v.p()}, *Bb[1] = {r0.p()};
                xk::dot_partials(prec, nv, n, 1, Aa, Bb, part.as<double>(), st);
                xk::dot_reduce_epi(0, n, 1, nv, part.as<double>(), S(S1), sc, st);
            }
            xk::bicg_s(prec, nv, n, sc, r.p(), v.p(), s.p(), precond ? s_.p() : nullptr, st);
            if (precond) {
                M->solve_from_zero(s_, s);
                ss = &s_;
            }
            spmv(*ss, t, st);
            {
                const void *Aa[3] = {t.p(), t.p(), s.p()}, *Bb[3] = {s.p(), t.p(), s.p()};
                xk::dot_partials(prec, nv, n, 3, Aa, Bb, part.as<double>(), st);
                xk::dot_reduce_epi(1, n, 3, nv, part.as<double>(), S(S2), sc, st);
            }
            xk::bicg_xr(prec, nv, n, sc, pp->p(), ss->p(), x.p(), s.p(), t.p(), r.p(), r0.p(), part.as<double>(),
                        st);
            if (seq_dot) {
                // (r, r0) in the sequential order replaces the fused pass's tree partials
                const void *Aa[1] = {r.p()}, *Bb[1] = {r0.p()};
                xk::dot_partials(prec, nv, n, 1, Aa, Bb, part.as<double>(), st);
            }
            XCUDA(cudaMemcpyAsync(hres_async.h, S(RES), sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
            XCUDA(cudaEventRecord(res_ready, st));
            // the next direction is formed before the host has looked at the
            // residuals; after the last iteration it is simply not used
            xk::dot_reduce_epi(2, n, 1, nv, part.as<double>(), S(S1), sc, st);
            xk::bicg_p(prec, nv, n, sc, r.p(), v.p(), p.p(), precond ? p_.p() : nullptr, st);
            XCUDA(cudaEventSynchronize(res_ready));
            conv.update(hres_async.h);
            conv.record();
            if (conv.check()) break;
            if (it >= max_iters) break;
        }
        XCUDA(cudaStreamSynchronize(st));
    }

    // PCG (pcg.inl:48-160).  The step's two inner products (r,z), (p,Ap) are
    // one fused launch, and so are (r,z) and (r,r) after the preconditioner;
    // beta and the new direction are formed after the convergence check
    // (they do not touch x).
    void solve_cg(DVec &x, const DVec &b) {
        cudaStream_t st = ctx().stream;
        int max_iters = (int)prm.get_int("max_iters");
        i64 n = x.n;
        const DCsr &a = dA();
        DVec &z = p_, &Ap = v;
        auto axpby = [&](const double *ca, const DVec &xx, const double *cb, const DVec &yy, DVec &zz) {
            xk::blas(prec, nv, n, xk::Op::AXPBY_Z, ca, xx.p(), cb, yy.p(), nullptr, zz.p(), st);
        };
        conv.init(nv);
        set_rhs_base(conv, b, part);
        {
            std::vector<double> one(nv, 1.0);
            XCUDA(cudaMemcpyAsync(S(ICONV), one.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        }
        // r = b - A x; res = (r, r)
        a.spmv(prec, nv, x.p(), r.p(), 2, b.p(), st);
        dot1(r, r, part, S(RES), st);
        read_res(RES, st);
        conv.res0.assign(hres.h, hres.h + nv);
        conv.update(hres.h);
        conv.record();
        if (conv.check()) return;
        set_iconv(st);
        xk::fill(prec, z.count(), 0.0, z.p(), st);
        M->solve_from_zero(z, r);
        xk::blas(prec, nv, n, xk::Op::COPY, nullptr, z.p(), nullptr, nullptr, nullptr, p.p(), st);
        for (int it = 1;; ++it) {
            conv.iters = it;
            a.spmv(prec, nv, p.p(), Ap.p(), 0, nullptr, st);
            {
                const void *Aa[2] = {r.p(), p.p()}, *Bb[2] = {z.p(), Ap.p()};
                xk::dots(prec, nv, n, 2, Aa, Bb, part.as<double>(), S(S1), st);
            }
            xk::pcg_alpha(nv, S(S1), S(S2), S(ICONV), S(ALPHA), S(AC), S(NALPHA), st);
            axpby(S(AC), p, S(ONES), x, x);
            axpby(S(NALPHA), Ap, S(ONES), r, r);
            xk::fill(prec, z.count(), 0.0, z.p(), st);
            M->solve_from_zero(z, r);
            {
                const void *Aa[2] = {r.p(), r.p()}, *Bb[2] = {z.p(), r.p()};
                xk::dots(prec, nv, n, 2, Aa, Bb, part.as<double>(), S(S3), st);  // S3 = (r,z), S4 = (r,r)
            }
            read_res(S4, st);
            conv.update(hres.h);
            conv.record();
            if (conv.check()) break;
            if (it >= max_iters) break;
            set_iconv(st);
            xk::bicg_alpha(nv, S(S3), S(S1), S(BETA), st);  // beta = (r,z)_new / (r,z)_old
            axpby(S(ONES), z, S(BETA), p, p);
        }
        XCUDA(cudaStreamSynchronize(st));
    }

    // RBiCGStab (rbicgstab.inl:48-225): the preconditioner is applied to r0 once
    // and to v and t in every iteration; x is updated before the convergence
    // check, so a converged iteration needs no further vector work.  The four
    // inner products of step 13 are one fused launch.
    void solve_reordered(DVec &x, const DVec &b) {
        cudaStream_t st = ctx().stream;
        int max_iters = (int)prm.get_int("max_iters");
        i64 n = x.n;
        const DCsr &a = dA();
        DVec &z = p, &v_ = p_, &t_ = s_;
        auto axpby = [&](const double *ca, const DVec &xx, const double *cb, const DVec &yy, DVec &zz) {
            xk::blas(prec, nv, n, xk::Op::AXPBY_Z, ca, xx.p(), cb, yy.p(), nullptr, zz.p(), st);
        };
        auto apply_m = [&](DVec &out, const DVec &in) {
            xk::fill(prec, out.count(), 0.0, out.p(), st);
            M->solve_from_zero(out, in);
        };
        conv.init(nv);
        set_rhs_base(conv, b, part);
        {
            std::vector<double> one(nv, 1.0);
            XCUDA(cudaMemcpyAsync(S(ICONV), one.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        }
        // 1-2: r0 = b - A x; rho = (r0, r0)
        a.spmv(prec, nv, x.p(), r0.p(), 2, b.p(), st);
        dot1(r0, r0, part, S(RHO), st);
        read_res(RHO, st);
        conv.res0.assign(hres.h, hres.h + nv);
        conv.update(hres.h);
        conv.record();
        if (conv.check()) return;
        set_iconv(st);
        xk::blas(prec, nv, n, xk::Op::COPY, nullptr, r0.p(), nullptr, nullptr, nullptr, r.p(), st);
        apply_m(z, r0);                                                      // 3
        xk::blas(prec, nv, n, xk::Op::COPY, nullptr, z.p(), nullptr, nullptr, nullptr, v_.p(), st);
        for (int it = 1;; ++it) {
            conv.iters = it;
            spmv(v_, v, st);                                                 // 6
            dot1(v, r0, part, S(DELTA), st);                                 // 7
            apply_m(s, v);                                                   // 8
            xk::rbicg_alpha(nv, S(RHO), S(DELTA), S(ALPHA), S(NALPHA), st);  // 9
            axpby(S(ONES), z, S(NALPHA), s, t_);                             // 10
            spmv(t_, t, st);                                                 // 11
            axpby(S(NALPHA), v, S(ONES), r, r);                              // 12
            {                                                                // 13
                const void *Aa[4] = {t.p(), t.p(), t.p(), r.p()}, *Bb[4] = {r.p(), t.p(), r0.p(), r.p()};
                xk::dots(prec, nv, n, 4, Aa, Bb, part.as<double>(), S(THETA), st);
            }
            apply_m(z, t);                                                   // 14
            // 15, 17: omega = theta/phi; res = 1*eta + (-1)*(omega*theta);
            // alpha_conv, omega_conv = iconv*alpha, iconv*omega
            xk::bicg_omega(nv, S(THETA), S(PHI), S(ETA), S(ALPHA), S(ICONV), S(OMEGA), S(RES), S(AC),
                           S(OC), st);
            xk::negate(nv, S(OMEGA), S(NOMEGA), st);
            axpby(S(NOMEGA), t, S(ONES), r, r);                              // 16
            xk::blas(prec, nv, n, xk::Op::AXPBYPCZ, S(AC), v_.p(), S(OC), t_.p(), S(ONES), x.p(), st);
            read_res(RES, st);
            conv.update(hres.h);
            conv.record();
            if (conv.check()) break;
            if (it >= max_iters) break;
            set_iconv(st);
            // 21-22, 25: rho = -(omega*psi); beta = rho/(delta*omega); delta = (-omega)*beta
            xk::rbicg_beta(nv, S(OMEGA), S(PSI), S(DELTA), S(RHO), S(BETA), S(NOMEGA), st);
            axpby(S(ONES), t_, S(NOMEGA), z, z);                             // 24
            xk::blas(prec, nv, n, xk::Op::AXPBYPCZ, S(ONES), z.p(), S(DELTA), s.p(), S(BETA), v_.p(), st);
        }
        XCUDA(cudaStreamSynchronize(st));
    }
    std::string info() const override { return method + (M ? "(" + M->info() + ")" : ""); }
};

// ------------------------------------------------------------------ IR
// IterativeRefinement (ir.inl:107-194).  Outer loop in FP64: r = b - A x,
// inner solve on r (FP32 when subsolver_reduced_precision), x += x_corr.
struct IterRefine : Solver {
    Matrix *A = nullptr;
    std::unique_ptr<Solver> inner;
    bool reduced = false;
    double inner_rel = 0.0;
    DVec r, xc, ix, ib;
    DBuf part, ones;
    Pinned hres;
    bool seq_dot = false;
    void setup(i64 n) {
        parse_conv(prm, conv);
        seq_dot = dot_order_sequential(prm);
        conv.init(nv);
        conv.prefix = "META";
        r.alloc(n, nv, Prec::F64);
        xc.alloc(n, nv, Prec::F64);
        if (reduced) { ix.alloc(n, nv, Prec::F32); ib.alloc(n, nv, Prec::F32); }
        ensure_part(part, n, 1, nv);
        std::vector<double> o(nv, 1.0);
        ones.alloc(sizeof(double) * nv);
        XCUDA(cudaMemcpy(ones.p, o.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
        hres.alloc(nv);
    }
    bool residual_check(DVec &x, const DVec &b, bool initial) {
        cudaStream_t s = ctx().stream;
        xk::DotOrderScope order(seq_dot);
        const DCsr &a = A->d;
        a.spmv(Prec::F64, nv, x.p(), r.p(), 2, b.p(), s);
        DBuf out(sizeof(double) * nv);
        dot1(r, r, part, out.as<double>(), s);
        XCUDA(cudaMemcpyAsync(hres.h, out.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, s));
        XCUDA(cudaStreamSynchronize(s));
        if (initial) conv.res0.assign(hres.h, hres.h + nv);
        conv.update(hres.h);
        conv.record();
        return conv.check();
    }
    void solve(DVec &x, const DVec &b) override {
        seq_dot = dot_order_sequential(prm);
        xk::DotOrderScope order(seq_dot);
        cudaStream_t s = ctx().stream;
        int max_iters = (int)prm.get_int("max_iters");
        conv.init(nv);
        set_rhs_base(conv, b, part);
        if (residual_check(x, b, true)) return;
        for (int it = 1; it <= max_iters; ++it) {
            conv.iters = it;
            // inner tolerance per column: the outer absolute tolerance, or a
            // fraction of the current residual (inner_rel_tolerance)
            std::vector<double> tol(nv);
            for (int k = 0; k < nv; ++k)
                tol[k] = std::max(conv.tol(k), inner_rel * std::sqrt(std::max(hres.h[k], 0.0)));
            inner->conv.ptol = tol;
            if (reduced) {
                xk::convert(Prec::F64, Prec::F32, r.count(), r.p(), ib.p(), s);
                xk::fill(Prec::F32, ix.count(), 0.0, ix.p(), s);
                inner->solve(ix, ib);
                xk::convert(Prec::F32, Prec::F64, ix.count(), ix.p(), xc.p(), s);
            } else {
                xk::fill(Prec::F64, xc.count(), 0.0, xc.p(), s);
                inner->solve(xc, r);
            }
            xk::blas(Prec::F64, nv, x.n, xk::Op::AXPBY_Z, ones.as<double>(), xc.p(), ones.as<double>(), x.p(), nullptr, x.p(), s);
            conv.sub_iters += inner->conv.iters;
            if (residual_check(x, b, false)) return;
        }
    }
    std::string info() const override { return "IterativeRefinement(" + inner->info() + ")"; }
};

// ------------------------------------------------------------------ factory
static std::unique_ptr<Solver> make_solver(const GlobalParams &gp, const std::string &role,
                                           Matrix &A, int nv, Prec prec) {
    const ParamList &pl = gp.get(role);
    std::string m = pl.get_string("method");
    i64 n = A.h.n;
    if (prec == Prec::F32) A.ensure32();
    if (m == "BiCGStab" || m == "MergedBiCGStab" || m == "PBiCGStab" || m == "MergedPBiCGStab" ||
        m == "RBiCGStab" || m == "MergedRBiCGStab" || m == "PCG") {
        auto k = std::unique_ptr<Krylov>(new Krylov());
        k->role = role; k->method = m; k->prm = pl; k->nv = nv; k->prec = prec; k->A = &A;
        k->reordered = (m == "RBiCGStab" || m == "MergedRBiCGStab");
        k->cg = m == "PCG";
        k->precond = (m == "PBiCGStab" || m == "MergedPBiCGStab" || k->reordered || k->cg);
        if (k->precond) {
            if (gp.has("preconditioner")) k->M = make_solver(gp, "preconditioner", A, nv, prec);
            else {
                auto id = std::unique_ptr<Identity>(new Identity());
                id->nv = nv; id->prec = prec; id->method = "Identity";
                k->M = std::move(id);
            }
        }
        k->setup(n);
        return k;
    }
    if (m == "MultiGrid") {
        auto g = std::unique_ptr<MultiGrid>(new MultiGrid());
        g->role = role; g->method = m; g->prm = pl; g->nv = nv; g->prec = prec;
        g->setup(gp, A);
        return g;
    }
    if (m == "Identity") {
        auto id = std::unique_ptr<Identity>(new Identity());
        id->role = role; id->method = m; id->prm = pl; id->nv = nv; id->prec = prec;
        return id;
    }
    if (m == "HSGS" || m == "Jacobi") {
        // standalone smoother solver on the fine operator
        struct Own : Solver {
            std::unique_ptr<Solver> s;
            DBuf invd64, invd32;
            GsPlan gs;
            void solve(DVec &x, const DVec &b) override {
                s->solve(x, b);
                conv = s->conv;
            }
        };
        auto o = std::unique_ptr<Own>(new Own());
        o->role = role; o->method = m; o->prm = pl; o->nv = nv; o->prec = prec;
        make_invd(A.h, prec == Prec::F64, prec == Prec::F32, o->invd64, o->invd32);
        LevelOp op;
        op.A = &A.d;
        op.invd = prec == Prec::F64 ? o->invd64.p : o->invd32.p;
        if (m == "HSGS") {
            i64 br = hsgs_block_rows(pl, A.h.n);
            o->gs.build(A.h, br, gs_mode_from(pl.has("gs_schedule") ? pl.get_string("gs_schedule") : "auto", br, A.h.n));
            o->gs.build_lcsr(A.h, prec);
            o->gs.build_offblock(A.h, prec);
            op.gs = &o->gs;
            auto h = std::unique_ptr<HSGS>(new HSGS());
            h->role = role; h->method = m; h->prm = pl; h->nv = nv; h->prec = prec;
            h->init(op, n);
            o->s = std::move(h);
        } else {
            auto j = std::unique_ptr<Jacobi>(new Jacobi());
            j->role = role; j->method = m; j->prm = pl; j->nv = nv; j->prec = prec;
            j->init(op, n);
            o->s = std::move(j);
        }
        return o;
    }
    throw Error("method not implemented on the device path: " + m, 4);
}

std::unique_ptr<Solver> make_role_solver(const GlobalParams &gp, const std::string &role, Matrix &A,
                                         int nv, Prec prec) {
    return make_solver(gp, role, A, nv, prec);
}

std::unique_ptr<Solver> build_solver_tree(const GlobalParams &gp, Matrix &A, int nv) {
    if (gp.has("meta_solver")) {
        const ParamList &ml = gp.get("meta_solver");
        XCHECK(ml.get_string("method") == "IterativeRefinement",
               "meta_solver must be IterativeRefinement");
        auto ir = std::unique_ptr<IterRefine>(new IterRefine());
        ir->role = "meta_solver"; ir->method = "IterativeRefinement"; ir->prm = ml; ir->nv = nv;
        ir->A = &A;
        ir->reduced = ml.has("subsolver_reduced_precision") && ml.get_bool("subsolver_reduced_precision");
        ir->inner_rel = ml.has("inner_rel_tolerance") ? ml.get_float("inner_rel_tolerance") : 0.0;
        ir->inner = make_solver(gp, "solver", A, nv, ir->reduced ? Prec::F32 : Prec::F64);
        ir->setup(A.h.n);
        return ir;
    }
    return make_solver(gp, "solver", A, nv, Prec::F64);
}

MultiGrid *find_multigrid(Solver *s) {
    if (!s) return nullptr;
    if (auto m = dynamic_cast<MultiGrid *>(s)) return m;
    if (auto k = dynamic_cast<Krylov *>(s)) return find_multigrid(k->M.get());
    if (auto ir = dynamic_cast<IterRefine *>(s)) return find_multigrid(ir->inner.get());
    return nullptr;
}
int mg_num_levels(MultiGrid *mg) { return (int)mg->lv.size(); }
const HostCsr &mg_level_A(MultiGrid *mg, int l) { return l == 0 ? mg->Afine->h : mg->lv[l].hA; }
const HostCsr &mg_level_P(MultiGrid *mg, int l) { return mg->lv[l].hP; }
const GsPlan &mg_level_gs(MultiGrid *mg, int l) { return mg->lv[l].gs_pre; }
const std::vector<double> &mg_coarse_inverse(MultiGrid *mg) { return mg->coarse_inv; }
void mg_set_spmv_variant(MultiGrid *mg, Prec p, int variant) {
    const int k = p == Prec::F64 ? 0 : 1;
    if (mg->Afine) mg->Afine->d.variant[k] = variant;
    for (MGLevel &m : mg->lv)
        for (const DCsr *d : {&m.A, &m.P, &m.R, &m.gs_pre.aoff, &m.gs_post.aoff}) d->variant[k] = variant;
}
void mg_level_eig(MultiGrid *mg, int l, double *mn, double *mx) {
    XCHECK(l >= 0 && l < (int)mg->lv.size(), "level out of range");
    *mn = mg->lv[l].min_eig;
    *mx = mg->lv[l].max_eig;
}

// Gauss-Jordan without pivoting (inverse.inl:31-106, same operation order);
// the independent row updates of each elimination step run in parallel.
void dense_inverse(int n, const double *A, double *Ainv) {
    int m = 2 * n;
    std::vector<double> e((size_t)n * m, 0.0);
    for (int i = 0; i < n; ++i) {
        e[(size_t)i * m + i + n] = 1.0;
        for (int j = 0; j < n; ++j) e[(size_t)i * m + j] = A[(size_t)i * n + j];
    }
    for (int i = 0; i < n; ++i) {
        double *ri = &e[(size_t)i * m];
        for (int k = m - 1; k > i; --k) ri[k] /= ri[i];
        ri[i] = 1.0;
#pragma omp parallel for schedule(static) if (n > 256)
        for (int j = i + 1; j < n; ++j) {
            double *rj = &e[(size_t)j * m];
            for (int k = m - 1; k > i; --k) rj[k] -= rj[i] * ri[k];
            rj[i] = 0.0;
        }
    }
    for (int ii = 0; ii < n; ++ii) {
        int row = n - 1 - ii;
        double *ri = &e[(size_t)row * m];
#pragma omp parallel for schedule(static) if (n > 256)
        for (int j = 0; j < row; ++j) {
            double *rj = &e[(size_t)j * m];
            for (int k = n; k < m; ++k) rj[k] -= rj[row] * ri[k];
            rj[row] = 0.0;
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) Ainv[(size_t)i * n + j] = e[(size_t)i * m + n + j];
}

}  // namespace xamg

namespace xamg {
// Sticky error flags of the bounded device waits in the Gauss-Seidel sweeps.
int mg_device_errors(MultiGrid *mg) {
    int e = 0;
    for (auto &l : mg->lv) {
        if (l.gs_pre.n) e |= l.gs_pre.error_flag();
        if (l.gs_post.n) e |= l.gs_post.error_flag();
    }
    return e;
}
}  // namespace xamg
