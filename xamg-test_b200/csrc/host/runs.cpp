// Shifted-row run plans (host side of xk::spmv_runs).
//
// Detection walks the rows once: row r joins the chunk of row r-1 when both
// have the same entry count and ci(r, e) = ci(r-1, e) + 1 for every entry,
// and the chunk has fewer than R rows.  Every row belongs to exactly one
// chunk (irregular rows are chunks of one row), so the run kernel alone
// evaluates the whole product.
#include "solve.h"
#include <omp.h>

namespace xamg {

void RunPlan::clear() {
    R = 0;
    nchunks = ntiles = nseg = 0;
    coverage = 0.0;
    hchunks.clear();
    hvoff.clear();
    chunks.release();
    toff.release();
    sg.release();
    v64.release();
    v32.release();
}

template <class T>
static void fill_values(const HostCsr &h, int R, const std::vector<int> &ch, const std::vector<i64> &vo,
                        std::vector<T> &vt) {
    const i64 ntiles = (i64)vo.size() - 1;
    vt.assign((size_t)std::max<i64>(vo[ntiles] * R, 2), T(0));
#pragma omp parallel for schedule(static)
    for (i64 t = 0; t < ntiles; ++t)
        for (int slot = 0; slot < 4; ++slot) {
            const int *c = &ch[(size_t)(4 * t + slot) * 4];
            for (int q = 0; q < c[1]; ++q) {
                const i64 base = h.rp[c[0] + q];
                for (int e = 0; e < c[2]; ++e) vt[(size_t)(vo[t] + 4 * e + slot) * R + q] = (T)h.v[base + e];
            }
        }
}

// Segments of a column list: runs of at most 3 consecutive columns, c0 | len << 30.
static int segments(const int *c, int m, int *out) {
    int ns = 0;
    for (int e = 0; e < m;) {
        int len = 1;
        while (len < 3 && e + len < m && c[e + len] == c[e + len - 1] + 1) ++len;
        if (out) out[ns] = c[e] | (len << 30);
        ++ns;
        e += len;
    }
    return ns;
}

// Chunks of up to R rows, {r0, cnt, m, segments} each; returns the entries
// that lie in chunks of exactly R rows.
static i64 detect_chunks(i64 n, const int *rp, const int *ci, int R, std::vector<int> &ch) {
    ch.clear();
    ch.reserve((size_t)n);
    i64 full = 0;
    for (i64 r = 0; r < n;) {
        const int m = rp[r + 1] - rp[r];
        int cnt = 1;
        while (cnt < R && r + cnt < n) {
            const i64 a = rp[r + cnt - 1], b = rp[r + cnt];
            if (rp[r + cnt + 1] - b != m) break;
            bool ok = true;
            for (int e = 0; e < m && ok; ++e) ok = ci[b + e] == ci[a + e] + 1;
            if (!ok) break;
            ++cnt;
        }
        const int ns = segments(ci + rp[r], m, nullptr);
        ch.insert(ch.end(), {(int)r, cnt, m, ns});
        if (cnt == R) full += (i64)cnt * m;
        r += cnt;
    }
    return full;
}

void run_plan_analyze(i64 n, const int *rp, const int *ci, int R, i64 *nchunks, double *coverage, i64 *nseg) {
    std::vector<int> ch;
    const i64 full = detect_chunks(n, rp, ci, R, ch);
    const i64 nnz = n > 0 ? rp[n] : 0;
    *nchunks = (i64)ch.size() / 4;
    *coverage = nnz ? (double)full / (double)nnz : 0.0;
    i64 s = 0;
    for (size_t c = 0; c < ch.size(); c += 4) s += ch[c + 3];
    *nseg = s;
}

bool RunPlan::build(const HostCsr &h, int R_, bool f64, bool f32, double min_cov) {
    clear();
    if (h.n <= 0 || h.n != h.ncols || h.n >= (i64(1) << 30) || R_ != 8) return false;
    std::vector<int> ch;
    const i64 full = detect_chunks(h.n, h.rp.data(), h.ci.data(), R_, ch);
    const i64 nnz = h.nnz();
    coverage = nnz ? (double)full / (double)nnz : 0.0;
    if (coverage < min_cov) {
        coverage = 0.0;
        return false;
    }
    R = R_;
    nchunks = (i64)ch.size() / 4;
    while (ch.size() % 16) ch.insert(ch.end(), {0, 0, 0, 0});  // whole tiles of four chunks
    ntiles = (i64)ch.size() / 16;
    std::vector<i64> vo((size_t)ntiles + 1, 0), so((size_t)ntiles + 1, 0);
    for (i64 t = 0; t < ntiles; ++t) {
        int mm = 0, ms = 0;
        for (int slot = 0; slot < 4; ++slot) {
            mm = std::max(mm, ch[(size_t)(4 * t + slot) * 4 + 2]);
            ms = std::max(ms, ch[(size_t)(4 * t + slot) * 4 + 3]);
        }
        vo[t + 1] = vo[t] + 4 * (i64)mm;
        so[t + 1] = so[t] + 4 * (i64)ms;
    }
    nseg = so[ntiles];
    std::vector<int> seg((size_t)std::max<i64>(nseg, 4), 0);
#pragma omp parallel for schedule(static)
    for (i64 t = 0; t < ntiles; ++t)
        for (int slot = 0; slot < 4; ++slot) {
            const int *c = &ch[(size_t)(4 * t + slot) * 4];
            if (c[2] == 0) continue;
            std::vector<int> tmp((size_t)c[3]);
            segments(&h.ci[h.rp[c[0]]], c[2], tmp.data());
            for (int k = 0; k < c[3]; ++k) seg[(size_t)(so[t] + 4 * k + slot)] = tmp[k];
        }
    std::vector<longlong2> to((size_t)ntiles + 1);
    for (i64 t = 0; t <= ntiles; ++t) to[t] = make_longlong2(vo[t], so[t]);
    hchunks = std::move(ch);
    hvoff = std::move(vo);
    cudaStream_t s = ctx().stream;
    chunks.alloc(sizeof(int) * hchunks.size());
    toff.alloc(sizeof(longlong2) * to.size());
    sg.alloc(sizeof(int) * seg.size());
    XCUDA(cudaMemcpyAsync(chunks.p, hchunks.data(), chunks.bytes, cudaMemcpyHostToDevice, s));
    XCUDA(cudaMemcpyAsync(toff.p, to.data(), toff.bytes, cudaMemcpyHostToDevice, s));
    XCUDA(cudaMemcpyAsync(sg.p, seg.data(), sg.bytes, cudaMemcpyHostToDevice, s));
    XCUDA(cudaStreamSynchronize(s));
    if (f64) add_values(h, Prec::F64);
    if (f32) add_values(h, Prec::F32);
    return true;
}

void RunPlan::add_values(const HostCsr &h, Prec p) {
    if (nchunks == 0 || has(p)) return;
    cudaStream_t s = ctx().stream;
    if (p == Prec::F64) {
        std::vector<double> vt;
        fill_values<double>(h, R, hchunks, hvoff, vt);
        v64.alloc(sizeof(double) * vt.size());
        XCUDA(cudaMemcpyAsync(v64.p, vt.data(), v64.bytes, cudaMemcpyHostToDevice, s));
        XCUDA(cudaStreamSynchronize(s));
    } else {
        std::vector<float> vt;
        fill_values<float>(h, R, hchunks, hvoff, vt);
        v32.alloc(sizeof(float) * vt.size());
        XCUDA(cudaMemcpyAsync(v32.p, vt.data(), v32.bytes, cudaMemcpyHostToDevice, s));
        XCUDA(cudaStreamSynchronize(s));
    }
}

void DCsr::spmv(Prec p, int nv, const void *x, void *y, int mode, const void *b, cudaStream_t s) const {
    const int own = variant[p == Prec::F64 ? 0 : 1];
    const int var = own >= 0 ? own : xk::get_spmv_variant();
    const double sv = (double)prec_size(p);
    // x read once, y written, y or b read for modes 1 and 2
    const double xy = (double)ncols * nv * sv + (double)n * nv * sv * (mode >= 1 ? 2 : 1);
    if ((var < 0 || var == 7) && runs.has(p) && xk::spmv_runs_supported(p, nv)) {
        // run format: values once, 4 B per segment, 20 B per chunk (descriptor
        // and its share of the tile offsets)
        KTimeScope kt(KClass::SPMV, n, (double)nnz * sv + 4.0 * runs.nseg + 20.0 * runs.nchunks + xy, s);
        xk::spmv_runs(p, nv, runs.nchunks, runs.ntiles, runs.chunks.as<int4>(), runs.toff.as<longlong2>(),
                      runs.sg.as<int>(), p == Prec::F64 ? runs.v64.p : runs.v32.p, x, y, mode, b, s);
        return;
    }
    KTimeScope kt(KClass::SPMV, n, (double)nnz * (sv + 4) + (double)(n + 1) * 4 + xy, s);
    xk::spmv(p, nv, n, rpp(), cip(), val(p), x, y, mode, b, s, var);
}

}  // namespace xamg
