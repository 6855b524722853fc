// Host-side algebraic multigrid setup.
//
// The reference builds its hierarchy with hypre BoomerAMG (hypre_base.h:121-217,
// hypre_base.inl:340-406) and copies A_l and P_l into its own CSR, forming
// R_l = P_l^T.  hypre 2.20.0 is not available here, so this file implements the
// same published algorithms on the host:
//   * classical strength of connection with threshold theta and the
//     max_row_sum rule (Ruge & Stueben 1987; hypre's CreateS semantics);
//   * C/F splitting by the Ruge-Stueben first pass; on one process hypre's
//     HMIS (coarsen type 10) reduces to this pass (De Sterck, Yang, Heys 2006),
//     and types 1/3/6 add the classical second pass;
//   * extended+i interpolation (De Sterck, Falgout, Nolting, Yang 2008) with
//     truncation by trunc_factor and P_max_elmts, row sums preserved;
//   * Galerkin coarse operator A_c = P^T A P.
// Row order of every coarse operator follows hypre's diag block convention:
// diagonal first, then ascending columns.  P rows are ascending.  The setup is
// deterministic (OpenMP only over independent rows with fixed per-row order).
#include "amg.h"
#include "params.h"
#include <algorithm>
#include <cmath>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace xamg {

// S_ij: row i strongly depends on j.
static void strength(const HostCsr &A, double theta, double mrs, std::vector<int> &srp,
                     std::vector<int> &sci) {
    i64 n = A.n;
    srp.assign(n + 1, 0);
    std::vector<std::vector<int>> rows(n);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) {
        double diag = 0.0, rsum = 0.0;
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            if (A.ci[j] == i) diag += A.v[j];
            rsum += A.v[j];
        }
        if (mrs < 1.0 && std::fabs(rsum) > std::fabs(diag) * mrs) continue;
        double s = diag < 0 ? -1.0 : 1.0;
        double scale = 0.0;
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j)
            if (A.ci[j] != i) scale = std::max(scale, -s * A.v[j]);
        if (scale <= 0.0) continue;
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            if (A.ci[j] == i) continue;
            double m = -s * A.v[j];
            if (m > 0.0 && m >= theta * scale) rows[i].push_back(A.ci[j]);
        }
    }
    for (i64 i = 0; i < n; ++i) srp[i + 1] = srp[i] + (int)rows[i].size();
    sci.resize(srp[n]);
    for (i64 i = 0; i < n; ++i) std::copy(rows[i].begin(), rows[i].end(), sci.begin() + srp[i]);
}

static void transpose_pattern(i64 n, const std::vector<int> &rp, const std::vector<int> &ci,
                              std::vector<int> &trp, std::vector<int> &tci) {
    trp.assign(n + 1, 0);
    for (int c : ci) trp[c + 1]++;
    for (i64 i = 0; i < n; ++i) trp[i + 1] += trp[i];
    tci.resize(ci.size());
    std::vector<int> pos(trp.begin(), trp.end() - 1);
    for (i64 i = 0; i < n; ++i)
        for (int j = rp[i]; j < rp[i + 1]; ++j) tci[pos[ci[j]]++] = (int)i;
}

enum { U_PT = 0, C_PT = 1, F_PT = -1 };

// Ruge-Stueben first pass with a bucket priority structure on the measure
// lambda_i = |S^T_i|.  Ties: the most recently (re)inserted point of the top
// bucket is taken first; initial insertion is in ascending index order.
static void rs_first_pass(i64 n, const std::vector<int> &srp, const std::vector<int> &sci,
                          const std::vector<int> &trp, const std::vector<int> &tci,
                          std::vector<int> &cf) {
    cf.assign(n, U_PT);
    std::vector<int> lam(n);
    int maxlam = 0;
    for (i64 i = 0; i < n; ++i) {
        lam[i] = trp[i + 1] - trp[i];
        maxlam = std::max(maxlam, lam[i]);
    }
    // points with no strong connection at all, or nobody depending on them
    for (i64 i = 0; i < n; ++i)
        if (lam[i] == 0) cf[i] = F_PT;
    int nb = maxlam + n + 2;  // measures can grow
    std::vector<int> head(nb, -1), nxt(n, -1), prv(n, -1);
    auto ins = [&](int i) {
        int b = lam[i];
        prv[i] = -1;
        nxt[i] = head[b];
        if (head[b] >= 0) prv[head[b]] = i;
        head[b] = i;
    };
    auto rem = [&](int i) {
        int b = lam[i];
        if (prv[i] >= 0) nxt[prv[i]] = nxt[i];
        else head[b] = nxt[i];
        if (nxt[i] >= 0) prv[nxt[i]] = prv[i];
        nxt[i] = prv[i] = -1;
    };
    int top = 0;
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == U_PT) {
            ins((int)i);
            top = std::max(top, lam[i]);
        }
    while (true) {
        while (top > 0 && head[top] < 0) --top;
        if (top <= 0) break;
        int i = head[top];
        rem(i);
        cf[i] = C_PT;
        for (int q = trp[i]; q < trp[i + 1]; ++q) {
            int j = tci[q];
            if (cf[j] != U_PT) continue;
            rem(j);
            cf[j] = F_PT;
            for (int r = srp[j]; r < srp[j + 1]; ++r) {
                int k = sci[r];
                if (cf[k] != U_PT) continue;
                rem(k);
                lam[k]++;
                ins(k);
                if (lam[k] > top) top = lam[k];
            }
        }
        for (int q = srp[i]; q < srp[i + 1]; ++q) {
            int j = sci[q];
            if (cf[j] != U_PT) continue;
            rem(j);
            lam[j]--;
            ins(j);
        }
    }
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == U_PT) cf[i] = F_PT;
}

// Classical second pass: an F point with a strong F neighbour that shares no
// strong C point with it makes that neighbour C (Ruge & Stueben, pass 2).
static void rs_second_pass(i64 n, const std::vector<int> &srp, const std::vector<int> &sci,
                           std::vector<int> &cf) {
    std::vector<int> mark(n, -1);
    for (i64 i = 0; i < n; ++i) {
        if (cf[i] != F_PT) continue;
        for (int q = srp[i]; q < srp[i + 1]; ++q)
            if (cf[sci[q]] == C_PT) mark[sci[q]] = (int)i;
        for (int q = srp[i]; q < srp[i + 1]; ++q) {
            int k = sci[q];
            if (cf[k] != F_PT) continue;
            bool shared = false;
            for (int r = srp[k]; r < srp[k + 1]; ++r)
                if (cf[sci[r]] == C_PT && mark[sci[r]] == (int)i) { shared = true; break; }
            if (!shared) {
                cf[k] = C_PT;
                mark[k] = (int)i;
            }
        }
    }
}

// Interpolation row truncation: drop weights below trunc * max|w|, keep the
// pmax largest (stable among equals, in the given order), rescale the kept
// weights to the row's original sum; then order by coarse index.
typedef std::vector<std::pair<int, double>> WRow;
static void truncate_row(WRow &w, double trunc, int pmax) {
    if (!w.empty() && (trunc > 0.0 || (pmax > 0 && (int)w.size() > pmax))) {
        double s0 = 0.0, mx = 0.0;
        for (auto &e : w) { s0 += e.second; mx = std::max(mx, std::fabs(e.second)); }
        WRow keep;
        for (auto &e : w)
            if (std::fabs(e.second) >= trunc * mx) keep.push_back(e);
        if (pmax > 0 && (int)keep.size() > pmax) {
            std::stable_sort(keep.begin(), keep.end(), [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                return std::fabs(a.second) > std::fabs(b.second);
            });
            keep.resize(pmax);
        }
        double s1 = 0.0;
        for (auto &e : keep) s1 += e.second;
        if (s1 != 0.0 && keep.size() != w.size())
            for (auto &e : keep) e.second *= s0 / s1;
        w.swap(keep);
    }
    std::sort(w.begin(), w.end());
}

// Extended+i interpolation with truncation.
static void ext_i_interp(const HostCsr &A, const std::vector<int> &srp,
                         const std::vector<int> &sci, const std::vector<int> &cf, double trunc,
                         int pmax, HostCsr &P) {
    i64 n = A.n;
    std::vector<int> cidx(n, -1);
    int nc = 0;
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == C_PT) cidx[i] = nc++;
    P.n = n;
    P.ncols = nc;
    std::vector<std::vector<std::pair<int, double>>> rows(n);
#pragma omp parallel
    {
        std::vector<int> pos(n, -1);     // column -> slot in hat-C list
        std::vector<char> isFs(n, 0);    // strong F neighbour flag
        std::vector<int> cl;
        std::vector<double> num;
#pragma omp for schedule(dynamic, 1024)
        for (i64 i = 0; i < n; ++i) {
            if (cf[i] == C_PT) {
                rows[i].push_back({cidx[i], 1.0});
                continue;
            }
            cl.clear();
            num.clear();
            std::vector<int> fs;
            for (int q = srp[i]; q < srp[i + 1]; ++q) {
                int j = sci[q];
                if (cf[j] == C_PT) {
                    if (pos[j] < 0) { pos[j] = (int)cl.size(); cl.push_back(j); num.push_back(0.0); }
                } else if (j != i) {
                    fs.push_back(j);
                    isFs[j] = 1;
                }
            }
            for (int k : fs)
                for (int q = srp[k]; q < srp[k + 1]; ++q) {
                    int l = sci[q];
                    if (cf[l] == C_PT && pos[l] < 0) {
                        pos[l] = (int)cl.size();
                        cl.push_back(l);
                        num.push_back(0.0);
                    }
                }
            double aii = 0.0;
            for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
                int c = A.ci[j];
                if (c == i) aii += A.v[j];
                else if (pos[c] >= 0) num[pos[c]] += A.v[j];
                else if (!isFs[c]) aii += A.v[j];  // weak: lumped to the diagonal
            }
            for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
                int k = A.ci[j];
                if (k == i || !isFs[k]) continue;
                double aik = A.v[j];
                double akk = 0.0;
                for (int q = A.rp[k]; q < A.rp[k + 1]; ++q)
                    if (A.ci[q] == k) akk += A.v[q];
                double sg = akk < 0 ? -1.0 : 1.0;
                double den = 0.0;
                for (int q = A.rp[k]; q < A.rp[k + 1]; ++q) {
                    int l = A.ci[q];
                    if (l == k) continue;
                    double v = A.v[q];
                    if (v * sg < 0 && (pos[l] >= 0 || l == i)) den += v;
                }
                if (den == 0.0) {
                    aii += aik;
                    continue;
                }
                for (int q = A.rp[k]; q < A.rp[k + 1]; ++q) {
                    int l = A.ci[q];
                    if (l == k) continue;
                    double v = A.v[q];
                    if (v * sg >= 0) continue;
                    if (pos[l] >= 0) num[pos[l]] += aik * v / den;
                    else if (l == i) aii += aik * v / den;
                }
            }
            std::vector<std::pair<int, double>> w;
            if (aii != 0.0)
                for (size_t q = 0; q < cl.size(); ++q) {
                    double wv = -num[q] / aii;
                    if (wv != 0.0) w.push_back({cidx[cl[q]], wv});
                }
            truncate_row(w, trunc, pmax);
            rows[i] = std::move(w);
            for (int c : cl) pos[c] = -1;
            for (int k : fs) isFs[k] = 0;
        }
    }
    P.rp.assign(n + 1, 0);
    for (i64 i = 0; i < n; ++i) P.rp[i + 1] = P.rp[i] + (int)rows[i].size();
    P.ci.resize(P.rp[n]);
    P.v.resize(P.rp[n]);
    for (i64 i = 0; i < n; ++i)
        for (size_t q = 0; q < rows[i].size(); ++q) {
            P.ci[P.rp[i] + q] = rows[i][q].first;
            P.v[P.rp[i] + q] = rows[i][q].second;
        }
}

// Aggressive coarsening, second stage (Stueben's A2 coarsening): among the
// first-stage C points, i depends on j when at least num_paths paths of
// length <= 2 lead from i to j along strong dependences (the direct one and
// one through every k with i -> k -> j); the C points are coarsened once
// more over that graph with the same passes.  A first-stage C point with no
// such connection in either direction stays C (it would otherwise be cut off
// from every coarse point).  cf is updated in place.
static void aggressive_second_stage(i64 n, const std::vector<int> &srp, const std::vector<int> &sci,
                                    int num_paths, int coarsen_type, std::vector<int> &cf) {
    std::vector<int> cid(n, -1), cpts;
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == C_PT) { cid[i] = (int)cpts.size(); cpts.push_back((int)i); }
    const i64 nc = (i64)cpts.size();
    std::vector<std::vector<int>> rows(nc);
#pragma omp parallel
    {
        std::vector<int> cnt(nc, 0), touched;
#pragma omp for schedule(dynamic, 512)
        for (i64 a = 0; a < nc; ++a) {
            const int i = cpts[a];
            touched.clear();
            auto hit = [&](int j) {
                if (j == i || cid[j] < 0) return;
                if (cnt[cid[j]]++ == 0) touched.push_back(cid[j]);
            };
            for (int q = srp[i]; q < srp[i + 1]; ++q) {
                const int k = sci[q];
                hit(k);
                for (int r = srp[k]; r < srp[k + 1]; ++r) hit(sci[r]);
            }
            std::sort(touched.begin(), touched.end());
            for (int b : touched) {
                if (cnt[b] >= num_paths) rows[a].push_back(b);
                cnt[b] = 0;
            }
        }
    }
    std::vector<int> s2rp(nc + 1, 0), s2ci, t2rp, t2ci, cf2;
    for (i64 a = 0; a < nc; ++a) s2rp[a + 1] = s2rp[a] + (int)rows[a].size();
    s2ci.reserve(s2rp[nc]);
    for (auto &r : rows) s2ci.insert(s2ci.end(), r.begin(), r.end());
    transpose_pattern(nc, s2rp, s2ci, t2rp, t2ci);
    rs_first_pass(nc, s2rp, s2ci, t2rp, t2ci, cf2);
    if (coarsen_type == 1 || coarsen_type == 3 || coarsen_type == 6) rs_second_pass(nc, s2rp, s2ci, cf2);
    for (i64 a = 0; a < nc; ++a) {
        const bool isolated = s2rp[a + 1] == s2rp[a] && t2rp[a + 1] == t2rp[a];
        if (cf2[a] != C_PT && !isolated) cf[cpts[a]] = F_PT;
    }
}

// Multipass interpolation (Stueben 2001, "multi-pass interpolation"): pass 1
// interpolates the F points with strong C neighbours directly from them; pass
// p > 1 interpolates the remaining F points that have strong neighbours
// interpolated in earlier passes through those neighbours' rows.  In every
// pass the weights of row i are -alpha a_ik / a_ii (negative a_ik) and -beta
// a_ik / a_ii (positive a_ik), with alpha (beta) the ratio of the sum of all
// negative (positive) off-diagonal entries of row i to the sum over the
// interpolating neighbours; positive entries with no positive interpolating
// neighbour are lumped into the diagonal.  F points that no pass reaches get
// an empty row.  Rows are truncated by trunc / pmax after all passes.
static void multipass_interp(const HostCsr &A, const std::vector<int> &srp, const std::vector<int> &sci,
                             const std::vector<int> &cf, double trunc, int pmax, HostCsr &P) {
    i64 n = A.n;
    std::vector<int> cidx(n, -1), pass(n, -1);
    int nc = 0;
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == C_PT) { cidx[i] = nc++; pass[i] = 0; }
    std::vector<WRow> rows(n);
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == C_PT) rows[i].push_back({cidx[i], 1.0});
    std::vector<char> strong(n, 0);
    for (int p = 1;; ++p) {
        std::vector<int> cur;
        for (i64 i = 0; i < n; ++i) {
            if (pass[i] >= 0) continue;
            for (int q = srp[i]; q < srp[i + 1]; ++q)
                if (pass[sci[q]] >= 0 && pass[sci[q]] < p) { cur.push_back((int)i); break; }
        }
        if (cur.empty()) break;
#pragma omp parallel
        {
            std::vector<char> isp(n, 0);
            std::vector<int> pos(nc, -1), cols;
            std::vector<double> vals;
#pragma omp for schedule(dynamic, 1024)
            for (size_t t = 0; t < cur.size(); ++t) {
                const int i = cur[t];
                for (int q = srp[i]; q < srp[i + 1]; ++q)
                    if (pass[sci[q]] >= 0 && pass[sci[q]] < p) isp[sci[q]] = 1;
                double aii = 0.0, nneg = 0.0, npos = 0.0, pneg = 0.0, ppos = 0.0;
                for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
                    const int c = A.ci[j];
                    const double a = A.v[j];
                    if (c == i) { aii += a; continue; }
                    if (a < 0) { nneg += a; if (isp[c]) pneg += a; }
                    else { npos += a; if (isp[c]) ppos += a; }
                }
                double beta = 0.0;
                if (ppos != 0.0) beta = npos / ppos;
                else aii += npos;
                const double alpha = pneg != 0.0 ? nneg / pneg : 0.0;
                cols.clear();
                vals.clear();
                if (aii != 0.0)
                    for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
                        const int k = A.ci[j];
                        if (k == i || !isp[k]) continue;
                        const double a = A.v[j];
                        const double f = -(a < 0 ? alpha : beta) * a / aii;
                        if (f == 0.0) continue;
                        for (auto &e : rows[k]) {
                            if (pos[e.first] < 0) {
                                pos[e.first] = (int)cols.size();
                                cols.push_back(e.first);
                                vals.push_back(0.0);
                            }
                            vals[pos[e.first]] += f * e.second;
                        }
                    }
                WRow w;
                for (size_t q = 0; q < cols.size(); ++q) {
                    if (vals[q] != 0.0) w.push_back({cols[q], vals[q]});
                    pos[cols[q]] = -1;
                }
                for (int q = srp[i]; q < srp[i + 1]; ++q) isp[sci[q]] = 0;
                rows[i].swap(w);
            }
        }
        for (int i : cur) pass[i] = p;
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (i64 i = 0; i < n; ++i)
        if (cf[i] != C_PT) truncate_row(rows[i], trunc, pmax);
    P.n = n;
    P.ncols = nc;
    P.rp.assign(n + 1, 0);
    for (i64 i = 0; i < n; ++i) P.rp[i + 1] = P.rp[i] + (int)rows[i].size();
    P.ci.resize(P.rp[n]);
    P.v.resize(P.rp[n]);
    for (i64 i = 0; i < n; ++i)
        for (size_t q = 0; q < rows[i].size(); ++q) {
            P.ci[P.rp[i] + q] = rows[i][q].first;
            P.v[P.rp[i] + q] = rows[i][q].second;
        }
}

// R = P^T in natural order (row c lists fine rows ascending).
void csr_transpose(const HostCsr &P, HostCsr &R) {
    R.n = P.ncols;
    R.ncols = P.n;
    R.rp.assign(R.n + 1, 0);
    for (int c : P.ci) R.rp[c + 1]++;
    for (i64 c = 0; c < R.n; ++c) R.rp[c + 1] += R.rp[c];
    R.ci.resize(P.ci.size());
    R.v.resize(P.v.size());
    std::vector<int> pos(R.rp.begin(), R.rp.end() - 1);
    for (i64 i = 0; i < P.n; ++i)
        for (int j = P.rp[i]; j < P.rp[i + 1]; ++j) {
            int p = pos[P.ci[j]]++;
            R.ci[p] = (int)i;
            R.v[p] = P.v[j];
        }
}

// A_c = R A P; coarse row I accumulates r_Ii * a_ij * p_jJ for i ascending in
// R_I, j in A_i order, J in P_j order.  Output: diagonal first, then ascending.
static void rap(const HostCsr &A, const HostCsr &P, const HostCsr &R, HostCsr &Ac) {
    i64 nc = P.ncols;
    Ac.n = Ac.ncols = nc;
    std::vector<std::vector<int>> cols(nc);
    std::vector<std::vector<double>> vals(nc);
#pragma omp parallel
    {
        std::vector<int> pos(nc, -1);
        std::vector<int> lc;
        std::vector<double> lv;
#pragma omp for schedule(dynamic, 256)
        for (i64 I = 0; I < nc; ++I) {
            lc.clear();
            lv.clear();
            for (int q = R.rp[I]; q < R.rp[I + 1]; ++q) {
                int i = R.ci[q];
                double r = R.v[q];
                for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
                    int c = A.ci[j];
                    double ra = r * A.v[j];
                    for (int t = P.rp[c]; t < P.rp[c + 1]; ++t) {
                        int J = P.ci[t];
                        if (pos[J] < 0) {
                            pos[J] = (int)lc.size();
                            lc.push_back(J);
                            lv.push_back(0.0);
                        }
                        lv[pos[J]] += ra * P.v[t];
                    }
                }
            }
            std::vector<int> ord(lc.size());
            std::iota(ord.begin(), ord.end(), 0);
            std::sort(ord.begin(), ord.end(), [&](int a, int b) {
                bool da = lc[a] == I, db = lc[b] == I;
                if (da != db) return da;
                return lc[a] < lc[b];
            });
            cols[I].resize(lc.size());
            vals[I].resize(lc.size());
            for (size_t q = 0; q < ord.size(); ++q) {
                cols[I][q] = lc[ord[q]];
                vals[I][q] = lv[ord[q]];
            }
            for (int c : lc) pos[c] = -1;
        }
    }
    Ac.rp.assign(nc + 1, 0);
    for (i64 I = 0; I < nc; ++I) Ac.rp[I + 1] = Ac.rp[I] + (int)cols[I].size();
    Ac.ci.resize(Ac.rp[nc]);
    Ac.v.resize(Ac.rp[nc]);
    for (i64 I = 0; I < nc; ++I) {
        std::copy(cols[I].begin(), cols[I].end(), Ac.ci.begin() + Ac.rp[I]);
        std::copy(vals[I].begin(), vals[I].end(), Ac.v.begin() + Ac.rp[I]);
    }
}

// Build the hierarchy.  levels[0].A is a copy of the fine operator.
void amg_setup(const HostCsr &A0, const AmgParams &prm, std::vector<AmgLevel> &levels) {
    amg_setup(A0, std::vector<AmgParams>(1, prm), levels);
}

void amg_setup(const HostCsr &A0, const std::vector<AmgParams> &prms, std::vector<AmgLevel> &levels) {
    levels.clear();
    levels.emplace_back();
    levels[0].A = A0;
    const AmgParams &top = prms.front();
    while ((int)levels.size() < top.max_levels) {
        const AmgParams &prm = prms[std::min(levels.size() - 1, prms.size() - 1)];
        HostCsr &A = levels.back().A;
        if (A.n <= top.coarse_size) break;
        std::vector<int> srp, sci, trp, tci, cf;
        strength(A, prm.theta, prm.max_row_sum, srp, sci);
        transpose_pattern(A.n, srp, sci, trp, tci);
        rs_first_pass(A.n, srp, sci, trp, tci, cf);
        if (prm.coarsen_type == 1 || prm.coarsen_type == 3 || prm.coarsen_type == 6)
            rs_second_pass(A.n, srp, sci, cf);
        if (prm.aggressive) aggressive_second_stage(A.n, srp, sci, prm.num_paths, prm.coarsen_type, cf);
        i64 nc = 0;
        for (int c : cf) nc += (c == C_PT);
        if (nc == 0 || nc == A.n) break;
        HostCsr P, R, Ac;
        if (prm.aggressive) multipass_interp(A, srp, sci, cf, prm.agg_trunc, prm.agg_pmax, P);
        else ext_i_interp(A, srp, sci, cf, prm.trunc, prm.pmax, P);
        csr_transpose(P, R);
        rap(A, P, R, Ac);
        levels.back().P = std::move(P);
        levels.emplace_back();
        levels.back().A = std::move(Ac);
    }
}

std::vector<AmgParams> amg_params_for(const GlobalParams &gp, const std::string &role) {
    const int L = std::max<int>(1, (int)gp.get(role).get_int("mg_max_levels"));
    std::vector<AmgParams> out;
    for (int l = 0; l < L; ++l) {
        const ParamList pl = gp.get_level(role, l);
        AmgParams ap;
        ap.max_levels = (int)pl.get_int("mg_max_levels");
        ap.coarse_size = (int)pl.get_int("mg_coarse_matrix_size");
        ap.theta = pl.get_float("mg_strength_threshold");
        ap.trunc = pl.get_float("mg_trunc_factor");
        ap.pmax = (int)pl.get_int("mg_Pmax_elements");
        ap.max_row_sum = pl.get_float("mg_max_row_sum");
        ap.coarsen_type = (int)pl.get_int("mg_coarsening_type");
        ap.interp_type = (int)pl.get_int("mg_interpolation_type");
        ap.aggressive = l < (int)pl.get_int("mg_agg_num_levels");
        ap.num_paths = std::max<int>(1, (int)pl.get_int("mg_num_paths"));
        ap.agg_interp = (int)pl.get_int("mg_agg_interpolation_type");
        ap.agg_trunc = pl.get_float("mg_agg_trunc_factor");
        ap.agg_pmax = (int)pl.get_int("mg_agg_Pmax_elements");
        if (ap.aggressive && ap.agg_interp != 4)
            throw Error("mg_agg_interpolation_type " + std::to_string(ap.agg_interp) +
                            " is not available (aggressive levels use multipass interpolation, type 4)",
                        4);
        out.push_back(ap);
    }
    return out;
}

}  // namespace xamg
