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
            // truncation: relative threshold, then at most pmax entries; keep row sum
            if (!w.empty() && (trunc > 0.0 || (pmax > 0 && (int)w.size() > pmax))) {
                double s0 = 0.0, mx = 0.0;
                for (auto &e : w) { s0 += e.second; mx = std::max(mx, std::fabs(e.second)); }
                std::vector<std::pair<int, double>> keep;
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
    levels.clear();
    levels.emplace_back();
    levels[0].A = A0;
    while ((int)levels.size() < prm.max_levels) {
        HostCsr &A = levels.back().A;
        if (A.n <= prm.coarse_size) break;
        std::vector<int> srp, sci, trp, tci, cf;
        strength(A, prm.theta, prm.max_row_sum, srp, sci);
        transpose_pattern(A.n, srp, sci, trp, tci);
        rs_first_pass(A.n, srp, sci, trp, tci, cf);
        if (prm.coarsen_type == 1 || prm.coarsen_type == 3 || prm.coarsen_type == 6)
            rs_second_pass(A.n, srp, sci, cf);
        i64 nc = 0;
        for (int c : cf) nc += (c == C_PT);
        if (nc == 0 || nc == A.n) break;
        HostCsr P, R, Ac;
        ext_i_interp(A, srp, sci, cf, prm.trunc, prm.pmax, P);
        csr_transpose(P, R);
        rap(A, P, R, Ac);
        levels.back().P = std::move(P);
        levels.emplace_back();
        levels.back().A = std::move(Ac);
    }
}

}  // namespace xamg
