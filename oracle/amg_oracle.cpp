// ORACLE-side problem generator and AMG hierarchy setup — test infrastructure
// only (loaded by the tests and by the CPU legs of the benchmark, never by
// the product library).
//
// The reference builds its hierarchy with hypre BoomerAMG (hypre 2.20.0,
// ThirdParty/dnb.sh:44, not vendored), configured at hypre_base.h:121-217:
// strength threshold (HYPRE_BoomerAMGSetStrongThreshold), max_row_sum,
// coarsening type (10 = HMIS, 6 = Falgout, ...), interpolation type
// (6 = extended+i), truncation factor and P_max.  hypre is absent here, so
// this file restates the published algorithms in the form a single process
// runs them, with the conventions below stated so that two independent
// restatements can be compared entry by entry:
//   * classical strength of connection (Ruge & Stueben 1987): j is a strong
//     dependence of i when -sign(a_ii) a_ij >= theta max_k(-sign(a_ii) a_ik)
//     and > 0; a row with |sum_j a_ij| > max_row_sum |a_ii| (max_row_sum < 1)
//     has no strong dependences;
//   * C/F splitting by the Ruge-Stueben first pass: repeatedly take the
//     undecided point with the largest measure |{j : j depends on it}|, make
//     it C and the undecided points that depend on it F, raise the measure of
//     the undecided points those new F points depend on, lower the measure of
//     the undecided points the new C point depends on.  Ties go to the point
//     whose measure changed last; before any change, to the larger index.
//     Points with measure 0 end as F.  On one process hypre's HMIS (type 10)
//     is this pass (De Sterck, Yang, Heys 2006); types 1, 3 and 6 add the
//     classical second pass (an F point with a strong F neighbour that shares
//     no strong C point with it turns that neighbour into C);
//   * extended+i interpolation (De Sterck, Falgout, Nolting, Yang 2008):
//     the interpolatory set of an F point i is its strong C neighbours and the
//     strong C neighbours of its strong F neighbours; entries of row i outside
//     that set and not strong F neighbours are lumped into the diagonal; each
//     strong F neighbour k is distributed over the set and i itself through
//     the entries of row k whose sign is opposite to a_kk (or lumped into the
//     diagonal when those sum to 0); weights w_ic = -num_c / diag;
//   * truncation: drop |w| < trunc_factor max|w|, keep the P_max largest
//     (stable among equals), rescale the kept weights to the row's original
//     sum;
//   * Galerkin coarse operator A_c = P^T A P, coarse rows diagonal first then
//     ascending columns.
// The accumulation orders (CSR order of A, discovery order of the
// interpolatory set, fine rows ascending in P^T) are part of the stated
// convention; the file is compiled with -ffp-contract=off.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <vector>
#include <omp.h>

typedef int64_t i64;

namespace orc_amg {

struct Csr {
    i64 n = 0, nc = 0;  // rows, columns
    std::vector<int> rp, ci;
    std::vector<double> v;
};

// ------------------------------------------------------------ 27-point operator
// The 27-point anisotropic diffusion operator of the benchmark: coupling to the
// neighbour at offset (dx,dy,dz) is -(kx dx^2 + ky dy^2 + kz dz^2) / |d|^4,
// the diagonal is the sum of all 26 couplings (Dirichlet boundary folded into
// the diagonal), rows lexicographic (x fastest), each row diagonal first then
// ascending columns.  Not a reference generator (the reference has none for
// this operator).
static void gen27(i64 n, double kx, double ky, double kz, Csr &A) {
    double wt[3][3][3];
    double diag = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
                int dz = a - 1, dy = b - 1, dx = c - 1;
                int r2 = dx * dx + dy * dy + dz * dz;
                wt[a][b][c] = r2 == 0 ? 0.0 : (kx * dx * dx + ky * dy * dy + kz * dz * dz) / double(r2 * r2);
                diag += wt[a][b][c];
            }
    i64 N = n * n * n;
    A.n = A.nc = N;
    A.rp.resize(N + 1);
    A.rp[0] = 0;
    auto span = [n](i64 t) { return 1 + (t > 0 ? 1 : 0) + (t < n - 1 ? 1 : 0); };
    for (i64 r = 0; r < N; ++r)
        A.rp[r + 1] = A.rp[r] + span(r % n) * span((r / n) % n) * span(r / (n * n));
    A.ci.resize(A.rp[N]);
    A.v.resize(A.rp[N]);
#pragma omp parallel for schedule(static)
    for (i64 r = 0; r < N; ++r) {
        i64 x = r % n, y = (r / n) % n, z = r / (n * n);
        int q = A.rp[r];
        A.ci[q] = (int)r;
        A.v[q++] = diag;
        for (int a = 0; a < 3; ++a) {
            i64 zz = z + a - 1;
            if (zz < 0 || zz >= n) continue;
            for (int b = 0; b < 3; ++b) {
                i64 yy = y + b - 1;
                if (yy < 0 || yy >= n) continue;
                for (int c = 0; c < 3; ++c) {
                    i64 xx = x + c - 1;
                    if (xx < 0 || xx >= n || (a == 1 && b == 1 && c == 1)) continue;
                    A.ci[q] = (int)((zz * n + yy) * n + xx);
                    A.v[q++] = -wt[a][b][c];
                }
            }
        }
    }
}

// ------------------------------------------------------------------ strength
struct Pattern {
    std::vector<int> rp, ci;
};

static Pattern strong_deps(const Csr &A, double theta, double max_row_sum) {
    i64 n = A.n;
    std::vector<std::vector<int>> row(n);
#pragma omp parallel for schedule(dynamic, 4096)
    for (i64 i = 0; i < n; ++i) {
        double aii = 0.0, sum = 0.0;
        for (int q = A.rp[i]; q < A.rp[i + 1]; ++q) {
            sum += A.v[q];
            if (A.ci[q] == i) aii += A.v[q];
        }
        if (max_row_sum < 1.0 && std::fabs(sum) > std::fabs(aii) * max_row_sum) continue;
        double sgn = aii < 0 ? -1.0 : 1.0, big = 0.0;
        for (int q = A.rp[i]; q < A.rp[i + 1]; ++q)
            if (A.ci[q] != i) big = std::max(big, -sgn * A.v[q]);
        if (!(big > 0.0)) continue;
        for (int q = A.rp[i]; q < A.rp[i + 1]; ++q) {
            if (A.ci[q] == i) continue;
            double m = -sgn * A.v[q];
            if (m > 0.0 && m >= theta * big) row[i].push_back(A.ci[q]);
        }
    }
    Pattern S;
    S.rp.assign(n + 1, 0);
    for (i64 i = 0; i < n; ++i) S.rp[i + 1] = S.rp[i] + (int)row[i].size();
    S.ci.reserve(S.rp[n]);
    for (i64 i = 0; i < n; ++i) S.ci.insert(S.ci.end(), row[i].begin(), row[i].end());
    return S;
}

// rows of the transpose list their sources ascending
static Pattern transpose(i64 n, const Pattern &S) {
    Pattern T;
    T.rp.assign(n + 1, 0);
    for (int c : S.ci) ++T.rp[c + 1];
    for (i64 i = 0; i < n; ++i) T.rp[i + 1] += T.rp[i];
    T.ci.resize(S.ci.size());
    std::vector<int> fill(T.rp.begin(), T.rp.end() - 1);
    for (i64 i = 0; i < n; ++i)
        for (int q = S.rp[i]; q < S.rp[i + 1]; ++q) T.ci[fill[S.ci[q]]++] = (int)i;
    return T;
}

// ---------------------------------------------------------------- coarsening
enum : signed char { UNDECIDED = 0, COARSE = 1, FINE = -1 };

// Ruge-Stueben first pass.  The undecided points sit in buckets by measure;
// each bucket is a stack with lazy deletion (an entry is live while its stamp
// is the point's current stamp), so the point pushed last is found first.
static std::vector<signed char> first_pass(i64 n, const Pattern &S, const Pattern &St) {
    std::vector<signed char> cf(n, UNDECIDED);
    std::vector<int> meas(n);
    std::vector<i64> stamp(n, -1);
    std::vector<std::vector<std::pair<int, i64>>> bucket(1);
    i64 clock = 0;
    int hi = 0;
    auto push = [&](int i) {
        stamp[i] = clock++;
        if ((int)bucket.size() <= meas[i]) bucket.resize(meas[i] + 1);
        bucket[meas[i]].push_back({i, stamp[i]});
        hi = std::max(hi, meas[i]);
    };
    for (i64 i = 0; i < n; ++i) {
        meas[i] = St.rp[i + 1] - St.rp[i];
        if (meas[i] == 0) cf[i] = FINE;
    }
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == UNDECIDED) push((int)i);
    for (;;) {
        int pick = -1;
        while (hi > 0 && pick < 0) {
            auto &bk = bucket[hi];
            while (!bk.empty()) {
                auto e = bk.back();
                bk.pop_back();
                if (cf[e.first] == UNDECIDED && stamp[e.first] == e.second && meas[e.first] == hi) {
                    pick = e.first;
                    break;
                }
            }
            if (pick < 0) --hi;
        }
        if (pick < 0) break;
        cf[pick] = COARSE;
        stamp[pick] = -1;
        for (int q = St.rp[pick]; q < St.rp[pick + 1]; ++q) {
            int j = St.ci[q];
            if (cf[j] != UNDECIDED) continue;
            cf[j] = FINE;
            stamp[j] = -1;
            for (int r = S.rp[j]; r < S.rp[j + 1]; ++r) {
                int k = S.ci[r];
                if (cf[k] != UNDECIDED) continue;
                ++meas[k];
                push(k);
            }
        }
        for (int q = S.rp[pick]; q < S.rp[pick + 1]; ++q) {
            int j = S.ci[q];
            if (cf[j] != UNDECIDED) continue;
            --meas[j];
            push(j);
        }
    }
    for (auto &c : cf)
        if (c == UNDECIDED) c = FINE;
    return cf;
}

static void second_pass(i64 n, const Pattern &S, std::vector<signed char> &cf) {
    std::vector<int> owner(n, -1);  // C point -> last F point that listed it
    for (i64 i = 0; i < n; ++i) {
        if (cf[i] != FINE) continue;
        for (int q = S.rp[i]; q < S.rp[i + 1]; ++q)
            if (cf[S.ci[q]] == COARSE) owner[S.ci[q]] = (int)i;
        for (int q = S.rp[i]; q < S.rp[i + 1]; ++q) {
            int k = S.ci[q];
            if (cf[k] != FINE) continue;
            bool common = false;
            for (int r = S.rp[k]; r < S.rp[k + 1] && !common; ++r)
                common = cf[S.ci[r]] == COARSE && owner[S.ci[r]] == (int)i;
            if (!common) {
                cf[k] = COARSE;
                owner[k] = (int)i;
            }
        }
    }
}

// ------------------------------------------------------ extended+i interpolation
static Csr interpolation(const Csr &A, const Pattern &S, const std::vector<signed char> &cf,
                         double trunc, int pmax) {
    i64 n = A.n;
    std::vector<int> cnum(n, -1);
    int nc = 0;
    for (i64 i = 0; i < n; ++i)
        if (cf[i] == COARSE) cnum[i] = nc++;
    std::vector<std::vector<std::pair<int, double>>> prow(n);
#pragma omp parallel
    {
        std::vector<int> slot(n, -1);       // interpolatory set membership
        std::vector<char> strongF(n, 0);
        std::vector<int> set;               // interpolatory set, discovery order
        std::vector<double> num;
        std::vector<int> fnb;
#pragma omp for schedule(dynamic, 2048)
        for (i64 i = 0; i < n; ++i) {
            if (cf[i] == COARSE) {
                prow[i] = {{cnum[i], 1.0}};
                continue;
            }
            set.clear();
            num.clear();
            fnb.clear();
            auto enter = [&](int c) {
                if (slot[c] < 0) {
                    slot[c] = (int)set.size();
                    set.push_back(c);
                    num.push_back(0.0);
                }
            };
            for (int q = S.rp[i]; q < S.rp[i + 1]; ++q) {
                int j = S.ci[q];
                if (cf[j] == COARSE) enter(j);
                else if (j != i) { fnb.push_back(j); strongF[j] = 1; }
            }
            for (int k : fnb)
                for (int q = S.rp[k]; q < S.rp[k + 1]; ++q)
                    if (cf[S.ci[q]] == COARSE) enter(S.ci[q]);
            double d = 0.0;
            for (int q = A.rp[i]; q < A.rp[i + 1]; ++q) {
                int c = A.ci[q];
                if (c == i) d += A.v[q];
                else if (slot[c] >= 0) num[slot[c]] += A.v[q];
                else if (!strongF[c]) d += A.v[q];
            }
            for (int q = A.rp[i]; q < A.rp[i + 1]; ++q) {
                int k = A.ci[q];
                if (k == i || !strongF[k]) continue;
                double aik = A.v[q];
                double akk = 0.0;
                for (int r = A.rp[k]; r < A.rp[k + 1]; ++r)
                    if (A.ci[r] == k) akk += A.v[r];
                bool neg = akk < 0;
                auto opposite = [neg](double x) { return neg ? x > 0 : x < 0; };
                double den = 0.0;
                for (int r = A.rp[k]; r < A.rp[k + 1]; ++r) {
                    int l = A.ci[r];
                    if (l != k && opposite(A.v[r]) && (slot[l] >= 0 || l == i)) den += A.v[r];
                }
                if (den == 0.0) {
                    d += aik;
                    continue;
                }
                for (int r = A.rp[k]; r < A.rp[k + 1]; ++r) {
                    int l = A.ci[r];
                    if (l == k || !opposite(A.v[r])) continue;
                    double share = aik * A.v[r] / den;
                    if (slot[l] >= 0) num[slot[l]] += share;
                    else if (l == i) d += share;
                }
            }
            std::vector<std::pair<int, double>> w;
            if (d != 0.0)
                for (size_t t = 0; t < set.size(); ++t) {
                    double x = -num[t] / d;
                    if (x != 0.0) w.push_back({cnum[set[t]], x});
                }
            bool cut = !w.empty() && (trunc > 0.0 || (pmax > 0 && (int)w.size() > pmax));
            if (cut) {
                double total = 0.0, wmax = 0.0;
                for (auto &e : w) {
                    total += e.second;
                    wmax = std::max(wmax, std::fabs(e.second));
                }
                std::vector<std::pair<int, double>> kept;
                for (auto &e : w)
                    if (std::fabs(e.second) >= trunc * wmax) kept.push_back(e);
                if (pmax > 0 && (int)kept.size() > pmax) {
                    std::stable_sort(kept.begin(), kept.end(),
                                     [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                                         return std::fabs(a.second) > std::fabs(b.second);
                                     });
                    kept.resize(pmax);
                }
                double ksum = 0.0;
                for (auto &e : kept) ksum += e.second;
                if (ksum != 0.0 && kept.size() != w.size())
                    for (auto &e : kept) e.second *= total / ksum;
                w.swap(kept);
            }
            std::sort(w.begin(), w.end());
            prow[i].swap(w);
            for (int c : set) slot[c] = -1;
            for (int k : fnb) strongF[k] = 0;
        }
    }
    Csr P;
    P.n = n;
    P.nc = nc;
    P.rp.assign(n + 1, 0);
    for (i64 i = 0; i < n; ++i) P.rp[i + 1] = P.rp[i] + (int)prow[i].size();
    P.ci.reserve(P.rp[n]);
    P.v.reserve(P.rp[n]);
    for (i64 i = 0; i < n; ++i)
        for (auto &e : prow[i]) {
            P.ci.push_back(e.first);
            P.v.push_back(e.second);
        }
    return P;
}

// ------------------------------------------------------------ Galerkin product
static Csr transpose(const Csr &P) {
    Csr R;
    R.n = P.nc;
    R.nc = P.n;
    R.rp.assign(R.n + 1, 0);
    for (int c : P.ci) ++R.rp[c + 1];
    for (i64 c = 0; c < R.n; ++c) R.rp[c + 1] += R.rp[c];
    R.ci.resize(P.ci.size());
    R.v.resize(P.v.size());
    std::vector<int> at(R.rp.begin(), R.rp.end() - 1);
    for (i64 i = 0; i < P.n; ++i)
        for (int q = P.rp[i]; q < P.rp[i + 1]; ++q) {
            int t = at[P.ci[q]]++;
            R.ci[t] = (int)i;
            R.v[t] = P.v[q];
        }
    return R;
}

static Csr galerkin(const Csr &A, const Csr &P, const Csr &R) {
    i64 nc = P.nc;
    std::vector<std::vector<std::pair<int, double>>> crow(nc);
#pragma omp parallel
    {
        std::vector<int> at(nc, -1);
        std::vector<int> cols;
        std::vector<double> vals;
#pragma omp for schedule(dynamic, 512)
        for (i64 I = 0; I < nc; ++I) {
            cols.clear();
            vals.clear();
            for (int q = R.rp[I]; q < R.rp[I + 1]; ++q) {
                int i = R.ci[q];
                double rI = R.v[q];
                for (int r = A.rp[i]; r < A.rp[i + 1]; ++r) {
                    int j = A.ci[r];
                    double ra = rI * A.v[r];
                    for (int t = P.rp[j]; t < P.rp[j + 1]; ++t) {
                        int J = P.ci[t];
                        if (at[J] < 0) {
                            at[J] = (int)cols.size();
                            cols.push_back(J);
                            vals.push_back(0.0);
                        }
                        vals[at[J]] += ra * P.v[t];
                    }
                }
            }
            auto &row = crow[I];
            row.resize(cols.size());
            for (size_t t = 0; t < cols.size(); ++t) {
                row[t] = {cols[t], vals[t]};
                at[cols[t]] = -1;
            }
            int II = (int)I;
            std::sort(row.begin(), row.end(),
                      [II](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                          if ((a.first == II) != (b.first == II)) return a.first == II;
                          return a.first < b.first;
                      });
        }
    }
    Csr Ac;
    Ac.n = Ac.nc = nc;
    Ac.rp.assign(nc + 1, 0);
    for (i64 I = 0; I < nc; ++I) Ac.rp[I + 1] = Ac.rp[I] + (int)crow[I].size();
    Ac.ci.reserve(Ac.rp[nc]);
    Ac.v.reserve(Ac.rp[nc]);
    for (i64 I = 0; I < nc; ++I)
        for (auto &e : crow[I]) {
            Ac.ci.push_back(e.first);
            Ac.v.push_back(e.second);
        }
    return Ac;
}

struct Hierarchy {
    std::vector<Csr> A, P;  // P[l]: n_l x n_{l+1}; empty on the coarsest level
};

struct Params {
    int max_levels, coarse_size, coarsen_type;
    double theta, trunc, max_row_sum;
    int pmax;
};

static void setup(const Csr &A0, const Params &p, Hierarchy &H) {
    H.A.clear();
    H.P.clear();
    H.A.push_back(A0);
    while ((int)H.A.size() < p.max_levels && H.A.back().n > p.coarse_size) {
        const Csr &A = H.A.back();
        Pattern S = strong_deps(A, p.theta, p.max_row_sum);
        Pattern St = transpose(A.n, S);
        std::vector<signed char> cf = first_pass(A.n, S, St);
        if (p.coarsen_type == 1 || p.coarsen_type == 3 || p.coarsen_type == 6) second_pass(A.n, S, cf);
        i64 nc = std::count(cf.begin(), cf.end(), (signed char)COARSE);
        if (nc == 0 || nc == A.n) break;
        Csr P = interpolation(A, S, cf, p.trunc, p.pmax);
        Csr R = transpose(P);
        Csr Ac = galerkin(A, P, R);
        H.P.push_back(std::move(P));
        H.A.push_back(std::move(Ac));
    }
    H.P.resize(H.A.size());
}

}  // namespace orc_amg

using namespace orc_amg;

extern "C" {

// 27-point operator: orc_gen27_size gives (rows, nnz); orc_gen27 fills.
void orc_gen27_size(i64 n, i64 *rows, i64 *nnz) {
    auto span = [n](i64 t) { return 1 + (t > 0 ? 1 : 0) + (t < n - 1 ? 1 : 0); };
    i64 s = 0;
    for (i64 t = 0; t < n; ++t) s += span(t);
    *rows = n * n * n;
    *nnz = s * s * s;
}
void orc_gen27(i64 n, double kx, double ky, double kz, int *rp, int *ci, double *v) {
    Csr A;
    gen27(n, kx, ky, kz, A);
    std::copy(A.rp.begin(), A.rp.end(), rp);
    std::copy(A.ci.begin(), A.ci.end(), ci);
    std::copy(A.v.begin(), A.v.end(), v);
}

void *orc_amg_setup(i64 n, const int *rp, const int *ci, const double *v, int max_levels, int coarse_size,
                    double theta, double trunc, int pmax, double max_row_sum, int coarsen_type) {
    Csr A;
    A.n = A.nc = n;
    A.rp.assign(rp, rp + n + 1);
    A.ci.assign(ci, ci + rp[n]);
    A.v.assign(v, v + rp[n]);
    Params p{max_levels, coarse_size, coarsen_type, theta, trunc, max_row_sum, pmax};
    auto *H = new Hierarchy;
    setup(A, p, *H);
    return H;
}
int orc_amg_num_levels(void *h) { return (int)((Hierarchy *)h)->A.size(); }
// info: rows, nnz of A_l, columns and nnz of P_l
void orc_amg_level_info(void *h, int l, i64 *info) {
    auto *H = (Hierarchy *)h;
    info[0] = H->A[l].n;
    info[1] = H->A[l].rp.back();
    info[2] = H->P[l].n ? H->P[l].nc : 0;
    info[3] = H->P[l].n ? H->P[l].rp.back() : 0;
}
void orc_amg_level_export(void *h, int l, int *arp, int *aci, double *av, int *prp, int *pci, double *pv) {
    auto *H = (Hierarchy *)h;
    const Csr &A = H->A[l], &P = H->P[l];
    std::copy(A.rp.begin(), A.rp.end(), arp);
    std::copy(A.ci.begin(), A.ci.end(), aci);
    std::copy(A.v.begin(), A.v.end(), av);
    if (P.n && prp) {
        std::copy(P.rp.begin(), P.rp.end(), prp);
        std::copy(P.ci.begin(), P.ci.end(), pci);
        std::copy(P.v.begin(), P.v.end(), pv);
    }
}
void orc_amg_destroy(void *h) { delete (Hierarchy *)h; }

}  // extern "C"
