// Row partition and halo plan of one system over several ranks (see dist.h).
#include "dist.h"
#include <algorithm>

namespace xamg {

std::vector<i64> row_blocks(i64 n, int p) {
    std::vector<i64> f((size_t)p + 1, 0);
    const i64 bs = n / p;
    for (int r = 0; r < p; ++r) f[r + 1] = r + 1 < p ? f[r] + bs : n;
    return f;
}

static int owner(const std::vector<i64> &first, i64 row) {
    return (int)(std::upper_bound(first.begin(), first.end(), row) - first.begin()) - 1;
}

// halo columns of rank r: the distinct columns of its rows outside its block
static std::vector<i64> halo_of(i64 r0, i64 r1, const int *rp, const int *ci) {
    std::vector<i64> h;
    for (i64 i = r0; i < r1; ++i)
        for (int j = rp[i]; j < rp[i + 1]; ++j)
            if (ci[j] < r0 || ci[j] >= r1) h.push_back(ci[j]);
    std::sort(h.begin(), h.end());
    h.erase(std::unique(h.begin(), h.end()), h.end());
    return h;
}

void RowPart::build(i64 n, const int *rp, const int *ci, int nranks_, int rank_) {
    XCHECK(nranks_ >= 1 && rank_ >= 0 && rank_ < nranks_ && n >= nranks_, "bad partition arguments");
    nranks = nranks_;
    rank = rank_;
    first = row_blocks(n, nranks);
    const i64 r0 = first[rank], r1 = first[rank + 1], nl = r1 - r0;
    halo = halo_of(r0, r1, rp, ci);
    halo_owner.resize(halo.size());
    for (size_t h = 0; h < halo.size(); ++h) halo_owner[h] = owner(first, halo[h]);
    lrp.assign((size_t)nl + 1, 0);
    lci.clear();
    lsrc.clear();
    for (i64 i = r0; i < r1; ++i) {
        for (int j = rp[i]; j < rp[i + 1]; ++j) {
            const i64 c = ci[j];
            i64 lc;
            if (c >= r0 && c < r1) lc = c - r0;
            else lc = nl + (std::lower_bound(halo.begin(), halo.end(), c) - halo.begin());
            lci.push_back((int)lc);
            lsrc.push_back(j);
        }
        lrp[i - r0 + 1] = (int)lci.size();
    }
    // send lists: the rows of this block in every peer's halo, in its order
    sends.assign(nranks, {});
    for (int p = 0; p < nranks; ++p) {
        if (p == rank) continue;
        for (i64 c : halo_of(first[p], first[p + 1], rp, ci))
            if (c >= r0 && c < r1) sends[p].push_back(c);
    }
}

}  // namespace xamg
