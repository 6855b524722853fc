// Row partition of one system over several ranks (host side of a multi-GPU
// solve).  Rank r owns the contiguous rows [first[r], first[r+1]) — the
// reference's block partition (part.h: equal blocks, the remainder on the
// last).  Its local matrix keeps every owned row's entries in CSR order with
// the columns renumbered: owned columns first (column - first[r]), then the
// halo columns (rows owned by other ranks) in ascending global order, so a
// product over [own x | halo x] runs each row's FMA chain exactly as the
// single-system product does.  Send lists give, per peer, the owned rows
// that peer needs, in the order of the peer's halo.
#pragma once
#include "common.h"

namespace xamg {

struct RowPart {
    int nranks = 1, rank = 0;
    std::vector<i64> first;        // nranks + 1 row boundaries
    std::vector<int> lrp, lci;     // local CSR (columns renumbered)
    std::vector<i64> lsrc;         // global entry index of every local entry
    std::vector<i64> halo;         // global row of every halo slot (ascending)
    std::vector<int> halo_owner;   // owning rank of every halo slot
    std::vector<std::vector<i64>> sends;  // per peer: owned rows (global) the peer needs
    i64 nrows() const { return first[rank + 1] - first[rank]; }
    void build(i64 n, const int *rp, const int *ci, int nranks_, int rank_);
};

// the reference's block boundaries for n rows over p ranks
std::vector<i64> row_blocks(i64 n, int p);

}  // namespace xamg
