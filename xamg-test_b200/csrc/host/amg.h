// Host-side AMG setup interface (see amg.cpp).
#pragma once
#include "common.h"

namespace xamg {

struct AmgParams {
    int max_levels = 25;
    int coarse_size = 100;
    double theta = 0.5;
    double trunc = 0.25;
    int pmax = 4;
    double max_row_sum = 0.9;
    int coarsen_type = 10;
    int interp_type = 6;
};

struct AmgLevel {
    HostCsr A;  // operator of this level
    HostCsr P;  // n_l x n_{l+1} (empty on the coarsest level)
};

void amg_setup(const HostCsr &A0, const AmgParams &prm, std::vector<AmgLevel> &levels);
void csr_transpose(const HostCsr &P, HostCsr &R);

}  // namespace xamg
