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
    // aggressive coarsening on this level (level < mg_agg_num_levels):
    // second-stage coarsening of the C points over paths of length <= 2,
    // interpolation of type agg_interp (4 = multipass) truncated by
    // agg_trunc / agg_pmax
    bool aggressive = false;
    int num_paths = 3;
    int agg_interp = 4;
    double agg_trunc = 0.25;
    int agg_pmax = 4;
};

struct GlobalParams;
// Per-level parameters of the MultiGrid role `role` of gp (its per-level
// overrides "value@levA-B" applied), levels 0 .. mg_max_levels - 1.
// Throws (code 4) for settings this setup does not provide.
std::vector<AmgParams> amg_params_for(const GlobalParams &gp, const std::string &role);

struct AmgLevel {
    HostCsr A;  // operator of this level
    HostCsr P;  // n_l x n_{l+1} (empty on the coarsest level)
};

void amg_setup(const HostCsr &A0, const AmgParams &prm, std::vector<AmgLevel> &levels);
// level l is coarsened with prm[min(l, size - 1)]
void amg_setup(const HostCsr &A0, const std::vector<AmgParams> &prm, std::vector<AmgLevel> &levels);
void csr_transpose(const HostCsr &P, HostCsr &R);

}  // namespace xamg
