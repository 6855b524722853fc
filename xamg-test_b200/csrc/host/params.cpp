#include "params.h"
#include "common.h"
#include <set>
#include <sstream>

namespace xamg {

std::string PValue::str() const {
    std::ostringstream o;
    switch (t) {
    case 'S': o << s; break;
    case 'I': o << i; break;
    case 'F': o << f; break;
    default: o << (b ? "true" : "false"); break;
    }
    return o.str();
}

static const PValue &need(const ParamList &l, const std::string &k) {
    auto it = l.m.find(k);
    if (it == l.m.end()) throw Error("parameter not set: " + k, 2);
    return it->second;
}
std::string ParamList::get_string(const std::string &k) const { return need(*this, k).str(); }
uint64_t ParamList::get_int(const std::string &k) const {
    const PValue &v = need(*this, k);
    if (v.t == 'I') return v.i;
    if (v.t == 'F') return (uint64_t)v.f;
    if (v.t == 'B') return v.b;
    return std::stoull(v.s);
}
double ParamList::get_float(const std::string &k) const {
    const PValue &v = need(*this, k);
    if (v.t == 'F') return v.f;
    if (v.t == 'I') return (double)v.i;
    if (v.t == 'B') return v.b;
    return std::stod(v.s);
}
bool ParamList::get_bool(const std::string &k) const {
    const PValue &v = need(*this, k);
    if (v.t == 'B') return v.b;
    if (v.t == 'I') return v.i != 0;
    if (v.t == 'F') return v.f != 0.0;
    return v.s == "1" || v.s == "true" || v.s == "yes";
}
void ParamList::set_s(const std::string &k, const std::string &v) { PValue p; p.t = 'S'; p.s = v; m[k] = p; }
void ParamList::set_i(const std::string &k, uint64_t v) { PValue p; p.t = 'I'; p.i = v; m[k] = p; }
void ParamList::set_f(const std::string &k, double v) { PValue p; p.t = 'F'; p.f = v; m[k] = p; }
void ParamList::set_b(const std::string &k, bool v) { PValue p; p.t = 'B'; p.b = v; m[k] = p; }

ParamList &GlobalParams::get(const std::string &role) {
    auto it = roles.find(role);
    if (it == roles.end()) throw Error("parameter role missing: " + role, 2);
    return it->second;
}
const ParamList &GlobalParams::get(const std::string &role) const {
    auto it = roles.find(role);
    if (it == roles.end()) throw Error("parameter role missing: " + role, 2);
    return it->second;
}

// "v@levA-B" / "v@levA" / "v"
static bool override_value(const std::string &raw, int level, std::string &val) {
    auto at = raw.find('@');
    if (at == std::string::npos) {
        val = raw;
        return true;
    }
    val = raw.substr(0, at);
    std::string r = raw.substr(at + 1);
    if (r.rfind("lev", 0) == 0) r = r.substr(3);
    int a = 0, b = 0;
    auto dash = r.find('-');
    if (dash == std::string::npos) a = b = std::stoi(r);
    else { a = std::stoi(r.substr(0, dash)); b = std::stoi(r.substr(dash + 1)); }
    return level >= a && level <= b;
}

ParamList GlobalParams::get_level(const std::string &role, int level) const {
    ParamList l = get(role);
    auto it = overrides.find(role);
    if (it == overrides.end() || level < 0) return l;
    for (auto &kv : it->second) {
        std::string v;
        if (!override_value(kv.second, level, v)) continue;
        auto cur = l.m.find(kv.first);
        char t = cur == l.m.end() ? 'S' : cur->second.t;
        if (t == 'I') l.set_i(kv.first, std::stoull(v));
        else if (t == 'F') l.set_f(kv.first, std::stod(v));
        else if (t == 'B') l.set_b(kv.first, v == "1" || v == "true");
        else l.set_s(kv.first, v);
    }
    return l;
}

static void str_split(const std::string &s, char d, std::set<std::string> &out) {
    std::string cur;
    for (char c : s) {
        if (c == d) { if (!cur.empty()) out.insert(cur); cur.clear(); }
        else cur += c;
    }
    if (!cur.empty()) out.insert(cur);
}

// set_family_defaults (xamg_params_details.h:171-289)
static void family_defaults(ParamList &l, const std::string &role) {
    std::string method = l.get_string("method");
    if (method == "Identity" || method == "Direct") return;
    if (method == "IterativeRefinement") {
        l.set_b_missing("subsolver_reduced_precision", false);
        l.set_f_missing("abs_tolerance", 1e-8);
        l.set_f_missing("rel_tolerance", 1e-8);
        l.set_s_missing("convergence_details", "check-L2,print");
        l.set_i_missing("max_iters", 20);
        return;
    }
    if (method == "Chebyshev") {
        l.set_s_missing("convergence_details", "nocheck,noprint");
        l.set_i_missing("polynomial_order", 2);
        l.set_f_missing("spectrum_fraction", 0.3);
        l.set_f_missing("abs_tolerance", 0);
        l.set_f_missing("rel_tolerance", 0);
        return;
    }
    uint64_t iters = 0;
    if (role == "solver" || role == "meta_solver") {
        l.set_f_missing("abs_tolerance", 1e-8);
        l.set_f_missing("rel_tolerance", 1e-8);
        l.set_s_missing("convergence_details", "check-L2,print");
    } else {
        l.set_f_missing("abs_tolerance", 0);
        l.set_f_missing("rel_tolerance", 0);
        l.set_s_missing("convergence_details", "nocheck,noprint");
    }
    if (method == "Jacobi" || method == "HSGS") {
        iters = role == "solver" ? 100 : 2;
        l.set_f_missing("relax_factor", 0.99);
        if (method == "HSGS") l.set_i_missing("hybrid_block_rows", 0);
    } else if (method == "MultiGrid") {
        iters = role == "solver" ? 30 : 1;
        l.set_b_missing("hypre_log", true);
        l.set_b_missing("hypre_per_level_hierarchy", false);
        l.set_b_missing("mg_reduced_precision", false);
        l.set_i_missing("mg_cycle", 0);
        l.set_i_missing("mg_max_levels", 25);
        l.set_i_missing("mg_coarse_matrix_size", 100);
        l.set_f_missing("mg_strength_threshold", 0.5);
        l.set_f_missing("mg_trunc_factor", 0.25);
        l.set_i_missing("mg_num_paths", 3);
        l.set_i_missing("mg_coarsening_type", 6);
        l.set_i_missing("mg_interpolation_type", 0);
        l.set_f_missing("mg_max_row_sum", 0.9);
        l.set_i_missing("mg_Pmax_elements", 4);
        l.set_f_missing("mg_nonGalerkin_tol", 0.0);
        l.set_i_missing("mg_agg_num_levels", 10);
        l.set_i_missing("mg_agg_interpolation_type", 4);
        l.set_f_missing("mg_agg_trunc_factor", 0.25);
        l.set_f_missing("mg_agg_P12_trunc_factor", 0.0);
        l.set_i_missing("mg_agg_Pmax_elements", 4);
        l.set_i_missing("mg_agg_P12max_elements", 4);
    } else if (method == "PCG" || method == "BiCGStab" || method == "MergedBiCGStab" ||
               method == "PBiCGStab" || method == "MergedPBiCGStab" || method == "RBiCGStab" ||
               method == "MergedRBiCGStab") {
        iters = role == "solver" ? 50 : 1;
    } else {
        throw Error("method not found: " + method, 2);
    }
    l.set_i_missing("max_iters", iters);
}

void GlobalParams::set_defaults() {
    bool mg = false;
    for (auto &r : roles)
        if (r.second.has("method") && r.second.get_string("method") == "MultiGrid") mg = true;
    if (mg) {
        if (!has("pre_smoother")) roles["pre_smoother"].set_s("method", "Jacobi");
        if (!has("post_smoother")) roles["post_smoother"].set_s("method", "Jacobi");
        if (!has("coarse_grid_solver")) roles["coarse_grid_solver"].set_s("method", "Direct");
    }
    for (auto &r : roles) {
        if (r.first == "residual_control") continue;
        if (!r.second.has("method")) throw Error("role without method: " + r.first, 2);
        family_defaults(r.second, r.first);
        if (r.second.has("convergence_details")) {
            std::set<std::string> cd;
            str_split(r.second.get_string("convergence_details"), ',', cd);
            if (cd.count("RR") && !has("residual_control"))
                throw Error("residual_control parameters block must be present in RR mode", 2);
        }
    }
}

void GlobalParams::print() const {
    for (auto &r : roles) {
        printf("[%s]\n", r.first.c_str());
        for (auto &kv : r.second.m) printf("  %-28s %s\n", kv.first.c_str(), kv.second.str().c_str());
    }
    for (auto &o : overrides)
        for (auto &kv : o.second) printf("  override %s.%s = %s\n", o.first.c_str(), kv.first.c_str(), kv.second.c_str());
}

std::string GlobalParams::validate(const std::string &key, char type) {
    static const std::map<std::string, char> known = {
        {"method", 'S'}, {"polynomial_order", 'I'}, {"spectrum_fraction", 'F'},
        {"max_iters", 'I'}, {"subsolver_reduced_precision", 'B'}, {"convergence_details", 'S'},
        {"abs_tolerance", 'F'}, {"rel_tolerance", 'F'}, {"RR_deviation", 'F'},
        {"RR_stepping", 'F'}, {"relax_factor", 'F'}, {"hypre_log", 'B'},
        {"hypre_per_level_hierarchy", 'B'}, {"mg_reduced_precision", 'B'}, {"mg_cycle", 'I'},
        {"mg_max_levels", 'I'}, {"mg_coarse_matrix_size", 'I'}, {"mg_strength_threshold", 'F'},
        {"mg_trunc_factor", 'F'}, {"mg_num_paths", 'I'}, {"mg_coarsening_type", 'I'},
        {"mg_interpolation_type", 'I'}, {"mg_Pmax_elements", 'I'}, {"mg_max_row_sum", 'F'},
        {"mg_nonGalerkin_tol", 'F'}, {"mg_agg_num_levels", 'I'},
        {"mg_agg_interpolation_type", 'I'}, {"mg_agg_trunc_factor", 'F'},
        {"mg_agg_P12_trunc_factor", 'F'}, {"mg_agg_Pmax_elements", 'I'},
        {"mg_agg_P12max_elements", 'I'},
        // extensions of this library (no reference counterpart)
        {"hybrid_block_rows", 'I'}, {"inner_rel_tolerance", 'F'}, {"gs_schedule", 'S'},
        {"rel_tolerance_base", 'S'}, {"hybrid_blocks", 'I'}, {"dot_order", 'S'}};
    auto it = known.find(key);
    if (it == known.end()) return "unknown parameter: " + key;
    if (it->second != type && !(it->second == 'F' && type == 'I'))
        return "parameter " + key + " has the wrong value type";
    return "";
}

}  // namespace xamg
