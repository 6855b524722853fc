// Solver parameter dictionary with the reference's roles, keys and defaults.
//
// Roles: meta_solver, solver, preconditioner, pre_smoother, post_smoother,
// coarse_grid_solver, residual_control (param/xamg_params_details.h:87-134).
// Defaults follow set_dictionary_defaults / set_family_defaults
// (xamg_params_details.h:142-289).  Per-level overrides use the reference's
// "value@levA-B" syntax (examples/c/example.c:190-193, mg.inl:84-113).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace xamg {

struct PValue {
    char t = 'S';  // 'S' string, 'I' integer, 'F' float, 'B' bool
    std::string s;
    uint64_t i = 0;
    double f = 0.0;
    bool b = false;
    std::string str() const;
};

struct ParamList {
    std::map<std::string, PValue> m;
    bool has(const std::string &k) const { return m.count(k) > 0; }
    std::string get_string(const std::string &k) const;
    uint64_t get_int(const std::string &k) const;
    double get_float(const std::string &k) const;
    bool get_bool(const std::string &k) const;
    void set(const std::string &k, const PValue &v) { m[k] = v; }
    void set_s(const std::string &k, const std::string &v);
    void set_i(const std::string &k, uint64_t v);
    void set_f(const std::string &k, double v);
    void set_b(const std::string &k, bool v);
    void set_s_missing(const std::string &k, const std::string &v) { if (!has(k)) set_s(k, v); }
    void set_i_missing(const std::string &k, uint64_t v) { if (!has(k)) set_i(k, v); }
    void set_f_missing(const std::string &k, double v) { if (!has(k)) set_f(k, v); }
    void set_b_missing(const std::string &k, bool v) { if (!has(k)) set_b(k, v); }
};

struct GlobalParams {
    std::map<std::string, ParamList> roles;
    // role -> key -> raw override string ("8@lev0-1")
    std::map<std::string, std::map<std::string, std::string>> overrides;
    bool has(const std::string &role) const { return roles.count(role) > 0; }
    ParamList &get(const std::string &role);
    const ParamList &get(const std::string &role) const;
    // role's list with the overrides that apply to `level`
    ParamList get_level(const std::string &role, int level) const;
    void set_defaults();
    void print() const;
    // Checks a key against the reference's expected-parameter table: known
    // key and value type.  Returns "" when fine, else a message.
    static std::string validate(const std::string &key, char type);
};

}  // namespace xamg
