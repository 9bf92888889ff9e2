// Parameter dictionary (see params.h).
#include "params.h"

#include <cmath>
#include <cstdlib>
#include <sstream>

#include "common.h"

namespace xg {

std::string PValue::str() const {
    if (type == 'I') return std::to_string(i);
    if (type == 'F') {
        std::ostringstream o;
        o << f;
        return o.str();
    }
    return s;
}

std::string PList::get_s(const std::string &k, const std::string &def) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : it->second.str();
}
uint16_t PList::get_i(const std::string &k, uint16_t def) const {
    auto it = kv.find(k);
    if (it == kv.end()) return def;
    if (it->second.type == 'I') return it->second.i;
    if (it->second.type == 'F') return (uint16_t)it->second.f;
    return (uint16_t)std::strtoul(it->second.s.c_str(), nullptr, 10);
}
float PList::get_f(const std::string &k, float def) const {
    auto it = kv.find(k);
    if (it == kv.end()) return def;
    if (it->second.type == 'F') return it->second.f;
    if (it->second.type == 'I') return (float)it->second.i;
    return std::strtof(it->second.s.c_str(), nullptr);
}

// xamg_params_details.h:79-123 (type, families, min/max, allowed values),
// plus the B200 keys
static const std::map<std::string, KeyInfo> &dictionary() {
    static const std::map<std::string, KeyInfo> d = {
        {"method", {'S', "", "", "", ""}},
        {"convergence_check", {'I', "!Identity,!Direct", "0", "1", ""}},
        {"convergence_info", {'I', "!Identity,!Direct", "0", "1", ""}},
        {"polynomial_order", {'I', "Chebyshev", "1", "4", ""}},
        {"spectrum_fraction", {'F', "Chebyshev", "0.0", "1.0", ""}},
        {"max_iters", {'I', "!Identity,!Direct", "0", "inf", ""}},
        {"abs_tolerance", {'F', "!Identity,!Direct", "0.0", "inf", ""}},
        {"rel_tolerance", {'F', "!Identity,!Direct", "0.0", "inf", ""}},
        {"relax_factor", {'F', "Jacobi,HSGS", "", "", ""}},
        {"hypre_log", {'I', "MultiGrid", "0", "1", ""}},
        {"hypre_per_level_hierarchy", {'I', "MultiGrid", "0", "1", ""}},
        {"mg_reduced_precision", {'I', "MultiGrid", "0", "1", ""}},
        {"mg_cycle", {'I', "MultiGrid", "", "", "0,1,2"}},
        {"mg_max_levels", {'I', "MultiGrid", "1", "50", ""}},
        {"mg_coarse_matrix_size", {'I', "MultiGrid", "1", "2000", ""}},
        {"mg_strength_threshold", {'F', "MultiGrid", "0.0", "1.0", ""}},
        {"mg_trunc_factor", {'F', "MultiGrid", "0.0", "1.0", ""}},
        {"mg_num_paths", {'I', "MultiGrid", "1", "10", ""}},
        {"mg_coarsening_type", {'I', "MultiGrid", "0", "22", "0,1,3,6,7,8,9,10,11,21,22"}},
        {"mg_interpolation_type", {'I', "MultiGrid", "0", "14", ""}},
        {"mg_Pmax_elements", {'I', "MultiGrid", "0", "inf", ""}},
        {"mg_max_row_sum", {'F', "MultiGrid", "0.0", "1.0", ""}},
        {"mg_nonGalerkin_tol", {'F', "MultiGrid", "0.0", "1.0", ""}},
        {"mg_agg_num_levels", {'I', "MultiGrid", "0", "50", ""}},
        {"mg_agg_interpolation_type", {'I', "MultiGrid", "1", "4", ""}},
        {"mg_agg_trunc_factor", {'F', "MultiGrid", "0.0", "1.0", ""}},
        {"mg_agg_P12_trunc_factor", {'F', "MultiGrid", "0.0", "1.0", ""}},
        {"mg_agg_Pmax_elements", {'I', "MultiGrid", "0", "inf", ""}},
        {"mg_agg_P12max_elements", {'I', "MultiGrid", "0", "inf", ""}},
        {"gpu_precond_f32", {'I', "", "0", "1", ""}},
        {"gpu_coarse_f64", {'I', "", "0", "1", ""}},
        {"gpu_index_compress", {'I', "", "0", "3", ""}},
        {"gpu_hsgs_rows", {'I', "", "1", "inf", ""}},
        {"gpu_graph", {'I', "", "0", "1", ""}},
        {"gpu_spmv_tune", {'I', "", "0", "5", ""}},
        {"gpu_level_bf16", {'I', "", "0", "50", ""}},
        {"gpu_level_fp16", {'I', "", "0", "1", ""}},
        {"gpu_seed", {'I', "", "", "", ""}},
        {"gpu_persistent", {'I', "", "0", "16", ""}},
        {"gpu_solve_graph", {'I', "", "0", "1", ""}},
    };
    return d;
}

const KeyInfo *key_info(const std::string &key) {
    auto &d = dictionary();
    auto it = d.find(key);
    return it == d.end() ? nullptr : &it->second;
}

PValue Params::parse_typed(const std::string &key, const std::string &text) {
    PValue v;
    const KeyInfo *ki = key_info(key);
    v.type = ki ? ki->type : 'S';
    if (v.type == 'I')
        v.i = (uint16_t)std::strtoul(text.c_str(), nullptr, 10);
    else if (v.type == 'F')
        v.f = std::strtof(text.c_str(), nullptr);
    else
        v.s = text;
    return v;
}

static void check_key(const std::string &key) {
    XG_REQUIRE(key_info(key) != nullptr, XAMG_ERR_INVALID_ARG, "unknown parameter key: " + key);
}

// The value's range and allowed set (xamg_params_details.h:79-123): integer
// keys compare as the stored uint16, float keys as the stored float32.
static void check_value(const std::string &key, const PValue &v) {
    const KeyInfo *ki = key_info(key);
    if (!ki || ki->type == 'S') return;
    const double x = v.type == 'I'   ? (double)v.i
                     : v.type == 'F' ? (double)v.f
                                     : std::strtod(v.s.c_str(), nullptr);
    XG_REQUIRE(!std::isnan(x), XAMG_ERR_INVALID_ARG,
               "parameter " + key + " is NaN");
    const std::string mn = ki->min, mx = ki->max;
    if (!mn.empty())
        XG_REQUIRE(x >= (double)std::strtof(mn.c_str(), nullptr), XAMG_ERR_INVALID_ARG,
                   "parameter " + key + " = " + v.str() + " is below its minimum " + mn);
    if (!mx.empty() && mx != "inf")
        XG_REQUIRE(x <= (double)std::strtof(mx.c_str(), nullptr), XAMG_ERR_INVALID_ARG,
                   "parameter " + key + " = " + v.str() + " is above its maximum " + mx);
    const std::string al = ki->allowed;
    if (!al.empty()) {
        bool ok = false;
        std::stringstream ss(al);
        std::string a;
        while (std::getline(ss, a, ','))
            if (x == (double)std::strtof(a.c_str(), nullptr)) ok = true;
        XG_REQUIRE(ok, XAMG_ERR_INVALID_ARG,
                   "parameter " + key + " = " + v.str() + " is not one of {" + al + "}");
    }
}

void Params::add_value(const std::string &role, const std::string &key, const PValue &v) {
    check_key(key);
    check_value(key, v);
    lists[role].set(key, v);
}

void Params::change_value(const std::string &role, const std::string &key, const PValue &v) {
    check_key(key);
    auto it = lists.find(role);
    XG_REQUIRE(it != lists.end() && it->second.has(key), XAMG_ERR_INVALID_ARG,
               "change_value: " + role + "." + key + " is not set");
    check_value(key, v);
    it->second.set(key, v);
}

void Params::forced_change_value(const std::string &role, const std::string &key,
                                 const PValue &v) {
    check_key(key);
    check_value(key, v);
    lists[role].set(key, v);
}

// "value@levA-B" or "value@levA"; several comma-separated specs allowed
void Params::add_override(const std::string &role, const std::map<std::string, std::string> &ov) {
    for (auto &kvp : ov) {
        check_key(kvp.first);
        std::stringstream ss(kvp.second);
        std::string spec;
        while (std::getline(ss, spec, ',')) {
            size_t at = spec.find("@lev");
            XG_REQUIRE(at != std::string::npos, XAMG_ERR_INVALID_ARG,
                       "override must read value@levA-B: " + spec);
            std::string val = spec.substr(0, at);
            std::string range = spec.substr(at + 4);
            int a, b;
            size_t dash = range.find('-');
            if (dash == std::string::npos) {
                a = b = std::atoi(range.c_str());
            } else {
                a = std::atoi(range.substr(0, dash).c_str());
                b = std::atoi(range.substr(dash + 1).c_str());
            }
            XG_REQUIRE(a >= 0 && b >= a && b < 50, XAMG_ERR_INVALID_ARG,
                       "override level range out of 0..49: " + spec);
            check_value(kvp.first, parse_typed(kvp.first, val));
            for (int l = a; l <= b; ++l) overrides[role][l][kvp.first] = val;
        }
    }
}

static void set_if_missing(PList &l, const std::string &k, const PValue &v) {
    if (!l.has(k)) l.set(k, v);
}
static PValue I(uint16_t i) {
    PValue v;
    v.type = 'I';
    v.i = i;
    return v;
}
static PValue Fv(float f) {
    PValue v;
    v.type = 'F';
    v.f = f;
    return v;
}

// xamg_params_details.h:146-236
static void family_defaults(PList &list, const std::string &family, const std::string &role) {
    if (family == "Identity" || family == "Direct") return;
    if (family == "Chebyshev") {
        set_if_missing(list, "convergence_check", I(0));
        set_if_missing(list, "convergence_info", I(0));
        set_if_missing(list, "polynomial_order", I(2));
        set_if_missing(list, "spectrum_fraction", Fv(0.3f));
        return;
    }
    uint16_t iters = 0;
    float abs_tol = 0.f, rel_tol = 0.f;
    const bool solver = (role == "solver");
    if (solver) {
        abs_tol = 1.e-8f;
        rel_tol = 1.e-8f;
        set_if_missing(list, "convergence_check", I(1));
    } else {
        set_if_missing(list, "convergence_check", I(0));
    }
    set_if_missing(list, "convergence_info", I(0));
    if (family == "Jacobi" || family == "HSGS") {
        iters = solver ? 100 : 2;
        set_if_missing(list, "relax_factor", Fv(0.99f));
    } else if (family == "MultiGrid") {
        iters = solver ? 30 : 1;
        set_if_missing(list, "hypre_log", I(1));
        set_if_missing(list, "hypre_per_level_hierarchy", I(0));
        set_if_missing(list, "mg_reduced_precision", I(0));
        set_if_missing(list, "mg_cycle", I(0));
        set_if_missing(list, "mg_max_levels", I(25));
        set_if_missing(list, "mg_coarse_matrix_size", I(100));
        set_if_missing(list, "mg_strength_threshold", Fv(0.5f));
        set_if_missing(list, "mg_trunc_factor", Fv(0.25f));
        set_if_missing(list, "mg_num_paths", I(3));
        set_if_missing(list, "mg_coarsening_type", I(6));
        set_if_missing(list, "mg_interpolation_type", I(0));
        set_if_missing(list, "mg_max_row_sum", Fv(0.9f));
        set_if_missing(list, "mg_Pmax_elements", I(4));
        set_if_missing(list, "mg_nonGalerkin_tol", Fv(0.0f));
        set_if_missing(list, "mg_agg_num_levels", I(10));
        set_if_missing(list, "mg_agg_interpolation_type", I(4));
        set_if_missing(list, "mg_agg_trunc_factor", Fv(0.25f));
        set_if_missing(list, "mg_agg_P12_trunc_factor", Fv(0.0f));
        set_if_missing(list, "mg_agg_Pmax_elements", I(4));
        set_if_missing(list, "mg_agg_P12max_elements", I(4));
    } else if (family == "PCG" || family == "BiCGStab" || family == "MergedBiCGStab" ||
               family == "PBiCGStab" || family == "MergedPBiCGStab" || family == "RBiCGStab" ||
               family == "MergedRBiCGStab") {
        iters = solver ? 50 : 1;
    } else {
        throw Error(XAMG_ERR_INVALID_ARG, "method not found: " + family);
    }
    set_if_missing(list, "abs_tolerance", Fv(abs_tol));
    set_if_missing(list, "rel_tolerance", Fv(rel_tol));
    set_if_missing(list, "max_iters", I(iters));
}

// xamg_params_details.h:131-144 then family defaults per list
void Params::set_defaults() {
    bool mg = false;
    for (auto &l : lists)
        if (l.second.get_s("method") == "MultiGrid") mg = true;
    if (mg) {
        PValue m;
        if (!has("pre_smoother")) {
            m.s = "Jacobi";
            lists["pre_smoother"].set("method", m);
        }
        if (!has("post_smoother")) {
            m.s = "Jacobi";
            lists["post_smoother"].set("method", m);
        }
        if (!has("coarse_grid_solver")) {
            m.s = "Direct";
            lists["coarse_grid_solver"].set("method", m);
        }
    }
    for (auto &l : lists) {
        std::string fam = l.second.get_s("method");
        XG_REQUIRE(!fam.empty(), XAMG_ERR_INVALID_ARG, "list '" + l.first + "' has no method");
        family_defaults(l.second, fam, l.first);
    }
}

PList Params::get(const std::string &role, int level) const {
    PList out;
    auto it = lists.find(role);
    if (it != lists.end()) out = it->second;
    if (level >= 0) {
        auto r = overrides.find(role);
        if (r != overrides.end()) {
            auto lv = r->second.find(level);
            if (lv != r->second.end())
                for (auto &kv : lv->second) out.set(kv.first, parse_typed(kv.first, kv.second));
        }
    }
    // family defaults for whatever is still missing (the reference requires
    // XAMG_param_set_default to have run; here a missing key takes its default)
    std::string fam = out.get_s("method");
    if (!fam.empty()) family_defaults(out, fam, role);
    return out;
}

std::string Params::to_string() const {
    std::ostringstream o;
    static const char *order[] = {"solver", "preconditioner", "pre_smoother", "post_smoother",
                                  "coarse_grid_solver"};
    o << "------------------------------------------------------------\n";
    o << "XAMG library (B200 solve phase)\n";
    for (const char *role : order) {
        auto it = lists.find(role);
        if (it == lists.end()) continue;
        o << "[" << role << "]\n";
        for (auto &kv : it->second.kv) o << "  " << kv.first << " = " << kv.second.str() << "\n";
        auto ov = overrides.find(role);
        if (ov != overrides.end())
            for (auto &lv : ov->second)
                for (auto &kv : lv.second)
                    o << "  " << kv.first << " = " << kv.second << " @lev" << lv.first << "\n";
    }
    o << "------------------------------------------------------------\n";
    return o.str();
}

SolverCfg resolve_cfg(const PList &l, const std::string &role) {
    SolverCfg c;
    c.method = l.get_s("method");
    c.convergence_check = l.get_i("convergence_check", role == "solver" ? 1 : 0);
    c.convergence_info = l.get_i("convergence_info", 0);
    c.max_iters = l.get_i("max_iters", 1);
    c.abs_tol = l.get_f("abs_tolerance", 0.f);
    c.rel_tol = l.get_f("rel_tolerance", 0.f);
    c.relax = l.get_f("relax_factor", 0.99f);
    c.spec_fraction = l.get_f("spectrum_fraction", 0.3f);
    c.poly_order = l.get_i("polynomial_order", 2);
    c.mg_cycle = l.get_i("mg_cycle", 0);
    c.mg_reduced_precision = l.get_i("mg_reduced_precision", 0);
    c.mg_max_levels = l.get_i("mg_max_levels", 25);
    c.mg_coarse_matrix_size = l.get_i("mg_coarse_matrix_size", 100);
    c.mg_strength_threshold = l.get_f("mg_strength_threshold", 0.5f);
    c.mg_trunc_factor = l.get_f("mg_trunc_factor", 0.25f);
    c.mg_max_row_sum = l.get_f("mg_max_row_sum", 0.9f);
    c.mg_coarsening_type = l.get_i("mg_coarsening_type", 6);
    c.mg_interpolation_type = l.get_i("mg_interpolation_type", 0);
    c.mg_Pmax_elements = l.get_i("mg_Pmax_elements", 4);
    c.mg_agg_num_levels = l.get_i("mg_agg_num_levels", 10);
    c.mg_num_paths = l.get_i("mg_num_paths", 3);
    c.gpu_precond_f32 = l.has("gpu_precond_f32") ? (int)l.get_i("gpu_precond_f32") : -1;
    c.gpu_coarse_f64 = l.get_i("gpu_coarse_f64", 0);
    c.gpu_index_compress = l.get_i("gpu_index_compress", 1);
    c.gpu_hsgs_rows = l.get_i("gpu_hsgs_rows", 32);
    c.gpu_graph = l.get_i("gpu_graph", 1);
    c.gpu_spmv_tune = l.get_i("gpu_spmv_tune", 1);
    c.gpu_level_bf16 = l.get_i("gpu_level_bf16", 0);
    c.gpu_level_fp16 = l.get_i("gpu_level_fp16", 0);
    c.gpu_seed = l.get_i("gpu_seed", 0);
    c.gpu_persistent = l.get_i("gpu_persistent", 1);
    c.gpu_solve_graph = l.get_i("gpu_solve_graph", 1);
    return c;
}

}  // namespace xg
