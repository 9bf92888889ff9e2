// Solver parameter dictionary with XAMG's surface: per-role lists
// ("solver", "preconditioner", "pre_smoother", "post_smoother",
// "coarse_grid_solver"), typed keys (string / uint16 / float32), the family
// defaults of src/param/xamg_params_details.h:131-236 and per-level overrides
// written "value@levA-B" (examples/c/example.c:185-190,
// yaml/multi_node/config-channel-cube2.yaml:28-30).
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace xg {

struct PValue {
    char type = 'S';  // 'S' string, 'I' uint16, 'F' float32
    std::string s;
    uint16_t i = 0;
    float f = 0.f;
    std::string str() const;
};

struct PList {
    std::map<std::string, PValue> kv;
    bool has(const std::string &k) const { return kv.count(k) > 0; }
    std::string get_s(const std::string &k, const std::string &def = "") const;
    uint16_t get_i(const std::string &k, uint16_t def = 0) const;
    float get_f(const std::string &k, float def = 0.f) const;
    void set(const std::string &k, const PValue &v) { kv[k] = v; }
};

// Keys the dictionary knows, with value type, the families they apply to,
// and the value range and allowed set (xamg_params_details.h:79-123).
struct KeyInfo {
    char type;
    const char *families;  // comma-separated; "!X" excludes; empty = all
    const char *min;       // "" = no bound
    const char *max;       // "" or "inf" = no bound
    const char *allowed;   // comma-separated allowed values; "" = any in range
};
const KeyInfo *key_info(const std::string &key);

class Params {
  public:
    std::map<std::string, PList> lists;
    // per role: level -> key -> value string
    std::map<std::string, std::map<int, std::map<std::string, std::string>>> overrides;

    // XAMG_param_add_value_* (xamg_c_api.cpp:115-128)
    void add_value(const std::string &role, const std::string &key, const PValue &v);
    // XAMG_param_change_value_* : key must already be present
    void change_value(const std::string &role, const std::string &key, const PValue &v);
    // XAMG_param_forced_change_value_* : set whether present or not
    void forced_change_value(const std::string &role, const std::string &key, const PValue &v);
    // XAMG_param_override_apply: "value@levA-B" strings per key
    void add_override(const std::string &role, const std::map<std::string, std::string> &ov);
    // XAMG_param_set_default: dictionary and family defaults
    void set_defaults();
    bool has(const std::string &role) const { return lists.count(role) > 0; }
    // the role's list with the overrides of `level` applied (level < 0: none)
    PList get(const std::string &role, int level = -1) const;
    std::string to_string() const;

    static PValue parse_typed(const std::string &key, const std::string &text);
};

// Resolved settings of one solver object.
struct SolverCfg {
    std::string method;
    int convergence_check = 0, convergence_info = 0, max_iters = 1;
    float abs_tol = 0.f, rel_tol = 0.f, relax = 0.99f, spec_fraction = 0.3f;
    int poly_order = 2;
    // MultiGrid
    int mg_cycle = 0, mg_reduced_precision = 0, mg_max_levels = 25, mg_coarse_matrix_size = 100;
    float mg_strength_threshold = 0.5f, mg_trunc_factor = 0.25f, mg_max_row_sum = 0.9f;
    int mg_coarsening_type = 6, mg_interpolation_type = 0, mg_Pmax_elements = 4;
    int mg_agg_num_levels = 10, mg_num_paths = 3;
    // B200 extension keys
    int gpu_precond_f32 = -1;   // -1: follow mg_reduced_precision
    int gpu_coarse_f64 = 0;     // keep the Direct coarse solve in FP64 when reduced
    int gpu_index_compress = 1; // XAMG narrowing of column indices on upload
    int gpu_hsgs_rows = 32;     // target rows per hybrid Gauss-Seidel block
    int gpu_graph = 1;          // replay preconditioner applications as CUDA graphs
    int gpu_spmv_tune = 1;      // SpMV launch shapes picked by measurement (2: no tuning,
                                // the grid-stencil kernel's 128-register form; 3: no
                                // tuning, the warp-per-row kernel on small matrices;
                                // 4: no tuning, the x-staged kernel where built; 5: no
                                // tuning, the plane walk where the matrix has one)
    int gpu_level_bf16 = 0;     // finest FP32 cycle levels whose matrix values are BF16
    int gpu_level_fp16 = 0;     // 1: those levels store FP16 values with a per-level
                                // power-of-two scale instead of BF16
    int gpu_seed = 0;           // seed of the host setup's random choices
    int gpu_persistent = 1;     // eligible BiCGStab solves in one cooperative launch, each
                                // block playing this many canonical blocks (0: off)
    int gpu_solve_graph = 1;    // whole BiCGStab solves as one graph with a device-side loop
};

SolverCfg resolve_cfg(const PList &l, const std::string &role);

}  // namespace xg
