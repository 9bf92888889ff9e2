// Inputs of the CPU oracle arm: the seeded test matrices and the multigrid
// hierarchy, for processes that must not load the CUDA library (the timed
// CPU baseline of bench.py).
//
// TEST INFRASTRUCTURE ONLY, like oracle.cpp. It compiles the library's two
// host-only input stages from their single source (csrc/generators.cpp and
// csrc/amg.cpp, no CUDA) so that the CPU arm solves exactly the matrix and
// hierarchy the GPU solves. In XAMG the hierarchy comes from hypre's
// BoomerAMG setup (hypre_base.inl:337-403; hypre 2.20.0 is not available),
// so both arms share one stand-in for that setup stage; everything after it
// (the solve phase) is restated separately in oracle.cpp.
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "../softx-d-21-00014_b200/csrc/amg.h"

using xg::HCsr;
using xg::Hierarchy;

extern "C" {

// Builds the hierarchy of the double matrix (row, col, val) with the
// multigrid parameters the library resolves for its preconditioner list
// (float fields as stored there). Returns a handle for os_hier_* below.
void *os_hier_build(uint64_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col,
                    const double *val, float strength, float max_row_sum, int max_levels,
                    int coarse_size, float trunc, int pmax, int seed) {
    HCsr A;
    A.nrows = n;
    A.ncols = n;
    A.row.assign(row, row + n + 1);
    A.col.assign(col, col + nnz);
    A.val.assign(val, val + nnz);
    xg::SolverCfg cfg;
    cfg.method = "MultiGrid";
    cfg.mg_strength_threshold = strength;
    cfg.mg_max_row_sum = max_row_sum;
    cfg.mg_max_levels = max_levels;
    cfg.mg_coarse_matrix_size = coarse_size;
    cfg.mg_trunc_factor = trunc;
    cfg.mg_Pmax_elements = pmax;
    cfg.gpu_seed = seed;
    return new Hierarchy(xg::build_hierarchy(A, cfg));
}

void os_hier_free(void *h) { delete (Hierarchy *)h; }

int os_hier_levels(void *h) { return (int)((Hierarchy *)h)->lv.size(); }

// which = 0: A_l, 1: P_l (absent on the last level: nrows = 0). With null
// arrays only the sizes are returned.
void os_hier_level(void *h, int level, int which, uint64_t *nrows, uint64_t *ncols, uint64_t *nnz,
                   uint32_t *row, uint32_t *col, double *val, double *min_eig, double *max_eig) {
    const xg::HLevel &L = ((Hierarchy *)h)->lv[level];
    const HCsr &m = which == 0 ? L.A : L.P;
    *nrows = m.row.empty() ? 0 : m.nrows;
    *ncols = m.ncols;
    *nnz = m.col.size();
    *min_eig = L.min_eig;
    *max_eig = L.max_eig;
    if (row && !m.row.empty()) std::memcpy(row, m.row.data(), m.row.size() * sizeof(uint32_t));
    if (col) std::memcpy(col, m.col.data(), m.col.size() * sizeof(uint32_t));
    if (val) std::memcpy(val, m.val.data(), m.val.size() * sizeof(double));
}

}  // extern "C"
