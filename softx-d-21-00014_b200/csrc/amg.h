// Host multigrid setup (amg.cpp): the hierarchy a hypre BoomerAMG setup would
// hand to XAMG (hypre_base.inl:337-403).
#pragma once

#include <vector>

#include "hcsr.h"
#include "params.h"

namespace xg {

// Level matrices A_l, interpolations P_l (n_l x n_{l+1}) and the eigenvalue
// estimates of D^-1/2 A_l D^-1/2 used by Chebyshev smoothing.
struct HLevel {
    HCsr A, P;
    double min_eig = 0.0, max_eig = 0.0;
};
struct Hierarchy {
    std::vector<HLevel> lv;
};

Hierarchy build_hierarchy(const HCsr &A0, const SolverCfg &mg);
void estimate_eigs(const HCsr &A, int iters, uint64_t seed, double &mn, double &mx);

}  // namespace xg
