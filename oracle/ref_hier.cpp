// Entry point of oracle/_ref/libxamg_ref_nv*.so beside the reference's own C
// API (api/c/xamg_c_api.cpp, compiled unmodified from where it lies): hands
// the hypre stand-in the hierarchy that its BoomerAMG setup returns.
// TEST INFRASTRUCTURE ONLY.
#include "ref_shim/prelude.h"
#include "ref_shim/HYPRE.h"

extern "C" void xamg_ref_set_hierarchy(int nlev, const int *n, const uint32_t *const *arow,
                                       const uint32_t *const *acol, const double *const *aval,
                                       const uint32_t *const *prow, const uint32_t *const *pcol,
                                       const double *const *pval, const double *min_eig,
                                       const double *max_eig) {
    xamg_ref_hypre_set_hierarchy(nlev, n, arow, acol, aval, prow, pcol, pval, min_eig, max_eig);
}
