// Host-side numerics of the setup phase that the device solve consumes:
// inverse diagonals, the dense coarse inverse and the Chebyshev coefficients.
// Compiled with -ffp-contract=off so that each multiply and add is rounded on
// its own, as in the reference build.
#pragma once

#include <cstdint>
#include <vector>

#include "hcsr.h"

namespace xg {

// csr_matrix.h:302-368: 1/a_ii (or sqrt(1/a_ii)) evaluated in double from the
// value as stored in the level precision, then stored in that precision.
std::vector<double> inv_diag_f64(const HCsr &A, bool sqrt_);
std::vector<float> inv_diag_f32(const HCsr &A, bool sqrt_);

// inverse.inl:31-106: Gauss-Jordan on [A | I] without pivoting, in the level
// precision, of the dense copy of a CSR matrix.
std::vector<double> dense_inverse_f64(const HCsr &A);
std::vector<float> dense_inverse_f32(const HCsr &A);

// chebyshev.inl:50-127 (double; the caller rounds to the level precision)
std::vector<double> cheby_coeffs(double min_eig, double max_eig, int order, double frac);

}  // namespace xg
