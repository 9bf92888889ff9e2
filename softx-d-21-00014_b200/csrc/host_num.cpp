// Host numerics of the setup phase (see host_num.h).
#include "host_num.h"

#include <cmath>

namespace xg {

template <typename T>
static std::vector<T> inv_diag_t(const HCsr &A, bool sqrt_) {
    std::vector<T> d(A.nrows, T(0));
    for (uint64_t i = 0; i < A.nrows; ++i)
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j)
            if ((uint64_t)A.col[j] == i) {
                const T v = (T)A.val[j];
                d[i] = sqrt_ ? (T)std::sqrt(1.0 / (double)v) : (T)(1.0 / (double)v);
            }
    return d;
}
std::vector<double> inv_diag_f64(const HCsr &A, bool s) { return inv_diag_t<double>(A, s); }
std::vector<float> inv_diag_f32(const HCsr &A, bool s) { return inv_diag_t<float>(A, s); }

template <typename T>
static std::vector<T> gj_inverse(const HCsr &A) {
    const uint64_t n = A.nrows, nc = 2 * n;
    std::vector<T> e(n * nc, T(0));
    for (uint64_t i = 0; i < n; ++i) {
        e[i * nc + i + n] = T(1.0);
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j) e[i * nc + A.col[j]] = (T)A.val[j];
    }
    for (uint64_t i = 0; i < n; ++i) {
        T *ri = &e[i * nc];
        for (uint64_t k = nc - 1; k > i; --k) ri[k] /= ri[i];
        ri[i] = T(1.0);
        for (uint64_t j = i + 1; j < n; ++j) {
            T *rj = &e[j * nc];
            for (uint64_t k = nc - 1; k > i; --k) rj[k] -= rj[i] * ri[k];
            rj[i] = T(0.0);
        }
    }
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t row = n - 1 - i;
        T *ri = &e[row * nc];
        for (uint64_t j = 0; j < row; ++j) {
            T *rj = &e[j * nc];
            for (uint64_t k = nc / 2; k < nc; ++k) rj[k] -= rj[row] * ri[k];
            rj[row] = T(0.0);
        }
    }
    std::vector<T> inv(n * n);
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = 0; j < n; ++j) inv[i * n + j] = e[i * nc + n + j];
    return inv;
}
std::vector<double> dense_inverse_f64(const HCsr &A) { return gj_inverse<double>(A); }
std::vector<float> dense_inverse_f32(const HCsr &A) { return gj_inverse<float>(A); }

std::vector<double> cheby_coeffs(double min_eig, double max_eig, int order, double frac) {
    const double upper = max_eig * 1.1;
    const double lower = (upper - min_eig) * frac + min_eig;
    const double theta = (upper + lower) / 2.;
    const double delta = (upper - lower) / 2.;
    std::vector<double> c(order > 0 ? order : 0, 0.0);
    double den;
    switch (order) {
    case 1:
        c[0] = 1. / theta;
        break;
    case 2:
        den = delta * delta - 2 * theta * theta;
        c[0] = -4 * theta / den;
        c[1] = 2 / den;
        break;
    case 3:
        den = 3 * (delta * delta) * theta - 4 * (theta * theta * theta);
        c[0] = (3 * delta * delta - 12 * theta * theta) / den;
        c[1] = 12 * theta / den;
        c[2] = -4 / den;
        break;
    case 4:
        den = std::pow(delta, 4) - 8 * delta * delta * theta * theta + 8 * std::pow(theta, 4);
        c[0] = (32 * std::pow(theta, 3) - 16 * delta * delta * theta) / den;
        c[1] = (8 * delta * delta - 48 * theta * theta) / den;
        c[2] = 32 * theta / den;
        c[3] = -8 / den;
        break;
    default:
        break;
    }
    return c;
}

}  // namespace xg
