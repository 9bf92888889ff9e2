// Matrix generators of the benchmark configurations (host, CSR with the
// diagonal first in every row).
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "../../include/xamg_b200.h"

namespace {

// examples/common/generator/cube.inl:28-174 (one rank): 7-point Laplacian
// with h = 1/n, boundary rows get 2q for the missing neighbour.
int64_t gen_cube(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t *row, uint32_t *col,
                 double *val) {
    const uint64_t n = nx * ny * nz;
    const double hx = 1.0 / nx, hy = 1.0 / ny, hz = 1.0 / nz;
    const double q1 = 1.0 / hx / hx, q2 = 1.0 / hy / hy, q3 = 1.0 / hz / hz;
    uint64_t c = 0;
    row[0] = 0;
    for (uint64_t indx = 0; indx < n; ++indx) {
        const uint64_t ii = indx % nx, jj = (indx / nx) % ny, kk = indx / (nx * ny);
        const uint64_t d = c;
        col[c] = (uint32_t)indx;
        val[c++] = 0.0;
        if (kk > 0) {
            val[d] += q3;
            col[c] = (uint32_t)(indx - nx * ny);
            val[c++] = -q3;
        } else if (nz > 1)
            val[d] += 2.0 * q3;
        if (jj > 0) {
            val[d] += q2;
            col[c] = (uint32_t)(indx - nx);
            val[c++] = -q2;
        } else if (ny > 1)
            val[d] += 2.0 * q2;
        if (ii > 0) {
            val[d] += q1;
            col[c] = (uint32_t)(indx - 1);
            val[c++] = -q1;
        } else if (nx > 1)
            val[d] += 2.0 * q1;
        if (ii < nx - 1) {
            val[d] += q1;
            col[c] = (uint32_t)(indx + 1);
            val[c++] = -q1;
        } else if (nx > 1)
            val[d] += 2.0 * q1;
        if (jj < ny - 1) {
            val[d] += q2;
            col[c] = (uint32_t)(indx + nx);
            val[c++] = -q2;
        } else if (ny > 1)
            val[d] += 2.0 * q2;
        if (kk < nz - 1) {
            val[d] += q3;
            col[c] = (uint32_t)(indx + nx * ny);
            val[c++] = -q3;
        } else if (nz > 1)
            val[d] += 2.0 * q3;
        row[indx + 1] = (uint32_t)c;
    }
    return (int64_t)c;
}

std::vector<double> cell_kappa(uint64_t cx, uint64_t cy, uint64_t cz, double sigma,
                               uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> N(0.0, 1.0);
    std::vector<double> k(cx * cy * cz);
    for (auto &v : k) v = std::exp(sigma * N(rng));
    return k;
}

// 7-point cell-centred finite volumes: unknown per cell, face transmissibility
// = harmonic mean of the two cell coefficients, Dirichlet boundary faces use
// 2*kappa (half-cell distance); z faces scaled by aniso_z.
int64_t gen_fv7(uint64_t nx, uint64_t ny, uint64_t nz, double sigma, double az, uint64_t seed,
                uint32_t *row, uint32_t *col, double *val) {
    const std::vector<double> kap = cell_kappa(nx, ny, nz, sigma, seed);
    const uint64_t n = nx * ny * nz;
    auto K = [&](uint64_t i, uint64_t j, uint64_t k) { return kap[(k * ny + j) * nx + i]; };
    auto harm = [](double a, double b) { return 2.0 * a * b / (a + b); };
    uint64_t c = 0;
    row[0] = 0;
    for (uint64_t idx = 0; idx < n; ++idx) {
        const uint64_t i = idx % nx, j = (idx / nx) % ny, k = idx / (nx * ny);
        const double kc = K(i, j, k);
        const uint64_t d = c;
        col[c] = (uint32_t)idx;
        val[c++] = 0.0;
        double diag = 0.0;
        auto nb = [&](bool inside, uint64_t nidx, double kn, double scale) {
            if (inside) {
                const double t = scale * harm(kc, kn);
                diag += t;
                col[c] = (uint32_t)nidx;
                val[c++] = -t;
            } else {
                diag += scale * 2.0 * kc;
            }
        };
        nb(k > 0, idx - nx * ny, k > 0 ? K(i, j, k - 1) : 0, az);
        nb(j > 0, idx - nx, j > 0 ? K(i, j - 1, k) : 0, 1.0);
        nb(i > 0, idx - 1, i > 0 ? K(i - 1, j, k) : 0, 1.0);
        nb(i + 1 < nx, idx + 1, i + 1 < nx ? K(i + 1, j, k) : 0, 1.0);
        nb(j + 1 < ny, idx + nx, j + 1 < ny ? K(i, j + 1, k) : 0, 1.0);
        nb(k + 1 < nz, idx + nx * ny, k + 1 < nz ? K(i, j, k + 1) : 0, az);
        val[d] = diag;
        row[idx + 1] = (uint32_t)c;
    }
    return (int64_t)c;
}

// 27-point trilinear (Q1) finite elements: unknowns at the nx*ny*nz interior
// nodes of an (nx+1)(ny+1)(nz+1) cell grid with per-cell kappa and Dirichlet
// boundary nodes eliminated. Element matrix on the unit cell:
// K_e[p][q] = kappa_e * sum_d a_d * S(p_d,q_d) * prod_{d' != d} M(p_d',q_d'),
// S = [[1,-1],[-1,1]], M = [[1/3,1/6],[1/6,1/3]], a = (1, 1, aniso_z).
int64_t gen_fe27(uint64_t nx, uint64_t ny, uint64_t nz, double sigma, double az, uint64_t seed,
                 uint32_t *row, uint32_t *col, double *val) {
    const uint64_t cx = nx + 1, cy = ny + 1, cz = nz + 1;
    const std::vector<double> kap = cell_kappa(cx, cy, cz, sigma, seed);
    const uint64_t n = nx * ny * nz;
    const double Sm[2][2] = {{1.0, -1.0}, {-1.0, 1.0}};
    const double Mm[2][2] = {{1.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 1.0 / 3.0}};
    const double a[3] = {1.0, 1.0, az};
    uint64_t c = 0;
    row[0] = 0;
    for (uint64_t idx = 0; idx < n; ++idx) {
        const int64_t P[3] = {(int64_t)(idx % nx) + 1, (int64_t)((idx / nx) % ny) + 1,
                              (int64_t)(idx / (nx * ny)) + 1};
        const int64_t dims[3] = {(int64_t)nx, (int64_t)ny, (int64_t)nz};
        const uint64_t dpos = c;
        col[c] = (uint32_t)idx;
        val[c++] = 0.0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int64_t Q[3] = {P[0] + dx, P[1] + dy, P[2] + dz};
                    bool inside = true;
                    for (int d = 0; d < 3; ++d)
                        if (Q[d] < 1 || Q[d] > dims[d]) inside = false;
                    if (!inside) continue;
                    // cells shared by nodes P and Q
                    int64_t lo[3], hi[3];
                    for (int d = 0; d < 3; ++d) {
                        if (P[d] == Q[d]) {
                            lo[d] = P[d] - 1;
                            hi[d] = P[d];
                        } else {
                            lo[d] = hi[d] = std::min(P[d], Q[d]);
                        }
                    }
                    double v = 0.0;
                    for (int64_t ez = lo[2]; ez <= hi[2]; ++ez)
                        for (int64_t ey = lo[1]; ey <= hi[1]; ++ey)
                            for (int64_t ex = lo[0]; ex <= hi[0]; ++ex) {
                                const int64_t e[3] = {ex, ey, ez};
                                int p[3], q[3];
                                for (int d = 0; d < 3; ++d) {
                                    p[d] = (int)(P[d] - e[d]);
                                    q[d] = (int)(Q[d] - e[d]);
                                }
                                double ke = 0.0;
                                for (int d = 0; d < 3; ++d) {
                                    double t = a[d] * Sm[p[d]][q[d]];
                                    for (int d2 = 0; d2 < 3; ++d2)
                                        if (d2 != d) t *= Mm[p[d2]][q[d2]];
                                    ke += t;
                                }
                                v += kap[((uint64_t)ez * cy + (uint64_t)ey) * cx + (uint64_t)ex] * ke;
                            }
                    const uint64_t qidx = ((uint64_t)(Q[2] - 1) * ny + (uint64_t)(Q[1] - 1)) * nx +
                                          (uint64_t)(Q[0] - 1);
                    if (qidx == idx) {
                        val[dpos] = v;
                    } else {
                        col[c] = (uint32_t)qidx;
                        val[c++] = v;
                    }
                }
        row[idx + 1] = (uint32_t)c;
    }
    return (int64_t)c;
}

}  // namespace

extern "C" {

int64_t XAMG_b200_generate_cube(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t *row,
                                uint32_t *col, double *val) {
    if (!row || !col || !val || nx == 0 || ny == 0 || nz == 0) return XAMG_ERR_INVALID_ARG;
    return gen_cube(nx, ny, nz, row, col, val);
}

int64_t XAMG_b200_generate_diffusion(int stencil, uint64_t nx, uint64_t ny, uint64_t nz,
                                     double sigma, double aniso_z, uint64_t seed, uint32_t *row,
                                     uint32_t *col, double *val) {
    if (!row || !col || !val || nx == 0 || ny == 0 || nz == 0) return XAMG_ERR_INVALID_ARG;
    if (stencil == 7) return gen_fv7(nx, ny, nz, sigma, aniso_z, seed, row, col, val);
    if (stencil == 27) return gen_fe27(nx, ny, nz, sigma, aniso_z, seed, row, col, val);
    return XAMG_ERR_INVALID_ARG;
}

}  // extern "C"
