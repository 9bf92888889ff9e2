// Host algebraic multigrid setup: the part of the solve-phase pipeline that
// the reference delegates to hypre 2.20.0 BoomerAMG (src/hypre/hypre_base.h:
// 118-213, hypre_base.inl:322-403). hypre is not available here, so the
// hierarchy is built by this restatement of the published algorithms:
//
//  * classical strength of connection with threshold theta and the
//    max-row-sum rule (Ruge-Stueben; hypre's CreateS convention: for a positive
//    diagonal, a_ij is strong when a_ij < theta * min_k a_ik);
//  * PMIS coarsening (De Sterck, Yang, Heys, SIAM J. Matrix Anal. Appl. 27,
//    2006): measure = number of points depending on i plus a seeded uniform
//    random number in [0,1); points that no one depends on start as F;
//  * extended+i interpolation (De Sterck, Falgout, Nolting, Yang, Numer. Linear
//    Algebra Appl. 15, 2008): distance-two C points, strong F neighbours
//    distributed over C_hat and i with the opposite-sign entries of their rows,
//    weak connections lumped into the diagonal;
//  * interpolation truncation by trunc_factor and P_max elements per row with
//    the row sum restored;
//  * Galerkin coarse operators A_c = P^T A P with the diagonal stored first in
//    each row;
//  * Chebyshev eigenvalue bounds of D^-1/2 A D^-1/2 from 10 steps of CG
//    (Lanczos tridiagonal eigenvalues), as hypre does for relax type 16.
//
// Parameters read: mg_strength_threshold, mg_max_row_sum, mg_trunc_factor,
// mg_Pmax_elements, mg_max_levels, mg_coarse_matrix_size, gpu_seed. Only
// PMIS coarsening (hypre type 8) and extended+i interpolation (type 6) without
// aggressive levels are implemented; the multigrid setup in solver.cu refuses
// any other mg_coarsening_type, mg_interpolation_type or mg_agg_num_levels
// with XAMG_ERR_UNSUPPORTED before calling build_hierarchy.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <random>

#include "amg.h"

namespace xg {

namespace {

struct Strength {
    std::vector<uint32_t> row, col;  // S: i strongly depends on col
};

Strength strength(const HCsr &A, double theta, double max_row_sum) {
    const uint64_t n = A.nrows;
    Strength S;
    S.row.assign(n + 1, 0);
    std::vector<uint32_t> cols;
    for (uint64_t i = 0; i < n; ++i) {
        double diag = 0.0, row_sum = 0.0;
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j) {
            if (A.col[j] == i) diag = A.val[j];
            row_sum += A.val[j];
        }
        const double sgn = diag < 0 ? -1.0 : 1.0;
        bool all_weak = false;
        if (max_row_sum < 1.0 && std::fabs(row_sum) > std::fabs(diag) * max_row_sum)
            all_weak = true;
        if (!all_weak) {
            double row_scale = 0.0;  // most "negative" (opposite to the diagonal) entry
            for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j)
                if (A.col[j] != i) row_scale = std::min(row_scale, sgn * A.val[j]);
            if (row_scale < 0.0)
                for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j)
                    if (A.col[j] != i && sgn * A.val[j] < theta * row_scale)
                        S.col.push_back(A.col[j]);
        }
        S.row[i + 1] = (uint32_t)S.col.size();
    }
    return S;
}

void transpose_pattern(const Strength &S, uint64_t n, std::vector<uint32_t> &trow,
                       std::vector<uint32_t> &tcol) {
    trow.assign(n + 1, 0);
    for (uint32_t c : S.col) ++trow[c + 1];
    for (uint64_t i = 0; i < n; ++i) trow[i + 1] += trow[i];
    tcol.resize(S.col.size());
    std::vector<uint32_t> pos(trow.begin(), trow.end() - 1);
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = S.row[i]; j < S.row[i + 1]; ++j) tcol[pos[S.col[j]]++] = (uint32_t)i;
}

enum : int8_t { UNDECIDED = 0, CPT = 1, FPT = -1 };

// PMIS: returns CF marker (1 = C, -1 = F)
std::vector<int8_t> pmis(const Strength &S, uint64_t n, uint64_t seed) {
    std::vector<uint32_t> trow, tcol;
    transpose_pattern(S, n, trow, tcol);
    std::mt19937_64 rng(seed * 0x9E3779B97F4A7C15ull + 12345);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::vector<double> measure(n);
    std::vector<int8_t> cf(n, UNDECIDED);
    for (uint64_t i = 0; i < n; ++i) {
        measure[i] = (double)(trow[i + 1] - trow[i]) + U(rng);
        if (measure[i] < 1.0) cf[i] = FPT;  // nobody depends on i
    }
    std::vector<uint32_t> undecided;
    for (uint64_t i = 0; i < n; ++i)
        if (cf[i] == UNDECIDED) undecided.push_back((uint32_t)i);
    std::vector<uint32_t> newc;
    while (!undecided.empty()) {
        newc.clear();
        for (uint32_t i : undecided) {
            bool is_max = true;
            for (uint32_t j = S.row[i]; j < S.row[i + 1] && is_max; ++j) {
                const uint32_t q = S.col[j];
                if (cf[q] == UNDECIDED && measure[q] >= measure[i] && q != i) is_max = false;
            }
            for (uint32_t j = trow[i]; j < trow[i + 1] && is_max; ++j) {
                const uint32_t q = tcol[j];
                if (cf[q] == UNDECIDED && measure[q] >= measure[i] && q != i) is_max = false;
            }
            if (is_max) newc.push_back(i);
        }
        if (newc.empty()) {  // ties of equal measures cannot occur with the random part;
            newc.push_back(undecided[0]);  // guard against a stall regardless
        }
        for (uint32_t c : newc) cf[c] = CPT;
        for (uint32_t c : newc)
            for (uint32_t j = trow[c]; j < trow[c + 1]; ++j) {
                const uint32_t q = tcol[j];  // q depends strongly on c
                if (cf[q] == UNDECIDED) cf[q] = FPT;
            }
        std::vector<uint32_t> next;
        next.reserve(undecided.size());
        for (uint32_t i : undecided)
            if (cf[i] == UNDECIDED) next.push_back(i);
        undecided.swap(next);
    }
    return cf;
}

// extended+i interpolation; returns P (n x nc)
HCsr ext_i_interp(const HCsr &A, const Strength &S, const std::vector<int8_t> &cf,
                  const std::vector<uint32_t> &cidx, uint64_t nc, double trunc, int pmax) {
    const uint64_t n = A.nrows;
    HCsr P;
    P.nrows = n;
    P.ncols = nc;
    P.row.assign(n + 1, 0);
    std::vector<int64_t> marker(n, -1);   // position in the current row's C_hat list
    std::vector<int8_t> strong(n, 0);     // strong flag for the current row's neighbours
    std::vector<uint32_t> chat;
    std::vector<double> w;
    std::vector<std::pair<double, uint32_t>> kept;
    for (uint64_t i = 0; i < n; ++i) {
        if (cf[i] == CPT) {
            P.col.push_back(cidx[i]);
            P.val.push_back(1.0);
            P.row[i + 1] = (uint32_t)P.col.size();
            continue;
        }
        chat.clear();
        for (uint32_t j = S.row[i]; j < S.row[i + 1]; ++j) strong[S.col[j]] = 1;
        // C_hat = strong C neighbours and the strong C neighbours of strong F neighbours
        for (uint32_t j = S.row[i]; j < S.row[i + 1]; ++j) {
            const uint32_t q = S.col[j];
            if (cf[q] == CPT) {
                if (marker[q] < 0) {
                    marker[q] = (int64_t)chat.size();
                    chat.push_back(q);
                }
            } else {
                for (uint32_t jj = S.row[q]; jj < S.row[q + 1]; ++jj) {
                    const uint32_t c = S.col[jj];
                    if (cf[c] == CPT && marker[c] < 0) {
                        marker[c] = (int64_t)chat.size();
                        chat.push_back(c);
                    }
                }
            }
        }
        w.assign(chat.size(), 0.0);
        double diag = 0.0;
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j)
            if (A.col[j] == i) diag += A.val[j];
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j) {
            const uint32_t q = A.col[j];
            if (q == i) continue;
            const double aiq = A.val[j];
            if (marker[q] >= 0) {
                w[marker[q]] += aiq;
            } else if (strong[q] && cf[q] == FPT) {
                // distribute over C_hat and i with the opposite-sign entries of row q
                double dq = 0.0;
                for (uint64_t jj = A.row[q]; jj < A.row[q + 1]; ++jj)
                    if (A.col[jj] == q) dq = A.val[jj];
                const double sgn = dq < 0 ? -1.0 : 1.0;
                double sum = 0.0;
                for (uint64_t jj = A.row[q]; jj < A.row[q + 1]; ++jj) {
                    const uint32_t l = A.col[jj];
                    const double v = A.val[jj];
                    if (sgn * v < 0 && (marker[l] >= 0 || l == i)) sum += v;
                }
                if (sum != 0.0) {
                    const double dist = aiq / sum;
                    for (uint64_t jj = A.row[q]; jj < A.row[q + 1]; ++jj) {
                        const uint32_t l = A.col[jj];
                        const double v = A.val[jj];
                        if (sgn * v < 0) {
                            if (marker[l] >= 0)
                                w[marker[l]] += dist * v;
                            else if (l == i)
                                diag += dist * v;
                        }
                    }
                } else {
                    diag += aiq;
                }
            } else {
                diag += aiq;  // weak connection lumped
            }
        }
        kept.clear();
        double maxw = 0.0, rowsum = 0.0;
        for (size_t c = 0; c < chat.size(); ++c) {
            const double v = (diag != 0.0) ? -w[c] / diag : 0.0;
            w[c] = v;
            maxw = std::max(maxw, std::fabs(v));
            rowsum += v;
        }
        for (size_t c = 0; c < chat.size(); ++c)
            if (w[c] != 0.0 && std::fabs(w[c]) >= trunc * maxw) kept.push_back({w[c], chat[c]});
        if (pmax > 0 && (int)kept.size() > pmax) {
            std::partial_sort(kept.begin(), kept.begin() + pmax, kept.end(),
                              [](const std::pair<double, uint32_t> &a,
                                 const std::pair<double, uint32_t> &b) {
                                  if (std::fabs(a.first) != std::fabs(b.first))
                                      return std::fabs(a.first) > std::fabs(b.first);
                                  return a.second < b.second;
                              });
            kept.resize(pmax);
        }
        double keptsum = 0.0;
        for (auto &e : kept) keptsum += e.first;
        const double scale = (keptsum != 0.0 && kept.size() < chat.size()) ? rowsum / keptsum : 1.0;
        std::sort(kept.begin(), kept.end(),
                  [&](const std::pair<double, uint32_t> &a, const std::pair<double, uint32_t> &b) {
                      return cidx[a.second] < cidx[b.second];
                  });
        for (auto &e : kept) {
            P.col.push_back(cidx[e.second]);
            P.val.push_back(e.first * scale);
        }
        P.row[i + 1] = (uint32_t)P.col.size();
        for (uint32_t c : chat) marker[c] = -1;
        for (uint32_t j = S.row[i]; j < S.row[i + 1]; ++j) strong[S.col[j]] = 0;
    }
    return P;
}

// C = A * B (sparse), columns sorted, the diagonal moved first when square
HCsr spgemm(const HCsr &A, const HCsr &B, bool diag_first) {
    HCsr C;
    C.nrows = A.nrows;
    C.ncols = B.ncols;
    C.row.assign(A.nrows + 1, 0);
    std::vector<int64_t> pos(B.ncols, -1);
    std::vector<uint32_t> cols;
    std::vector<double> acc;
    for (uint64_t i = 0; i < A.nrows; ++i) {
        cols.clear();
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j) {
            const uint32_t k = A.col[j];
            const double a = A.val[j];
            for (uint64_t jj = B.row[k]; jj < B.row[k + 1]; ++jj) {
                const uint32_t c = B.col[jj];
                if (pos[c] < 0) {
                    pos[c] = (int64_t)acc.size();
                    cols.push_back(c);
                    acc.push_back(a * B.val[jj]);
                } else {
                    acc[pos[c]] += a * B.val[jj];
                }
            }
        }
        std::vector<uint32_t> sorted = cols;
        std::sort(sorted.begin(), sorted.end());
        if (diag_first) {
            auto it = std::find(sorted.begin(), sorted.end(), (uint32_t)i);
            if (it != sorted.end()) std::rotate(sorted.begin(), it, it + 1);
        }
        for (uint32_t c : sorted) {
            C.col.push_back(c);
            C.val.push_back(acc[pos[c]]);
        }
        for (uint32_t c : cols) pos[c] = -1;
        acc.clear();
        C.row[i + 1] = (uint32_t)C.col.size();
    }
    return C;
}

HCsr transpose(const HCsr &P) {
    HCsr R;
    R.nrows = P.ncols;
    R.ncols = P.nrows;
    R.row.assign(P.ncols + 1, 0);
    for (uint32_t c : P.col) ++R.row[c + 1];
    for (uint64_t c = 0; c < P.ncols; ++c) R.row[c + 1] += R.row[c];
    R.col.resize(P.nnz());
    R.val.resize(P.nnz());
    std::vector<uint32_t> pos(R.row.begin(), R.row.end() - 1);
    for (uint64_t i = 0; i < P.nrows; ++i)
        for (uint64_t j = P.row[i]; j < P.row[i + 1]; ++j) {
            const uint32_t c = P.col[j];
            R.col[pos[c]] = (uint32_t)i;
            R.val[pos[c]] = P.val[j];
            ++pos[c];
        }
    return R;
}

// eigenvalues of a symmetric tridiagonal matrix by bisection (Sturm counts)
void tridiag_extremes(const std::vector<double> &d, const std::vector<double> &e, double &mn,
                      double &mx) {
    const int m = (int)d.size();
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < m; ++i) {
        double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(e[i]) : 0.0);
        lo = std::min(lo, d[i] - r);
        hi = std::max(hi, d[i] + r);
    }
    auto count_below = [&](double x) {  // number of eigenvalues < x
        int cnt = 0;
        double q = 1.0;
        for (int i = 0; i < m; ++i) {
            q = d[i] - x - (i > 0 ? e[i - 1] * e[i - 1] / q : 0.0);
            if (q == 0.0) q = -1e-300;
            if (q < 0) ++cnt;
        }
        return cnt;
    };
    auto kth = [&](int k) {
        double a = lo, b = hi;
        for (int it = 0; it < 200; ++it) {
            double c = 0.5 * (a + b);
            if (count_below(c) > k)
                b = c;
            else
                a = c;
        }
        return 0.5 * (a + b);
    };
    mn = kth(0);
    mx = kth(m - 1);
}

}  // namespace

void estimate_eigs(const HCsr &A, int iters, uint64_t seed, double &mn, double &mx) {
    const uint64_t n = A.nrows;
    std::vector<double> isd(n, 1.0);
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j)
            if (A.col[j] == i && A.val[j] > 0) isd[i] = 1.0 / std::sqrt(A.val[j]);
    auto apply = [&](const std::vector<double> &x, std::vector<double> &y) {
        for (uint64_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (uint64_t j = A.row[i]; j < A.row[i + 1]; ++j) s += A.val[j] * isd[A.col[j]] * x[A.col[j]];
            y[i] = isd[i] * s;
        }
    };
    std::mt19937_64 rng(seed + 7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> r(n), p(n), q(n), x(n, 0.0);
    for (auto &v : r) v = U(rng);
    p = r;
    double rr = std::inner_product(r.begin(), r.end(), r.begin(), 0.0);
    std::vector<double> alphas, betas;
    const int m = (int)std::min<uint64_t>(iters, n);
    for (int it = 0; it < m && rr > 0; ++it) {
        apply(p, q);
        const double pq = std::inner_product(p.begin(), p.end(), q.begin(), 0.0);
        if (pq <= 0) break;
        const double alpha = rr / pq;
        for (uint64_t i = 0; i < n; ++i) r[i] -= alpha * q[i];
        const double rr2 = std::inner_product(r.begin(), r.end(), r.begin(), 0.0);
        const double beta = rr2 / rr;
        alphas.push_back(alpha);
        betas.push_back(beta);
        for (uint64_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        rr = rr2;
    }
    const int k = (int)alphas.size();
    if (k == 0) {
        mn = mx = 1.0;
        return;
    }
    std::vector<double> d(k), e(k > 1 ? k - 1 : 0);
    for (int j = 0; j < k; ++j) {
        d[j] = 1.0 / alphas[j] + (j > 0 ? betas[j - 1] / alphas[j - 1] : 0.0);
        if (j + 1 < k) e[j] = std::sqrt(betas[j]) / alphas[j];
    }
    tridiag_extremes(d, e, mn, mx);
}

Hierarchy build_hierarchy(const HCsr &A0, const SolverCfg &mg) {
    Hierarchy H;
    H.lv.emplace_back();
    H.lv[0].A = A0;
    const double theta = mg.mg_strength_threshold;
    const double mrs = mg.mg_max_row_sum;
    const int max_levels = std::max(1, mg.mg_max_levels);
    const uint64_t coarse_size = (uint64_t)std::max(1, mg.mg_coarse_matrix_size);
    for (int l = 0;; ++l) {
        HCsr &A = H.lv[l].A;
        estimate_eigs(A, 10, (uint64_t)mg.gpu_seed * 131 + l, H.lv[l].min_eig, H.lv[l].max_eig);
        if (l + 1 >= max_levels || A.nrows <= coarse_size) break;
        Strength S = strength(A, theta, mrs);
        std::vector<int8_t> cf = pmis(S, A.nrows, (uint64_t)mg.gpu_seed * 7919 + l + 1);
        std::vector<uint32_t> cidx(A.nrows, 0);
        uint64_t nc = 0;
        for (uint64_t i = 0; i < A.nrows; ++i)
            if (cf[i] == CPT) cidx[i] = (uint32_t)nc++;
        if (nc == 0 || nc >= A.nrows) break;
        HCsr P = ext_i_interp(A, S, cf, cidx, nc, mg.mg_trunc_factor, mg.mg_Pmax_elements);
        HCsr AP = spgemm(A, P, false);
        HCsr R = transpose(P);
        HCsr Ac = spgemm(R, AP, true);
        H.lv[l].P = std::move(P);
        H.lv.emplace_back();
        H.lv[l + 1].A = std::move(Ac);
    }
    return H;
}

}  // namespace xg
