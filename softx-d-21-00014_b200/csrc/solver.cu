// Solver objects (see solver.h). Each solve() restates the reference
// solver's control flow; the comments name the reference lines.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>

#include "host_num.h"
#include "ops.h"
#include "solver.h"

namespace xg {

static cudaStream_t S() { return ctx().stream; }

void SolverBase::reset_stats() {
    // solver_stats::reset (solver.h:54-65)
    st.iters = 0;
    if ((int)st.conv.size() != NV) {
        st.conv.assign(NV, 0);
        st.abs_res.assign(NV, 0.0);
        st.rel_res.assign(NV, 0.0);
    }
    if (cfg.convergence_check) {
        std::fill(st.conv.begin(), st.conv.end(), 0);
        std::fill(st.abs_res.begin(), st.abs_res.end(), 0.0);
        std::fill(st.rel_res.begin(), st.rel_res.end(), 0.0);
    }
}

void SolverBase::alloc_buffers(int count) {
    buf.resize(count);
    for (auto &v : buf) v.alloc(n, NV, f32);
}

// Residual table (io/detail/print.inl:41-111)
static void print_header(int nv) {
    printf("%s |\n", std::string(10 + nv * 30, '-').c_str());
    printf("%7s | ", "Iter");
    for (int i = 0; i < nv; ++i) printf("%12s | %12s | ", "res", "res / res0");
    printf("\n");
}
static void print_row(int it, const double *res, const double *res0,
                      const std::vector<double> &conv) {
    printf("%7d | ", it);
    for (size_t k = 0; k < conv.size(); ++k) {
        if (conv[k] != 0)
            printf("%12e | %12e | ", std::sqrt(res[k]), std::sqrt(res[k] / res0[k]));
        else
            printf("%12s | %12s | ", "-", "-");
    }
    printf("\n");
}

// base_solver::convergence_check + converged + convergence_status
// (solver.h:173-241): tolerances are float32, compared against double norms.
static bool host_converged(SolverBase &sv, const double *res, const double *res0,
                           std::vector<double> &iconv) {
    if (!sv.cfg.convergence_check) return false;
    if (sv.cfg.convergence_info) {
        if (!sv.st.iters) print_header(sv.NV);
        print_row(sv.st.iters, res, res0, iconv);
    }
    const float abs_tol = sv.cfg.abs_tol, rel_tol = sv.cfg.rel_tol;
    bool flag = true;
    for (int k = 0; k < sv.NV; ++k) {
        if (iconv[k] != 0) {
            const double a = std::sqrt(res[k]);
            const double r = a / std::sqrt(res0[k]);
            if ((a > abs_tol) && (r > rel_tol)) {
                flag = false;
            } else if (!sv.st.conv[k]) {
                sv.st.abs_res[k] = a;
                sv.st.rel_res[k] = r;
                sv.st.conv[k] = 1;
            }
        }
    }
    if (flag) {
        if (sv.cfg.convergence_info) printf("%s |\n", std::string(10 + sv.NV * 30, '-').c_str());
        return true;
    }
    for (int k = 0; k < sv.NV; ++k) iconv[k] *= (double)(!sv.st.conv[k]);
    return false;
}

// Reads nv doubles of device scalars into host memory (synchronises).
static void read_scalars(const double *dev, double *host, int nv) {
    Ctx &c = ctx();
    XG_CUDA(cudaMemcpyAsync(c.pinned, dev, nv * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    XG_CUDA(cudaStreamSynchronize(c.stream));
    std::memcpy(host, c.pinned, nv * sizeof(double));
}

// Posts nv device scalars to the current lane's pinned slots; take_scalars
// reads them once the lane's stream has been synchronised.
static void post_scalars(const double *dev, int nv) {
    Ctx &c = ctx();
    XG_CUDA(cudaMemcpyAsync(c.pinned, dev, nv * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
}
static void take_scalars(double *host, int nv) { std::memcpy(host, ctx().pinned, nv * sizeof(double)); }

// get_residual (solver.h:243-256) with the norm into res (host)
template <typename F>
static void residual_norm(const DCsr &A, DVec &x, DVec &b, DVec &r, int nv, double *res_host) {
    double *dn = ctx().red_out.as<double>();
    if (x.zero) {
        // Ax_y leaves r zero-flagged; axpby(1, b, -1, r) takes its ax_y branch: r = 1*b
        ops::convert<F, F>(r.p<F>(), b.p<F>(), r.elems(), S());
        ops::dot<F>(r.n, r.p<F>(), r.p<F>(), dn, nv, S());
    } else {
        ops::residual<F>(A, x.p<F>(), b.p<F>(), r.p<F>(), nv, dn, S());
    }
    r.zero = false;
    r.init = true;
    read_scalars(dn, res_host, nv);
}

// ===========================================================================
// Jacobi (jacobi.inl:49-120)
// ===========================================================================
template <typename F>
struct Jacobi : public SolverBase {
    DevBuf d;  // inverse diagonal, level precision
    DevBuf relax_dev;
    void setup_from(const HCsr &hA) {
        if (f32)
            upload(d, inv_diag_f32(hA, false), S());
        else
            upload(d, inv_diag_f64(hA, false), S());
        alloc_buffers(2);
        relax_dev.alloc(32 * sizeof(double));
        XG_CUDA(cudaStreamSynchronize(S()));
    }
    void solve(DVec &x, DVec &b, const std::vector<double> &conv) override {
        reset_stats();
        const F relax = (F)cfg.relax;
        const int m = std::max(1, cfg.max_iters);
        if (cfg.convergence_check) {
            solve_checked(x, b, conv);
            return;
        }
        // x_out alternates between x and buf[1]; sweep j lands in x when
        // (m - j) is even so that the last one does.
        DVec &T = buf[1];
        auto tgt = [&](int j) -> DVec & { return ((m - j) % 2 == 0) ? x : T; };
        DVec *cur = &x;
        int j = 1;
        if (x.zero) {
            DVec &o = tgt(1);
            ops::jacobi_zero<F>(n, o.p<F>(), b.p<F>(), d.as<F>(), relax, NV, S());
            cur = &o;
            j = 2;
        } else if ((m - 1) % 2 == 0) {
            ops::convert<F, F>(T.p<F>(), x.p<F>(), x.elems(), S());
            cur = &T;
        }
        for (; j <= m; ++j) {
            DVec &o = tgt(j);
            ops::jacobi_sweep<F>(*A, cur->p<F>(), o.p<F>(), b.p<F>(), d.as<F>(), relax, NV, S());
            cur = &o;
        }
        st.iters = m;
        x.zero = false;
        x.init = true;
    }
    // jacobi.inl:93-112
    void solve_checked(DVec &x, DVec &b, const std::vector<double> &conv) {
        std::vector<double> iconv = conv, rho0(NV), res(NV), relax_h(NV, (double)(F)cfg.relax);
        DVec &r = buf[0];
        residual_norm<F>(*A, x, b, r, NV, rho0.data());
        if (host_converged(*this, rho0.data(), rho0.data(), iconv)) return;
        do {
            ++st.iters;
            ops::scale_rows<F>(r.p<F>(), d.as<F>(), n, NV, S());
            for (int k = 0; k < NV; ++k) relax_h[k] = (double)(F)(relax_h[k] * iconv[k]);
            XG_CUDA(cudaMemcpyAsync(relax_dev.p, relax_h.data(), NV * sizeof(double),
                                    cudaMemcpyHostToDevice, S()));
            ops::axpy_k<F>(x.p<F>(), r.p<F>(), relax_dev.as<double>(), n, NV, x.zero, S());
            x.zero = false;
            residual_norm<F>(*A, x, b, r, NV, res.data());
            if (host_converged(*this, res.data(), rho0.data(), iconv)) return;
        } while (st.iters < cfg.max_iters);
    }
};

// ===========================================================================
// Hybrid symmetric Gauss-Seidel (hsgs.inl:50-115, blas2.h:184-281,
// csr_gs.inl:32-134). GS blocks play the role of XAMG's cores: rows are split
// with XAMG's core rule into nb = max(1, n / gpu_hsgs_rows) blocks; entries
// coupling a block to another one are lagged (use x from before the sweep).
// ===========================================================================
template <typename F>
struct Hsgs : public SolverBase {
    DevBuf d, boff, relax_dev;
    std::vector<double> relax_on_dev;  // what relax_dev holds (host mirror)
    DCsr Adiag, Aoff;
    int nblocks = 1;
    void setup_from(const HCsr &hA) {
        const uint64_t rows = cfg.gpu_hsgs_rows > 0 ? (uint64_t)cfg.gpu_hsgs_rows : 32;
        nblocks = (int)std::max<uint64_t>(1, n / rows);
        const uint64_t cs = split_range_f64(n, nblocks);
        std::vector<uint64_t> off(nblocks + 1);
        for (int c = 0; c <= nblocks; ++c) off[c] = std::min<uint64_t>(n, cs * (uint64_t)c);
        off[nblocks] = n;
        // block id of every row
        std::vector<uint32_t> bid(n);
        for (int c = 0; c < nblocks; ++c)
            for (uint64_t i = off[c]; i < off[c + 1]; ++i) bid[i] = c;
        HCsr dg, od;
        dg.nrows = od.nrows = n;
        od.ncols = n;
        uint64_t maxb = 1;
        for (int c = 0; c < nblocks; ++c) maxb = std::max<uint64_t>(maxb, off[c + 1] - off[c]);
        dg.ncols = maxb;
        dg.row.assign(n + 1, 0);
        od.row.assign(n + 1, 0);
        std::vector<std::pair<uint32_t, uint64_t>> tmp;
        for (uint64_t i = 0; i < n; ++i) {
            const uint32_t c = bid[i];
            tmp.clear();
            for (uint64_t j = hA.row[i]; j < hA.row[i + 1]; ++j) {
                const uint32_t col = hA.col[j];
                if (bid[col] == c) {
                    dg.col.push_back((uint32_t)(col - off[c]));
                    dg.val.push_back(hA.val[j]);
                } else {
                    tmp.push_back({bid[col], j});
                }
            }
            // off-core chunks are visited in block order, entries in row order
            std::stable_sort(tmp.begin(), tmp.end(),
                             [](const std::pair<uint32_t, uint64_t> &a,
                                const std::pair<uint32_t, uint64_t> &b) { return a.first < b.first; });
            for (auto &t : tmp) {
                od.col.push_back(hA.col[t.second]);
                od.val.push_back(hA.val[t.second]);
            }
            dg.row[i + 1] = (uint32_t)dg.col.size();
            od.row[i + 1] = (uint32_t)od.col.size();
        }
        upload_csr(dg, Adiag, f32, cfg.gpu_index_compress, S());
        upload_csr(od, Aoff, f32, cfg.gpu_index_compress, S(), cfg.gpu_spmv_tune);
        upload(boff, off, S());
        if (f32)
            upload(d, inv_diag_f32(hA, false), S());
        else
            upload(d, inv_diag_f64(hA, false), S());
        relax_dev.alloc(32 * sizeof(double));
        relax_on_dev.assign(32, (double)(F)cfg.relax);
        XG_CUDA(cudaMemcpyAsync(relax_dev.p, relax_on_dev.data(), 32 * sizeof(double),
                                cudaMemcpyHostToDevice, S()));
        alloc_buffers(2);
        XG_CUDA(cudaStreamSynchronize(S()));
    }
    void solve(DVec &x, DVec &b, const std::vector<double> &conv) override {
        reset_stats();
        std::vector<double> iconv = conv, rho0(NV), res(NV);
        std::vector<double> relax_h(NV, (double)(F)cfg.relax);
        bool ones = true;
        for (int k = 0; k < NV; ++k) ones = ones && (iconv[k] == 1.0);
        DVec &r = buf[0];
        DVec &t = buf[1];
        if (cfg.convergence_check) {
            residual_norm<F>(*A, x, b, r, NV, rho0.data());
            if (host_converged(*this, rho0.data(), rho0.data(), iconv)) return;
        }
        do {
            ++st.iters;
            // scal(iconv, relax_conv) (hsgs.inl:102); the device copy is
            // refreshed whenever it differs, so a solve that starts with every
            // right-hand side active does not inherit the factors an earlier
            // solve froze
            if (!ones || cfg.convergence_check)
                for (int k = 0; k < NV; ++k) relax_h[k] = (double)(F)(relax_h[k] * iconv[k]);
            if (!std::equal(relax_h.begin(), relax_h.end(), relax_on_dev.begin())) {
                std::copy(relax_h.begin(), relax_h.end(), relax_on_dev.begin());
                XG_CUDA(cudaMemcpyAsync(relax_dev.p, relax_on_dev.data(), NV * sizeof(double),
                                        cudaMemcpyHostToDevice, S()));
            }
            if (x.zero) {
                // no lagged term: t = 1*b + (-1)*0 = b; x = 0 (blas2.h:226-262)
                ops::convert<F, F>(t.p<F>(), b.p<F>(), t.elems(), S());
                ops::fill<F>(x.p<F>(), x.elems(), F(0), S());
            } else {
                ops::residual<F>(Aoff, x.p<F>(), b.p<F>(), t.p<F>(), NV, nullptr, S());
            }
            ops::hsgs_sweep<F>(Adiag, boff.as<uint64_t>(), nblocks, t.p<F>(), x.p<F>(), d.as<F>(),
                               relax_dev.as<double>(), NV, S());
            x.zero = false;
            x.init = true;
            if (cfg.convergence_check) {
                residual_norm<F>(*A, x, b, r, NV, res.data());
                if (host_converged(*this, res.data(), rho0.data(), iconv)) return;
            }
        } while (st.iters < cfg.max_iters);
    }
};

// ===========================================================================
// Chebyshev (chebyshev.inl:129-206)
// ===========================================================================
template <typename F>
struct Chebyshev : public SolverBase {
    DevBuf isd;
    double min_eig = 0, max_eig = 0;
    std::vector<F> coef;
    void setup_from(const HCsr &hA) {
        if (f32)
            upload(isd, inv_diag_f32(hA, true), S());
        else
            upload(isd, inv_diag_f64(hA, true), S());
        alloc_buffers(3);
        XG_CUDA(cudaStreamSynchronize(S()));
    }
    void solve(DVec &x, DVec &b, const std::vector<double> &conv) override {
        reset_stats();
        const int order = cfg.poly_order;
        XG_REQUIRE(order >= 1 && order <= 4, XAMG_ERR_INVALID_ARG,
                   "Chebyshev polynomial_order must be 1..4");
        std::vector<double> cd = cheby_coeffs(min_eig, max_eig, order, (double)cfg.spec_fraction);
        coef.resize(order);
        for (int i = 0; i < order; ++i) coef[i] = (F)cd[i];
        std::vector<double> rho0(NV), res(NV);
        const bool x_zero = x.zero;
        if (cfg.convergence_check && cfg.convergence_info) {
            residual_norm<F>(*A, x, b, buf[0], NV, rho0.data());
            print_header(NV);
            print_row(0, rho0.data(), rho0.data(), conv);
        }
        DVec &rs = buf[0];
        DVec *t1s = &buf[1], *other = &buf[2];
        ops::cheby_first<F>(*A, x.p<F>(), x_zero, b.p<F>(), isd.as<F>(), coef[order - 1],
                            rs.p<F>(), t1s->p<F>(), NV, S());
        if (order == 1) {
            ops::add_into<F>(x.p<F>(), t1s->p<F>(), x.elems(), x_zero, S());
        } else {
            for (int i = order - 2; i >= 0; --i) {
                const bool last = (i == 0);
                DVec &out = last ? x : *other;
                ops::cheby_step<F>(*A, t1s->p<F>(), rs.p<F>(), isd.as<F>(), coef[i], out.p<F>(),
                                   last, x_zero, NV, S());
                if (!last) std::swap(t1s, other);
            }
        }
        x.zero = false;
        x.init = true;
        if (cfg.convergence_check && cfg.convergence_info) {
            residual_norm<F>(*A, x, b, buf[0], NV, res.data());
            print_row(0, res.data(), rho0.data(), conv);
        }
    }
};

// ===========================================================================
// Direct coarse solve (direct.inl:31-56): dense Gauss-Jordan inverse built on
// the host at setup, applied as a dense multi-RHS product.
// ===========================================================================
template <typename F>
struct Direct : public SolverBase {
    DevBuf inv;
    // The explicit inverse is dense (n^2 values, inverse.inl:31-106): refuse
    // sizes whose inverse would not fit host and device memory comfortably
    // instead of running out of memory (the hierarchy's coarsest level is
    // this large when mg_max_levels stops the coarsening early).
    static constexpr uint64_t MAX_N = 16384;
    void setup_from(const HCsr &hA) {
        XG_REQUIRE(hA.nrows <= MAX_N, XAMG_ERR_UNSUPPORTED,
                   "direct solver on " + std::to_string(hA.nrows) +
                       " rows (at most 16384): coarsen further (mg_max_levels, "
                       "mg_coarse_matrix_size)");
        // stored column by column for k_dense's coalesced reads
        if (f32)
            upload(inv, transposed(dense_inverse_f32(hA), hA.nrows), S());
        else
            upload(inv, transposed(dense_inverse_f64(hA), hA.nrows), S());
        XG_CUDA(cudaStreamSynchronize(S()));
    }
    template <typename T>
    static std::vector<T> transposed(const std::vector<T> &a, uint64_t n) {
        std::vector<T> t(a.size());
        for (uint64_t i = 0; i < n; ++i)
            for (uint64_t j = 0; j < n; ++j) t[j * n + i] = a[i * n + j];
        return t;
    }
    void solve(DVec &x, DVec &b, const std::vector<double> &) override {
        // blas2::Ax_y short-circuit on a zero-flagged input (blas2.h:309-313)
        if (b.zero) {
            x.zero = true;
            return;
        }
        ops::dense_apply<F>(inv.as<F>(), n, b.p<F>(), x.p<F>(), NV, S());
        x.zero = false;
        x.init = true;
    }
};

// Identity (solver.h:340-368): x = b
template <typename F>
struct Identity : public SolverBase {
    void solve(DVec &x, DVec &b, const std::vector<double> &) override {
        if (b.zero) {
            x.zero = true;
            x.init = true;
            return;
        }
        ops::convert<F, F>(x.p<F>(), b.p<F>(), x.elems(), S());
        x.zero = false;
        x.init = true;
    }
};

template <typename F>
static std::unique_ptr<SolverBase> make_smoother_t(const SolverCfg &cfg, const std::string &role,
                                                   const DCsr &A, const HCsr &hA, int nv,
                                                   double min_eig, double max_eig) {
    std::unique_ptr<SolverBase> s;
    const std::string &m = cfg.method;
    auto init = [&](SolverBase *b) {
        b->cfg = cfg;
        b->role = role;
        b->NV = nv;
        b->f32 = std::is_same<F, float>::value;
        b->A = &A;
        b->n = A.nrows;
    };
    if (m == "Jacobi") {
        auto *j = new Jacobi<F>();
        init(j);
        j->setup_from(hA);
        s.reset(j);
    } else if (m == "HSGS") {
        auto *h = new Hsgs<F>();
        init(h);
        h->setup_from(hA);
        s.reset(h);
    } else if (m == "Chebyshev") {
        auto *c = new Chebyshev<F>();
        init(c);
        c->min_eig = min_eig;
        c->max_eig = max_eig;
        c->setup_from(hA);
        s.reset(c);
    } else if (m == "Direct") {
        auto *d = new Direct<F>();
        init(d);
        d->setup_from(hA);
        s.reset(d);
    } else if (m == "Identity") {
        auto *d = new Identity<F>();
        init(d);
        s.reset(d);
    } else {
        throw Error(XAMG_ERR_UNSUPPORTED, "method '" + m + "' cannot be used as " + role);
    }
    return s;
}

std::unique_ptr<SolverBase> make_smoother(const SolverCfg &cfg, const std::string &role,
                                          const DCsr &A, const HCsr &hA, bool f32, int nv,
                                          double min_eig, double max_eig) {
    if (f32) return make_smoother_t<float>(cfg, role, A, hA, nv, min_eig, max_eig);
    return make_smoother_t<double>(cfg, role, A, hA, nv, min_eig, max_eig);
}

// ===========================================================================
// MultiGrid (mg.inl:97-334)
// ===========================================================================
std::string hierarchy_key(const SolverCfg &c) {
    char buf[256];
    snprintf(buf, sizeof(buf), "th=%.9g mrs=%.9g tf=%.9g pmax=%d ml=%d cs=%d ct=%d it=%d seed=%d",
             (double)c.mg_strength_threshold, (double)c.mg_max_row_sum, (double)c.mg_trunc_factor,
             c.mg_Pmax_elements, c.mg_max_levels, c.mg_coarse_matrix_size, c.mg_coarsening_type,
             c.mg_interpolation_type, c.gpu_seed);
    return buf;
}

void MultiGrid::build(const HCsr &A0, const DCsr *A0dev, const Params &P, const std::string &rl,
                      int nv, HierCache *cache) {
    role = rl;
    NV = nv;
    cfg = resolve_cfg(P.get(role), role);
    A = A0dev;
    n = A0.nrows;
    f32 = false;
    const std::string key = hierarchy_key(cfg);
    if (cache && cache->count(key)) {
        H = (*cache)[key];
    } else {
        // The host setup implements PMIS coarsening (hypre type 8) with
        // extended+i interpolation (type 6) and no aggressive levels; hypre
        // offers more (hypre_base.h:155-163). Other choices, on any level the
        // hierarchy can reach, are refused rather than replaced.
        for (int l = 0; l < std::max(1, cfg.mg_max_levels); ++l) {
            const SolverCfg c = resolve_cfg(P.get(role, l), role);
            XG_REQUIRE(c.mg_coarsening_type == 8, XAMG_ERR_UNSUPPORTED,
                       "mg_coarsening_type " + std::to_string(c.mg_coarsening_type) +
                           " (level " + std::to_string(l) +
                           "): only PMIS (8) is implemented by the host setup");
            XG_REQUIRE(c.mg_interpolation_type == 6, XAMG_ERR_UNSUPPORTED,
                       "mg_interpolation_type " + std::to_string(c.mg_interpolation_type) +
                           " (level " + std::to_string(l) +
                           "): only extended+i (6) is implemented by the host setup");
            XG_REQUIRE(c.mg_agg_num_levels == 0, XAMG_ERR_UNSUPPORTED,
                       "mg_agg_num_levels " + std::to_string(c.mg_agg_num_levels) +
                           ": aggressive coarsening is not implemented by the host setup");
        }
        H = std::make_shared<const Hierarchy>(build_hierarchy(A0, cfg));
        if (cache) (*cache)[key] = H;
    }
    const Hierarchy &HH = *H;
    const int nl = (int)HH.lv.size();
    XG_REQUIRE(nl >= 2, XAMG_ERR_UNSUPPORTED, "multigrid hierarchy has fewer than 2 levels");
    const bool reduced = cfg.gpu_precond_f32 >= 0 ? cfg.gpu_precond_f32 != 0
                                                  : cfg.mg_reduced_precision != 0;
    full32 = (cfg.gpu_precond_f32 == 1) && role == "preconditioner";
    const int narrow = cfg.gpu_index_compress;
    const int tune = cfg.gpu_spmv_tune;
    L.clear();
    L.resize(nl);
    for (int l = 0; l < nl; ++l) {
        MgLevel &lv = L[l];
        lv.f32 = (l >= 1 || full32) && reduced;
        lv.tf32 = reduced;
        lv.min_eig = HH.lv[l].min_eig;
        lv.max_eig = HH.lv[l].max_eig;
        // gpu_level_bf16: the l < gpu_level_bf16 finest FP32 cycle operators store
        // BF16 values, or with gpu_level_fp16 = 1 FP16 values with a per-level
        // power-of-two scale (the smoothers' diagonals stay float from the
        // exact values)
        if (l >= 1 || full32) {
            const bool half = lv.f32 && l < cfg.gpu_level_bf16;
            upload_csr(HH.lv[l].A, lv.A, lv.f32, narrow, S(), tune,
                       half && cfg.gpu_level_fp16 == 0, nv, half && cfg.gpu_level_fp16 == 1);
        }
        if (l + 1 < nl) {
            // R = P^T (hypre_base.inl:400-401, transpose.inl:31-108)
            const HCsr &Ph = HH.lv[l].P;
            HCsr R;
            R.nrows = Ph.ncols;
            R.ncols = Ph.nrows;
            std::vector<uint32_t> cnt(Ph.ncols + 1, 0);
            for (uint32_t c : Ph.col) ++cnt[c + 1];
            R.row.assign(Ph.ncols + 1, 0);
            for (uint64_t c = 0; c < Ph.ncols; ++c) R.row[c + 1] = R.row[c] + cnt[c + 1];
            R.col.resize(Ph.nnz());
            R.val.resize(Ph.nnz());
            std::vector<uint32_t> pos(R.row.begin(), R.row.end() - 1);
            for (uint64_t i = 0; i < Ph.nrows; ++i)
                for (uint64_t j = Ph.row[i]; j < Ph.row[i + 1]; ++j) {
                    const uint32_t c = Ph.col[j];
                    R.col[pos[c]] = (uint32_t)i;
                    R.val[pos[c]] = Ph.val[j];
                    ++pos[c];
                }
            upload_csr(Ph, lv.P, lv.tf32, narrow, S(), tune, false, nv);
            upload_csr(R, lv.R, lv.tf32, narrow, S(), tune, false, nv);
        }
        const uint64_t nrow = HH.lv[l].A.nrows;
        if (l == 0) {
            lv.temp.alloc(nrow, nv, lv.f32);
            if (full32) {
                b32.alloc(nrow, nv, true);
                x32.alloc(nrow, nv, true);
            }
        } else {
            lv.temp.alloc(nrow, nv, lv.f32);
            lv.bH.alloc(nrow, nv, lv.f32);
            lv.xH.alloc(nrow, nv, lv.f32);
        }
    }
    pre.clear();
    post.clear();
    for (int l = 0; l + 1 < nl; ++l) {
        const DCsr &Al = (l == 0 && !full32) ? *A0dev : L[l].A;
        SolverCfg pc = resolve_cfg(P.get("pre_smoother", l), "pre_smoother");
        SolverCfg qc = resolve_cfg(P.get("post_smoother", l), "post_smoother");
        pc.gpu_index_compress = qc.gpu_index_compress = cfg.gpu_index_compress;
        pc.gpu_spmv_tune = qc.gpu_spmv_tune = cfg.gpu_spmv_tune;
        pre.push_back(make_smoother(pc, "pre_smoother", Al, HH.lv[l].A, L[l].f32, nv,
                                    L[l].min_eig, L[l].max_eig));
        post.push_back(make_smoother(qc, "post_smoother", Al, HH.lv[l].A, L[l].f32, nv,
                                     L[l].min_eig, L[l].max_eig));
    }
    SolverCfg cc = resolve_cfg(P.get("coarse_grid_solver"), "coarse_grid_solver");
    coarse = make_smoother(cc, "coarse_grid_solver", L[nl - 1].A, HH.lv[nl - 1].A, L[nl - 1].f32,
                           nv, L[nl - 1].min_eig, L[nl - 1].max_eig);
    buf.resize(1);
    buf[0].alloc(n, nv, false);
    XG_CUDA(cudaStreamSynchronize(S()));
}

// mg.inl:166-260
void MultiGrid::cycle(int level, DVec &x, DVec &b, int cyc, const std::vector<double> &iconv) {
    MgLevel &lv = L[level];
    const DCsr &Al = (level == 0 && !full32) ? *A : lv.A;
    const int nl = (int)L.size();
    MgLevel &nx = L[level + 1];
    DVec &temp = lv.temp, &bH = nx.bH, &xH = nx.xH;
    const bool mixed = (lv.f32 != nx.f32);  // level 0 -> 1 with reduced precision
    if (cyc != 1) pre[level]->solve(x, b, iconv);
    // residual temp = b - A x (Ax_y + axpby(a1, b, a_1, temp))
    const DVec *rin = &temp;
    if (x.zero) {
        rin = &b;  // temp = 1*b, bitwise b
    } else if (lv.f32) {
        ops::residual<float>(Al, x.p<float>(), b.p<float>(), temp.p<float>(), NV, nullptr, S());
    } else {
        ops::residual<double>(Al, x.p<double>(), b.p<double>(), temp.p<double>(), NV, nullptr,
                              S());
    }
    // restriction (with the float conversion fused when the precision changes)
    if (b.zero && x.zero) {
        bH.zero = true;
    } else if (mixed) {
        ops::spmv_f32_from_f64(lv.R, rin->p<double>(), bH.p<float>(), NV, S());
        bH.zero = false;
    } else if (nx.f32) {
        ops::spmv<float>(lv.R, rin->p<float>(), bH.p<float>(), NV, false, S());
        bH.zero = false;
    } else {
        ops::spmv<double>(lv.R, rin->p<double>(), bH.p<double>(), NV, false, S());
        bH.zero = false;
    }
    bH.init = true;
    xH.zero = true;  // set_const(x_H, 0)
    xH.init = true;
    if (level + 1 == nl - 1) {
        coarse->solve(xH, bH, iconv);
    } else {
        cycle(level + 1, xH, bH, cyc, iconv);
        if (cyc == 2)
            cycle(level + 1, xH, bH, 2, iconv);
        else if (cyc == 1)
            cycle(level + 1, xH, bH, 0, iconv);
    }
    // prolongation
    if (!xH.zero) {
        if (mixed) {
            ops::prolong_mixed(lv.P, xH.p<float>(), x.p<double>(), x.zero, NV, S());
        } else {
            // Axpy(P, x_H, x) accumulates into x's memory whatever its zero
            // flag says (blas2.h:284-326, csr_matvec.inl:33-144): after the
            // F-cycle's first visit of a level (no pre-smoothing,
            // mg.inl:198) x still holds what the previous cycle left in it,
            // and the reference adds to that
            if (lv.f32)
                ops::spmv<float>(lv.P, xH.p<float>(), x.p<float>(), NV, true, S());
            else
                ops::spmv<double>(lv.P, xH.p<double>(), x.p<double>(), NV, true, S());
        }
        x.zero = false;
        x.init = true;
    }
    post[level]->solve(x, b, iconv);
}

// The gpu_precond_f32 = 1 preconditioner with its result left in float in
// x32 (a caller's buffer): the same cycles as solve(); a caller that reads
// x32 widened exactly sees the values solve() would write into x.
void MultiGrid::solve_to32(DVec &x32o, DVec &b, const std::vector<double> &conv) {
    reset_stats();
    std::vector<double> iconv = conv;
    b32.zero = b.zero;
    if (!b.zero) ops::convert<float, double>(b32.p<float>(), b.p<double>(), b.elems(), S());
    b32.init = true;
    x32o.init = true;
    do {
        ++st.iters;
        cycle(0, x32o, b32, cfg.mg_cycle, iconv);
    } while (st.iters < cfg.max_iters);
}

// mg.inl:262-334
void MultiGrid::solve(DVec &x, DVec &b, const std::vector<double> &conv) {
    reset_stats();
    std::vector<double> iconv = conv, rho0(NV), res(NV);
    DVec &r = buf[0];
    if (full32) {
        // preconditioner in float throughout: convert the input, cycle, convert
        // the result back (zero flags carried across)
        b32.zero = b.zero;
        if (!b.zero) ops::convert<float, double>(b32.p<float>(), b.p<double>(), b.elems(), S());
        x32.zero = x.zero;
        if (!x.zero) ops::convert<float, double>(x32.p<float>(), x.p<double>(), x.elems(), S());
        b32.init = x32.init = true;
        do {
            ++st.iters;
            cycle(0, x32, b32, cfg.mg_cycle, iconv);
        } while (st.iters < cfg.max_iters);
        x.zero = x32.zero;
        if (!x32.zero) ops::convert<double, float>(x.p<double>(), x32.p<float>(), x.elems(), S());
        x.init = true;
        return;
    }
    if (cfg.convergence_check) {
        residual_norm<double>(*A, x, b, r, NV, rho0.data());
        if (host_converged(*this, rho0.data(), rho0.data(), iconv)) return;
    }
    do {
        ++st.iters;
        cycle(0, x, b, cfg.mg_cycle, iconv);
        if (cfg.convergence_check) {
            residual_norm<double>(*A, x, b, r, NV, res.data());
            if (host_converged(*this, res.data(), rho0.data(), iconv)) return;
        }
    } while (st.iters < cfg.max_iters);
}

// ===========================================================================
// BiCGStab family (merged_pbicgstab.inl:44-225, merged_bicgstab.inl:44-208,
// pbicgstab.inl, bicgstab.inl)
// ===========================================================================
void Krylov::setup() {
    alloc_buffers(8);
    sc.alloc(k::SC_COUNT * k::SC_STRIDE * sizeof(double));
    XG_CUDA(cudaMemset(sc.p, 0, sc.bytes));
}

void Krylov::upload_iconv(const std::vector<double> &iconv) {
    std::vector<double> h(iconv);
    XG_CUDA(cudaMemcpyAsync(sc.as<double>() + k::SC_ICONV * k::SC_STRIDE, h.data(),
                            NV * sizeof(double), cudaMemcpyHostToDevice, S()));
}

bool Krylov::check(const double *res, const double *res0, std::vector<double> &iconv) {
    const std::vector<double> before = iconv;
    const bool done = host_converged(*this, res, res0, iconv);
    if (!done && iconv != before) upload_iconv(iconv);
    return done;
}

void Krylov::run_M(DVec &out, DVec &in) {
    static const std::vector<double> ones(32, 1.0);
    std::vector<double> o(ones.begin(), ones.begin() + NV);
    if (f32io && out.f32)
        static_cast<MultiGrid *>(M.get())->solve_to32(out, in, o);
    else
        M->solve(out, in, o);
}

// An FP32 multigrid preconditioner (gpu_precond_f32 = 1) whose cycle never
// reads its output's old contents (V- and W-cycles; the F-cycle adds to
// them) leaves its results in float: the Krylov kernels then read pa32/sa32
// widened to double, exactly the values converting them back to FP64 would
// write, without that conversion and with half the bytes in the SpMV's x
// gathers. The merged BiCGStab forms only (PCG and RBiCGStab keep FP64).
void Krylov::enable_f32io() {
    auto *g = dynamic_cast<MultiGrid *>(M.get());
    if (!g || !g->full32 || pcg || rbicgstab || !precond_form) return;
    f32io_ready = true;
    pa32.alloc(n, NV, true);
    sa32.alloc(n, NV, true);
}

Krylov::~Krylov() { drop_graphs(); }

// set_const(out, 0) then precond->solve(out, in) with conv = ones. With
// gpu_graph (default) the application is recorded once per (out, in,
// in.zero) as a CUDA graph, on its second call (the first one settles every
// buffer and flag of the preconditioner), and replayed from then on: the
// same kernels on the same buffers in one launch. A preconditioner whose
// application cannot be captured runs directly.
void Krylov::apply_M(DVec &out, DVec &in) {
    out.zero = true;
    out.init = true;
    if (!cfg.gpu_graph || capturing_) {
        run_M(out, in);
        return;
    }
    MGraph &g =
        graphs_[std::make_tuple(out.p<const void>(), in.p<const void>(), in.zero, ctx().lane)];
    if (g.exec) {
        XG_CUDA(cudaGraphLaunch(g.exec, S()));
        g_kernel_launches += g.launches;
        out.zero = g.out_zero;
        return;
    }
    if (g.failed || g.calls++ < 1) {
        run_M(out, in);
        return;
    }
    const bool in_zero = in.zero, in_init = in.init;
    XG_CUDA(cudaStreamSynchronize(S()));
    XG_CUDA(cudaStreamBeginCapture(S(), cudaStreamCaptureModeThreadLocal));
    const uint64_t l0 = g_kernel_launches;
    cudaGraph_t graph = nullptr;
    bool ok = true;
    try {
        run_M(out, in);  // recorded, not run
    } catch (...) {
        ok = false;  // e.g. a preconditioner that reads back a residual
    }
    const cudaError_t e = cudaStreamEndCapture(S(), &graph);
    if (!ok || e != cudaSuccess || !graph ||
        cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
        // nothing ran during the capture: run directly from now on, from the
        // flags the recording started with (it zero-flagged out, and may have
        // cleared that flag as if its kernels had run)
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
        g.exec = nullptr;
        g.failed = true;
        g_kernel_launches = l0;
        out.zero = true;
        out.init = true;
        in.zero = in_zero;
        in.init = in_init;
        run_M(out, in);
        return;
    }
    cudaGraphDestroy(graph);
    g.launches = g_kernel_launches - l0;
    g.out_zero = out.zero;
    XG_CUDA(cudaGraphLaunch(g.exec, S()));
}

// pcg.inl:44-162: fused as Ap = A p with (p, Ap) and alpha; the x and r
// updates; z = M^-1 r; (r, z), (r, r) and beta; p = z + beta p. The first
// (r, z) comes from the same dot kernel after z0 = M^-1 r0.
void Krylov::solve_pcg(DVec &x, DVec &b, const std::vector<double> &conv) {
    cudaStream_t s = S();
    std::vector<double> iconv = conv;
    upload_iconv(iconv);
    double *SC = sc.as<double>();
    for (auto &v : buf) {
        v.zero = true;
        v.init = true;
    }
    DVec &r = buf[0], &z = buf[1], &p = buf[2], &Ap = buf[3];
    std::vector<double> rho0(NV), res(NV);
    residual_norm<double>(*A, x, b, r, NV, rho0.data());
    if (check(rho0.data(), rho0.data(), iconv)) return;
    apply_M(z, r);
    // copy(z, p), zero flag included (blas.inl:224-246)
    p.zero = z.zero;
    if (!z.zero) ops::convert<double, double>(p.p<double>(), z.p<double>(), p.elems(), s);
    ops::pcg_dots(n, r.p<double>(), z.p<double>(), SC, true, NV, s);
    // one iteration up to the copy of its residual; with gpu_graph (default)
    // one graph per (lane, x.zero, x) through run_graphed
    auto body = [&] {
        ops::pcg_ap(*A, p.p<double>(), Ap.p<double>(), SC, NV, s);
        Ap.zero = false;
        ops::pcg_xr(n, x.p<double>(), r.p<double>(), p.p<double>(), Ap.p<double>(), SC, x.zero,
                    NV, s);
        x.zero = false;
        x.init = true;
        apply_M(z, r);
        ops::pcg_dots(n, r.p<double>(), z.p<double>(), SC, false, NV, s);
        ops::pcg_p(n, p.p<double>(), z.p<double>(), SC, NV, s);
        post_scalars(SC + k::SC_RES * k::SC_STRIDE, NV);
    };
    do {
        ++st.iters;
        if (cfg.gpu_graph)
            run_graphed(step_graph(std::make_tuple(ctx().lane, x.zero, x.p<const void>())), &x,
                        body);
        else
            body();
        XG_CUDA(cudaStreamSynchronize(s));
        take_scalars(res.data(), NV);
        if (check(res.data(), rho0.data(), iconv)) return;
    } while (st.iters < cfg.max_iters);
    XG_CUDA(cudaStreamSynchronize(s));
}

// rbicgstab.inl:44-243 (rb_merged = false), merged_rbicgstab.inl:44-230
// (true). Kernels: v = A v_ with delta = (v, r0) and alpha; s = M^-1 v;
// t_ = z - alpha s; t = A t_; group 1 (r update, four dots, the scalar
// recurrences); z = M^-1 t; r = r - omega t (with the unmerged x update);
// convergence test; group 2.
void Krylov::solve_rbicgstab(DVec &x, DVec &b, const std::vector<double> &conv) {
    cudaStream_t s = S();
    std::vector<double> iconv = conv;
    upload_iconv(iconv);
    double *SC = sc.as<double>();
    for (auto &v : buf) {
        v.zero = true;
        v.init = true;
    }
    DVec &r0 = buf[0], &r = buf[1], &z = buf[2], &v_ = buf[3], &v = buf[4], &s_ = buf[5],
         &t_ = buf[6], &t = buf[7];
    std::vector<double> rho0(NV), res(NV);
    residual_norm<double>(*A, x, b, r0, NV, rho0.data());
    // copy(r0, r); rho = rho0
    ops::convert<double, double>(r.p<double>(), r0.p<double>(), r.elems(), s);
    r.zero = false;
    if (check(rho0.data(), rho0.data(), iconv)) return;
    XG_CUDA(cudaMemcpyAsync(SC + k::SC_RHO * k::SC_STRIDE, ctx().red_out.as<double>(),
                            NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
    apply_M(z, r0);
    v_.zero = z.zero;
    if (!z.zero) ops::convert<double, double>(v_.p<double>(), z.p<double>(), v_.elems(), s);
    // group 2 of a non-converged iteration runs at the start of the next
    // one, so that from the second iteration on the whole iteration up to
    // the copy of its residual is one graph per (lane, x.zero, x) through
    // run_graphed (gpu_graph, default)
    auto group2 = [&] {
        ops::rb_group2(n, x.p<double>(), v_.p<double>(), z.p<double>(), t_.p<double>(),
                       s_.p<double>(), SC, rb_merged, x.zero, NV, s);
        z.zero = v_.zero = false;
        if (rb_merged) {
            x.zero = false;
            x.init = true;
        }
    };
    bool tail = false;
    auto body = [&] {
        if (tail) group2();
        ops::spmv_dot_alpha(*A, v_.p<double>(), v.p<double>(), r0.p<double>(), SC, NV, s);
        v.zero = false;
        apply_M(s_, v);
        ops::rb_t(n, t_.p<double>(), z.p<double>(), s_.p<double>(), SC, z.zero, s_.zero, NV, s);
        t_.zero = false;
        ops::spmv<double>(*A, t_.p<double>(), t.p<double>(), NV, false, s);
        t.zero = false;
        ops::rb_group1(n, r.p<double>(), v.p<double>(), t.p<double>(), r0.p<double>(), SC, NV, s);
        apply_M(z, t);
        ops::rb_r(n, r.p<double>(), rb_merged ? nullptr : x.p<double>(), t.p<double>(),
                  v_.p<double>(), t_.p<double>(), SC, x.zero, NV, s);
        if (!rb_merged) {
            x.zero = false;
            x.init = true;
        }
        post_scalars(SC + k::SC_RES * k::SC_STRIDE, NV);
    };
    do {
        ++st.iters;
        if (cfg.gpu_graph && tail)
            run_graphed(step_graph(std::make_tuple(ctx().lane, x.zero, x.p<const void>())), &x,
                        body);
        else
            body();
        tail = false;
        XG_CUDA(cudaStreamSynchronize(s));
        take_scalars(res.data(), NV);
        if (check(res.data(), rho0.data(), iconv)) {
            if (rb_merged) {
                ops::rb_x(n, x.p<double>(), v_.p<double>(), t_.p<double>(), SC, x.zero, NV, s);
                x.zero = false;
                x.init = true;
            }
            return;
        }
        tail = true;
    } while (st.iters < cfg.max_iters);
    group2();
    XG_CUDA(cudaStreamSynchronize(s));
}

void Krylov::solve(DVec &x, DVec &b, const std::vector<double> &conv) {
    reset_stats();
    if (pcg) {
        solve_pcg(x, b, conv);
        return;
    }
    if (rbicgstab) {
        solve_rbicgstab(x, b, conv);
        return;
    }
    if (loop_ok() && launch_loop(x, b)) {
        loop_done(x);
        return;
    }
    begin(x, b, conv);
    XG_CUDA(cudaStreamSynchronize(S()));
    if (started()) return;
    if (persistent_ok()) {
        run_persistent(x);
        return;
    }
    while (true) {
        step();
        XG_CUDA(cudaStreamSynchronize(S()));
        if (stepped()) return;
        if (st.iters >= cfg.max_iters) break;
    }
    finish();
    XG_CUDA(cudaStreamSynchronize(S()));
}


// The whole solve as one graph (gpu_solve_graph): for the root solver of a
// merged BiCGStab form, with graphs on, no per-iteration printing and no
// persistent launch taking the solve.
bool Krylov::loop_ok() const {
    return cfg.gpu_solve_graph && cfg.gpu_graph && steppable() && !cfg.convergence_info &&
           role == "solver" && !persistent_ok();
}

static void graph_check(cudaError_t e) {
    if (e != cudaSuccess) throw Error(XAMG_ERR_CUDA, cudaGetErrorString(e));
}

// A conditional node of `type` after the capture's current dependencies on
// stream s; the capture then depends on the new node. Returns its body.
static cudaGraph_t add_conditional(cudaStream_t s, cudaGraphConditionalHandle h,
                                   cudaGraphConditionalNodeType type, cudaGraphNode_t *node) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    graph_check(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    XG_REQUIRE(st == cudaStreamCaptureStatusActive, XAMG_ERR_INTERNAL, "not capturing");
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    graph_check(cudaGraphAddNode(node, g, deps, nd, &np));
    graph_check(cudaStreamUpdateCaptureDependencies(s, node, 1, cudaStreamSetCaptureDependencies));
    return np.conditional.phGraph_out[0];
}

// Records the solve graph: [r0 = b - A x; test rho0 (k_loop_start)]
// WHILE(loop) { iteration up to its residual; test (k_loop_check);
// IF(rest) { the rest of the iteration }; IF(last) { final x update } }.
// The recording runs the host side of one solve (flags, pointers) without
// running its kernels; `flags` keeps the work vectors' flags it leaves.
bool Krylov::record_loop(LoopGraph &g, DVec &x, DVec &b) {
    cudaStream_t s = S();
    double *SC = sc.as<double>();
    if (!lout.bytes) lout.alloc(k::LOOP_COUNT * sizeof(double));
    XG_CUDA(cudaStreamSynchronize(s));
    auto code = [](const DVec &v) { return (uint8_t)((v.zero ? 1 : 0) | (v.init ? 2 : 0)); };
    std::vector<uint8_t> before(buf.size() + 1);
    for (size_t i = 0; i < buf.size(); ++i) before[i] = code(buf[i]);
    before[buf.size()] = code(x);
    cudaGraph_t G = nullptr;
    cudaGraph_t body = nullptr, rest = nullptr, last = nullptr;
    bool ok = true;
    const uint64_t l0 = g_kernel_launches;
    capturing_ = true;
    try {
        graph_check(cudaGraphCreate(&G, 0));
        k::LoopCtl c{NV, cfg.max_iters, cfg.convergence_check, cfg.abs_tol, cfg.rel_tol, 0, 0, 0};
        graph_check(cudaGraphConditionalHandleCreate(&c.loop, G, 0, cudaGraphCondAssignDefault));
        // start: the host side of begin(), r0 = b - A x, the test of rho0
        graph_check(cudaStreamBeginCaptureToGraph(s, G, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
        reset_stats();
        f32io = f32io_ready && static_cast<MultiGrid *>(M.get())->cfg.mg_cycle != 1;
        run_.x = &x;
        run_.b = &b;
        run_.tail = false;
        run_.iconv.assign(NV, 1.0);
        for (auto &v : buf) {
            v.zero = true;
            v.init = true;
        }
        DVec &r0 = buf[0], &r = buf[1], &p = buf[2];
        if (x.zero)
            ops::group1_zero(n, b.p<double>(), r0.p<double>(), p.p<double>(), r.p<double>(), SC,
                             NV, s);
        else
            ops::group1(*A, x.p<double>(), b.p<double>(), r0.p<double>(), p.p<double>(),
                        r.p<double>(), SC, NV, s);
        r0.zero = p.zero = r.zero = false;
        ops::loop_start(SC, lout.as<double>(), c, s);
        g.n_start = g_kernel_launches - l0;
        cudaGraphNode_t wn;
        body = add_conditional(s, c.loop, cudaGraphCondTypeWhile, &wn);
        graph_check(cudaStreamEndCapture(s, &G));
        // the loop body
        graph_check(cudaGraphConditionalHandleCreate(&c.rest, body, 0, cudaGraphCondAssignDefault));
        graph_check(cudaGraphConditionalHandleCreate(&c.last, body, 0, cudaGraphCondAssignDefault));
        graph_check(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
        run_.pa = M ? &buf[6] : &buf[2];
        run_.sa = M ? &buf[7] : &buf[4];
        in_loop_ = true;  // the residual stays on the device
        uint64_t l1 = g_kernel_launches;
        step_body();
        in_loop_ = false;
        ops::loop_check(SC, lout.as<double>(), c, s);
        g.n_body = g_kernel_launches - l1;
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        graph_check(cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, &deps, &nd));
        std::vector<cudaGraphNode_t> check_deps(deps, deps + nd);
        cudaGraphNode_t rn, ln;
        rest = add_conditional(s, c.rest, cudaGraphCondTypeIf, &rn);
        graph_check(cudaStreamUpdateCaptureDependencies(s, check_deps.data(), check_deps.size(),
                                                        cudaStreamSetCaptureDependencies));
        last = add_conditional(s, c.last, cudaGraphCondTypeIf, &ln);
        graph_check(cudaStreamEndCapture(s, &body));
        // IF(rest): the rest of a non-converged iteration
        graph_check(cudaStreamBeginCaptureToGraph(s, rest, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
        l1 = g_kernel_launches;
        step_tail();
        g.n_rest = g_kernel_launches - l1;
        graph_check(cudaStreamEndCapture(s, &rest));
        // IF(last): the final x update
        graph_check(cudaStreamBeginCaptureToGraph(s, last, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
        DVec &p2 = buf[2], &s2 = buf[4];
        l1 = g_kernel_launches;
        if (f32io)
            ops::x_update(n, x.p<double>(), pa32.p<float>(), sa32.p<float>(), SC, NV, s);
        else if (precond_form)
            ops::x_update(n, x.p<double>(), run_.pa->p<double>(), run_.sa->p<double>(), SC, NV,
                          s);
        else
            ops::x_update(n, x.p<double>(), p2.p<double>(), s2.p<double>(), SC, NV, s);
        x.zero = false;
        g.n_last = g_kernel_launches - l1;
        graph_check(cudaStreamEndCapture(s, &last));
        graph_check(cudaGraphInstantiate(&g.exec, G, 0));
    } catch (...) {
        ok = false;
        in_loop_ = false;
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(s, &junk);
        }
        cudaGetLastError();
        g.exec = nullptr;
    }
    capturing_ = false;
    if (G) cudaGraphDestroy(G);
    g_kernel_launches = l0;
    g.flags.resize(buf.size());
    for (size_t i = 0; i < buf.size(); ++i) g.flags[i] = code(buf[i]);
    // the flags the solve starts from (nothing of the recording ran)
    for (size_t i = 0; i < buf.size(); ++i) {
        buf[i].zero = before[i] & 1;
        buf[i].init = before[i] & 2;
    }
    x.zero = before[buf.size()] & 1;
    x.init = before[buf.size()] & 2;
    return ok;
}

// Runs the solve as one graph launch; false where it is run by steps instead
// (its first two calls for a key, which also tune the SpMVs, and solves that
// cannot be recorded).
bool Krylov::launch_loop(DVec &x, DVec &b) {
    LoopGraph &g = loop_graphs_[std::make_tuple(ctx().lane, x.p<const void>(), b.p<const void>(),
                                                x.zero)];
    if (g.failed || (!g.exec && g.calls++ < 2)) return false;
    if (!g.exec && !record_loop(g, x, b)) {
        g.failed = true;
        return false;
    }
    reset_stats();
    loop_x_zero_ = x.zero;
    run_.x = &x;
    run_.b = &b;
    run_.tail = false;
    XG_CUDA(cudaGraphLaunch(g.exec, S()));
    loop_run_ = &g;
    for (size_t i = 0; i < buf.size(); ++i) {
        buf[i].zero = g.flags[i] & 1;
        buf[i].init = g.flags[i] & 2;
    }
    return true;
}

// After the stream has passed a loop graph: statistics, and x's flags (x is
// written unless rho0 passed the test already).
void Krylov::loop_done(DVec &x) {
    Ctx &c = ctx();
    XG_CUDA(cudaMemcpyAsync(c.pinned, lout.p, k::LOOP_COUNT * sizeof(double),
                            cudaMemcpyDeviceToHost, S()));
    XG_CUDA(cudaStreamSynchronize(S()));
    const double *o = c.pinned;
    st.iters = (int)o[k::LOOP_ITERS];
    for (int kk = 0; kk < NV; ++kk) {
        st.conv[kk] = o[k::LOOP_CONV + kk] != 0.0 ? 1 : 0;
        st.abs_res[kk] = o[k::LOOP_ABS + kk];
        st.rel_res[kk] = o[k::LOOP_REL + kk];
    }
    x.zero = loop_x_zero_ && st.iters == 0;
    x.init = true;
    // the kernels the device loop ran: each iteration's body and test, then
    // the rest of the iteration, or the final x update when it converged
    if (loop_run_) {
        const LoopGraph &g = *loop_run_;
        const uint64_t it = (uint64_t)st.iters;
        const bool done = o[k::LOOP_DONE] != 0.0;
        g_kernel_launches += g.n_start + it * g.n_body;
        if (it) g_kernel_launches += done ? (it - 1) * g.n_rest + g.n_last : it * g.n_rest;
        loop_run_ = nullptr;
    }
}

// merged_bicgstab.inl:44-208 / merged_pbicgstab.inl:44-225
void Krylov::begin(DVec &x, DVec &b, const std::vector<double> &conv) {
    reset_stats();
    // the cycle type may have been renewed since the solver was built
    f32io = f32io_ready && static_cast<MultiGrid *>(M.get())->cfg.mg_cycle != 1;
    cudaStream_t s = S();
    run_.x = &x;
    run_.b = &b;
    run_.tail = false;
    run_.iconv = conv;
    run_.rho0.assign(NV, 0.0);
    run_.res.assign(NV, 0.0);
    upload_iconv(run_.iconv);
    double *SC = sc.as<double>();
    for (auto &v : buf) {
        v.zero = true;
        v.init = true;
    }
    DVec &r0 = buf[0], &r = buf[1], &p = buf[2];
    // 1-2: r0 = b - A x; rho0 = (r0, r0); p = r = r0 (rho = rho0)
    if (x.zero)
        ops::group1_zero(n, b.p<double>(), r0.p<double>(), p.p<double>(), r.p<double>(), SC, NV, s);
    else
        ops::group1(*A, x.p<double>(), b.p<double>(), r0.p<double>(), p.p<double>(),
                    r.p<double>(), SC, NV, s);
    r0.zero = p.zero = r.zero = false;
    post_scalars(SC + k::SC_RHO0 * k::SC_STRIDE, NV);
}

bool Krylov::started() {
    take_scalars(run_.rho0.data(), NV);
    return check(run_.rho0.data(), run_.rho0.data(), run_.iconv);
}

// gpu_persistent (default 1): the preconditioned forms (PBiCGStab,
// MergedPBiCGStab) with the Identity (no preconditioner list) or a Jacobi
// preconditioner without its own convergence test run every iteration in
// one cooperative launch when its blocks (the canonical blocks, 128 for the
// 32^3 Poisson system, shared gpu_persistent to a block) fit the GPU at
// once; printing residuals (convergence_info) keeps the host loop.
bool Krylov::persistent_ok() const {
    if (!cfg.gpu_persistent || !precond_form || cfg.convergence_info || f32) return false;
    if (M && !dynamic_cast<const Identity<double> *>(M.get())) {
        auto *j = dynamic_cast<const Jacobi<double> *>(M.get());
        if (!j || j->cfg.convergence_check || j->f32) return false;
    }
    return ops::pbicgstab_persist_fits(*A, NV, cfg.gpu_persistent);
}

void Krylov::run_persistent(DVec &x) {
    cudaStream_t s = S();
    auto *jac = M ? dynamic_cast<Jacobi<double> *>(M.get()) : nullptr;
    if (!psync.bytes) psync.alloc(2 * sizeof(unsigned));
    if (!pout.bytes) pout.alloc(128 * sizeof(double));
    XG_CUDA(cudaMemsetAsync(psync.p, 0, psync.bytes, s));
    const k::RedArgs ra = ctx().red();
    k::PersistArgs P{};
    P.x = x.p<double>();
    P.r0 = buf[0].p<double>();
    P.r = buf[1].p<double>();
    P.p = buf[2].p<double>();
    P.v = buf[3].p<double>();
    P.s = buf[4].p<double>();
    P.t = buf[5].p<double>();
    P.pa = M ? buf[6].p<double>() : P.p;
    P.sa = M ? buf[7].p<double>() : P.s;
    P.tmp = jac ? jac->buf[1].p<double>() : nullptr;
    P.d = jac ? jac->d.as<double>() : nullptr;
    P.ident = (M && !jac) ? 1 : 0;
    P.relax = jac ? (double)jac->cfg.relax : 0.0;
    P.sweeps = jac ? std::max(1, jac->cfg.max_iters) : 0;
    P.sc = sc.as<double>();
    P.out = pout.as<double>();
    P.max_iters = cfg.max_iters;
    P.check = cfg.convergence_check;
    P.abs_tol = cfg.abs_tol;
    P.rel_tol = cfg.rel_tol;
    P.ra = ra;
    P.gs = k::GridSync{psync.as<unsigned long long>(), ra.flag, 1000000000ull};
    ops::pbicgstab_persist(*A, P, NV, cfg.gpu_persistent, s);
    double out[97];
    XG_CUDA(cudaMemcpyAsync(out, pout.p, sizeof(out), cudaMemcpyDeviceToHost, s));
    ctx().check_flags();  // synchronises; XAMG_ERR_TIMEOUT if a grid wait ran out
    st.iters = (int)out[96];
    for (int k = 0; k < NV; ++k)
        if (out[64 + k] != 0.0) {
            st.conv[k] = 1;
            st.abs_res[k] = out[k];
            st.rel_res[k] = out[32 + k];
        }
    for (int i = 1; i < 8; ++i) buf[i].zero = false;
    x.zero = false;
    x.init = true;
}

void Krylov::drop_graphs() {
    for (auto &kv : graphs_)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto &kv : step_graphs_)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto &kv : loop_graphs_)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs_.clear();
    step_graphs_.clear();
    loop_graphs_.clear();
}

// The step graph for key; past 32 keys (many solution vectors) the graphs
// start over rather than keep one for each.
MGraph &Krylov::step_graph(const std::tuple<int, bool, const void *> &key) {
    if (step_graphs_.size() >= 32 && !step_graphs_.count(key)) {
        for (auto &kv : step_graphs_)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        step_graphs_.clear();
    }
    return step_graphs_[key];
}

// Runs body() directly on its first two calls for g (they settle the
// preconditioner's graphs, flags and launch shapes), records it as a CUDA
// graph on the third (the preconditioner's kernels inline) and replays it
// from then on: the same kernels and copies on the same buffers in one
// launch. The work vectors' flags, and x's when given (a body that writes
// x), are restored as the recording left them. A body that cannot be
// captured runs directly from then on.
void Krylov::run_graphed(MGraph &g, DVec *x, const std::function<void()> &body) {
    if (g.exec) {
        XG_CUDA(cudaGraphLaunch(g.exec, S()));
        g_kernel_launches += g.launches;
        for (size_t i = 0; i < buf.size(); ++i) {
            buf[i].zero = g.flags[i] & 1;
            buf[i].init = g.flags[i] & 2;
        }
        if (x) {
            x->zero = g.flags[buf.size()] & 1;
            x->init = g.flags[buf.size()] & 2;
        }
        return;
    }
    if (g.failed || g.calls++ < 2) {
        body();
        return;
    }
    auto code = [](const DVec &v) { return (uint8_t)((v.zero ? 1 : 0) | (v.init ? 2 : 0)); };
    auto snapshot = [&](std::vector<uint8_t> &f) {
        f.resize(buf.size() + 1);
        for (size_t i = 0; i < buf.size(); ++i) f[i] = code(buf[i]);
        f[buf.size()] = x ? code(*x) : 0;
    };
    auto restore = [&](const std::vector<uint8_t> &f) {
        for (size_t i = 0; i < buf.size(); ++i) {
            buf[i].zero = f[i] & 1;
            buf[i].init = f[i] & 2;
        }
        if (x) {
            x->zero = f[buf.size()] & 1;
            x->init = f[buf.size()] & 2;
        }
    };
    // The recording changes the host-side flags (x.zero, the work vectors'
    // zero/init) as if the body had run. When the capture fails, the direct
    // run below must start from the flags the body was called with, or its
    // kernels would treat a zero-flagged x as holding values.
    std::vector<uint8_t> before;
    snapshot(before);
    XG_CUDA(cudaStreamSynchronize(S()));
    XG_CUDA(cudaStreamBeginCapture(S(), cudaStreamCaptureModeThreadLocal));
    const uint64_t l0 = g_kernel_launches;
    cudaGraph_t graph = nullptr;
    bool ok = true;
    capturing_ = true;
    try {
        body();  // recorded, not run
    } catch (...) {
        ok = false;
    }
    capturing_ = false;
    const cudaError_t e = cudaStreamEndCapture(S(), &graph);
    if (!ok || e != cudaSuccess || !graph ||
        cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
        // nothing ran during the capture: run directly from now on
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
        g.exec = nullptr;
        g.failed = true;
        g_kernel_launches = l0;
        restore(before);
        body();
        return;
    }
    cudaGraphDestroy(graph);
    g.launches = g_kernel_launches - l0;
    snapshot(g.flags);
    XG_CUDA(cudaGraphLaunch(g.exec, S()));
}

// The previous iteration's tail (when its residual did not converge) and
// this iteration up to its residual; with gpu_graph (default) one graph per
// (lane, tail or not, x) through run_graphed.
void Krylov::step() {
    ++st.iters;
    run_.pa = M ? &buf[6] : &buf[2];
    run_.sa = M ? &buf[7] : &buf[4];
    const bool tail = run_.tail;
    run_.tail = false;
    auto body = [&] {
        if (tail) step_tail();
        step_body();
    };
    if (!cfg.gpu_graph) {
        body();
        return;
    }
    run_graphed(step_graph(std::make_tuple(ctx().lane, tail, run_.x->p<const void>())),
                tail ? run_.x : nullptr, body);
}

void Krylov::step_body() {
    cudaStream_t s = S();
    double *SC = sc.as<double>();
    DVec &r0 = buf[0], &r = buf[1], &p = buf[2], &v = buf[3], &s_ = buf[4], &t = buf[5],
         &p_ = buf[6], &s2 = buf[7];
    run_.pa = &p;
    run_.sa = &s_;
    if (f32io) {
        apply_M(pa32, p);
        ops::spmv_dot_alpha(*A, pa32.p<float>(), v.p<double>(), r0.p<double>(), SC, NV, s);
        v.zero = false;
        ops::s_update(n, s_.p<double>(), r.p<double>(), v.p<double>(), SC, NV, s);
        s_.zero = false;
        apply_M(sa32, s_);
        ops::spmv_dot3(*A, sa32.p<float>(), t.p<double>(), s_.p<double>(), SC, NV, s);
        t.zero = false;
        if (!in_loop_) post_scalars(SC + k::SC_RES * k::SC_STRIDE, NV);
        return;
    }
    if (M) {
        apply_M(p_, p);
        run_.pa = &p_;
    }
    // v = A p_; alpha = rho / (v, r0)
    ops::spmv_dot_alpha(*A, run_.pa->p<double>(), v.p<double>(), r0.p<double>(), SC, NV, s);
    v.zero = false;
    // s = r - alpha v
    ops::s_update(n, s_.p<double>(), r.p<double>(), v.p<double>(), SC, NV, s);
    s_.zero = false;
    if (M) {
        apply_M(s2, s_);
        run_.sa = &s2;
    }
    // t = A s_; omega = (t,s)/(t,t); res = (s,s) - omega (t,s)
    ops::spmv_dot3(*A, run_.sa->p<double>(), t.p<double>(), s_.p<double>(), SC, NV, s);
    t.zero = false;
    if (!in_loop_) post_scalars(SC + k::SC_RES * k::SC_STRIDE, NV);
}

bool Krylov::stepped() {
    cudaStream_t s = S();
    double *SC = sc.as<double>();
    DVec &p = buf[2], &s_ = buf[4];
    DVec &x = *run_.x;
    take_scalars(run_.res.data(), NV);
    const bool done = check(run_.res.data(), run_.rho0.data(), run_.iconv);
    if (!done) {
        run_.tail = true;  // launched by the next step() or by finish()
        return false;
    }
    if (f32io)
        ops::x_update(n, x.p<double>(), pa32.p<float>(), sa32.p<float>(), SC, NV, s);
    else if (precond_form)
        ops::x_update(n, x.p<double>(), run_.pa->p<double>(), run_.sa->p<double>(), SC, NV, s);
    else
        ops::x_update(n, x.p<double>(), p.p<double>(), s_.p<double>(), SC, NV, s);
    x.zero = false;
    return true;
}

void Krylov::finish() {
    if (!run_.tail) return;
    run_.tail = false;
    step_tail();
}

// The rest of an iteration whose residual did not converge.
void Krylov::step_tail() {
    cudaStream_t s = S();
    double *SC = sc.as<double>();
    DVec &r0 = buf[0], &r = buf[1], &p = buf[2], &v = buf[3], &s_ = buf[4], &t = buf[5];
    DVec &x = *run_.x;
    if (f32io) {
        ops::group4(n, s_.p<double>(), t.p<double>(), r0.p<double>(), r.p<double>(),
                    x.p<double>(), pa32.p<float>(), sa32.p<float>(), SC, NV, s);
        ops::p_update(n, p.p<double>(), r.p<double>(), v.p<double>(), SC, NV, s);
    } else if (precond_form) {
        // x update fused with r = s - omega t; rho = (r, r0); beta
        ops::group4(n, s_.p<double>(), t.p<double>(), r0.p<double>(), r.p<double>(),
                    x.p<double>(), run_.pa->p<double>(), run_.sa->p<double>(), true, SC, NV, s);
        ops::p_update(n, p.p<double>(), r.p<double>(), v.p<double>(), SC, NV, s);
    } else {
        ops::group4(n, s_.p<double>(), t.p<double>(), r0.p<double>(), r.p<double>(), nullptr,
                    nullptr, nullptr, false, SC, NV, s);
        ops::group5(n, x.p<double>(), p.p<double>(), s_.p<double>(), r.p<double>(),
                    v.p<double>(), SC, NV, s);
    }
    x.zero = false;
}

// ===========================================================================
// construct_solver_hierarchy (solver.h:259-276, 481-500)
// ===========================================================================
void SolverHierarchy::build(const Params &P, const HCsr &hA_, const DCsr *A_, int nv,
                            HierCache *cache) {
    params = P;
    hA = hA_;
    A = A_;
    NV = nv;
    XG_REQUIRE(P.has("solver"), XAMG_ERR_INVALID_ARG, "parameters have no 'solver' list");
    SolverCfg c = resolve_cfg(P.get("solver"), "solver");
    const std::string &m = c.method;
    mg = nullptr;
    if (m == "MultiGrid") {
        auto *g = new MultiGrid();
        g->build(hA, A, P, "solver", nv, cache);
        mg = g;
        root.reset(g);
        return;
    }
    if (m == "MergedPBiCGStab" || m == "PBiCGStab" || m == "MergedBiCGStab" || m == "BiCGStab" ||
        m == "PCG" || m == "RBiCGStab" || m == "MergedRBiCGStab") {
        auto *kr = new Krylov();
        kr->cfg = c;
        kr->role = "solver";
        kr->NV = nv;
        kr->A = A;
        kr->n = hA.nrows;
        kr->precond_form = (m != "MergedBiCGStab");
        kr->pcg = (m == "PCG");
        kr->rbicgstab = (m == "RBiCGStab" || m == "MergedRBiCGStab");
        kr->rb_merged = (m == "MergedRBiCGStab");
        kr->setup();
        const bool wants_M = (m == "MergedPBiCGStab" || m == "PBiCGStab" || m == "PCG" ||
                              kr->rbicgstab);
        if (wants_M && P.has("preconditioner")) {
            SolverCfg pc = resolve_cfg(P.get("preconditioner"), "preconditioner");
            if (pc.method == "MultiGrid") {
                auto *g = new MultiGrid();
                g->build(hA, A, P, "preconditioner", nv, cache);
                mg = g;
                kr->M.reset(g);
            } else {
                kr->M = make_smoother(pc, "preconditioner", *A, hA, false, nv, 0, 0);
                if (pc.method == "Chebyshev") {
                    double mn, mx;
                    estimate_eigs(hA, 10, pc.gpu_seed, mn, mx);
                    auto *ch = dynamic_cast<Chebyshev<double> *>(kr->M.get());
                    if (ch) {
                        ch->min_eig = mn;
                        ch->max_eig = mx;
                    }
                }
            }
        } else if (wants_M) {
            // no preconditioner list: Identity (p_ = p), as XAMG's default
            SolverCfg ic;
            ic.method = "Identity";
            kr->M = make_smoother(ic, "preconditioner", *A, hA, false, nv, 0, 0);
        }
        kr->enable_f32io();
        root.reset(kr);
        return;
    }
    if (m == "Jacobi" || m == "HSGS" || m == "Chebyshev" || m == "Direct" || m == "Identity") {
        double mn = 0, mx = 0;
        if (m == "Chebyshev") estimate_eigs(hA, 10, c.gpu_seed, mn, mx);
        root = make_smoother(c, "solver", *A, hA, false, nv, mn, mx);
        return;
    }
    throw Error(XAMG_ERR_UNSUPPORTED, "solver method not implemented: " + m);
}

void SolverHierarchy::solve(DVec &x, DVec &b) {
    std::vector<double> ones(NV, 1.0);
    root->solve(x, b, ones);
    XG_CUDA(cudaStreamSynchronize(ctx().stream));
}

void solve_batch(const std::vector<SolverHierarchy *> &hs, const std::vector<DVec *> &xs,
                 const std::vector<DVec *> &bs) {
    Ctx &c = ctx();
    XG_REQUIRE(c.lane == 0, XAMG_ERR_INTERNAL, "batch solve started off lane 0");
    const int m = (int)hs.size();
    struct Guard {  // lane 0 current again on every exit; events released
        cudaEvent_t ev = nullptr;
        ~Guard() {
            try {
                ctx().use_lane(0);
            } catch (...) {
            }
            if (ev) cudaEventDestroy(ev);
        }
    } guard;
    XG_CUDA(cudaEventCreateWithFlags(&guard.ev, cudaEventDisableTiming));
    XG_CUDA(cudaEventRecord(guard.ev, c.stream));
    std::vector<Krylov *> kr(m, nullptr);
    std::vector<char> live(m, 0);
    for (int i = 0; i < m; ++i) {
        c.use_lane(i + 1);
        XG_CUDA(cudaStreamWaitEvent(c.stream, guard.ev, 0));
    }
    // systems whose whole solve runs as one graph launch (gpu_solve_graph)
    std::vector<char> looped(m, 0);
    for (int i = 0; i < m; ++i) {
        c.use_lane(i + 1);
        std::vector<double> ones(hs[i]->NV, 1.0);
        kr[i] = dynamic_cast<Krylov *>(hs[i]->root.get());
        if (kr[i] && kr[i]->loop_ok() && kr[i]->launch_loop(*xs[i], *bs[i])) {
            looped[i] = 1;
        } else if (kr[i] && kr[i]->steppable()) {
            kr[i]->begin(*xs[i], *bs[i], ones);
            live[i] = 1;
        } else {
            hs[i]->root->solve(*xs[i], *bs[i], ones);
        }
    }
    for (int i = 0; i < m; ++i)
        if (live[i]) {
            c.use_lane(i + 1);
            XG_CUDA(cudaStreamSynchronize(c.stream));
            if (kr[i]->started()) live[i] = 0;
        }
    for (;;) {
        bool any = false;
        for (int i = 0; i < m; ++i)
            if (live[i]) {
                c.use_lane(i + 1);
                kr[i]->step();
                any = true;
            }
        if (!any) break;
        for (int i = 0; i < m; ++i)
            if (live[i]) {
                c.use_lane(i + 1);
                XG_CUDA(cudaStreamSynchronize(c.stream));
                if (kr[i]->stepped()) {
                    live[i] = 0;
                } else if (kr[i]->st.iters >= kr[i]->cfg.max_iters) {
                    kr[i]->finish();
                    live[i] = 0;
                }
            }
    }
    for (int i = 0; i < m; ++i)
        if (looped[i]) {
            c.use_lane(i + 1);
            kr[i]->loop_done(*xs[i]);
        }
    // join: lane 0 waits for every lane; then each lane's wait-timeout flag
    for (int i = 0; i < m; ++i) {
        c.use_lane(i + 1);
        XG_CUDA(cudaEventRecord(guard.ev, c.stream));
        c.use_lane(0);
        XG_CUDA(cudaStreamWaitEvent(c.stream, guard.ev, 0));
    }
    for (int i = 0; i < m; ++i) {
        c.use_lane(i + 1);
        c.check_flags();
    }
    c.use_lane(0);
    XG_CUDA(cudaStreamSynchronize(c.stream));
}


}  // namespace xg
