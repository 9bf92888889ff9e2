// XAMG solve-phase oracle: a CPU restatement of the reference algorithm.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg use it, and only as the checker.
//
// Every function cites the reference file:line it restates (paths relative to
// the XAMG source tree). Build flags: -O2 -ffp-contract=off, so that every
// a*x+b*y is a rounded multiply followed by a rounded add, as in the
// reference's -std=c++11 build (no FMA contraction).
//
// Reduction order. XAMG sums dot products sequentially over each core's row
// range and then adds the per-core partials (blas.inl:465-532,
// shm_allreduce.h:112-163). The oracle offers that order (mode 0, `ncores`
// core ranges as in part.h:115-134) and, as a second mode, the fixed order the
// B200 kernels use (mode 1, see canon_reduce below), so that a whole GPU solve
// can be compared bit for bit.
//
// Parity status: the hierarchy comes from the product's host AMG builder (the
// reference obtains it from hypre 2.20.0, which is not available); the oracle
// restates everything XAMG does after hypre returns.

#ifdef _OPENMP
#include <omp.h>
#endif
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>


namespace orc {

// ----------------------------------------------------------------------------
// Integer type coding and narrowing: xamg_types.h:49-75, bit_operations.h:67-131
// ----------------------------------------------------------------------------
static const uint16_t I8_TYPE = 0, I16_TYPE = 1, I32_TYPE = 2, I64_TYPE = 3;
static const uint16_t F32_TYPE = 5, F64_TYPE = 6;
static const uint16_t I1_OFFSET = 3, I2_OFFSET = 5, I3_OFFSET = 7, I4_OFFSET = 9;
static const uint16_t F_MASK = 7;

// bit_operations.h:119-129
static uint16_t define_int_type(uint64_t range) {
    if (range <= UINT8_MAX) return I8_TYPE;
    if (range <= UINT16_MAX) return I16_TYPE;
    if (range <= UINT32_MAX) return I32_TYPE;
    return I64_TYPE;
}

// csr_matrix.h:455-461 plus the reduced-precision override of matrix.h:80-84
static uint16_t encode_hash(uint64_t nonzeros, uint64_t ncols, uint64_t block_nrows,
                            uint64_t block_ncols, bool f32, bool reduced_prec) {
    uint16_t hash = (define_int_type(nonzeros) << I1_OFFSET) |
                    (define_int_type(ncols) << I2_OFFSET) |
                    (define_int_type(block_nrows) << I3_OFFSET) |
                    (define_int_type(block_ncols) << I4_OFFSET);
    hash |= f32 ? F32_TYPE : F64_TYPE;
    if (reduced_prec) {
        hash |= F_MASK;
        hash &= (uint16_t)(~F_MASK | F32_TYPE);
    }
    return hash;
}

// ----------------------------------------------------------------------------
// Core partition: misc.h:47-55 (split_range<float64_t>), part.h:115-134
// ----------------------------------------------------------------------------
static uint64_t split_range_f64(uint64_t size, int nblocks) {
    const uint32_t factor = 64 / 8;  // XAMG_ALIGN_SIZE / sizeof(float64_t)
    uint64_t core_size = size / nblocks;
    core_size += factor - (core_size % factor);
    return core_size;
}

static void core_range(uint64_t n, int ncores, int core, uint64_t &offset, uint64_t &size) {
    uint64_t cs = split_range_f64(n, ncores);
    offset = std::min<uint64_t>(n, cs * core);
    size = std::min<uint64_t>(cs, n - offset);
}

// ----------------------------------------------------------------------------
// Reduction orders
// ----------------------------------------------------------------------------
// Element-wise loops over vector entries are independent (each entry is
// computed by one thread from its own inputs), so threads change no result.
#define OR_PAR _Pragma("omp parallel for schedule(static)")

struct RedCfg {
    int mode = 0;    // 0: XAMG core-partitioned sequential, 1: B200 canonical
    int ncores = 1;  // XAMG cores of the single NUMA domain
};
static RedCfg g_red;

// B200 canonical order (restates the kernels' fixed schedule): a block of 256
// threads, thread t handles row slot t/NV and component t%NV; tiles of
// 256/NV rows are dealt to B = min(ntiles, 1184) blocks round-robin; each
// thread sums its rows in tile order; lanes with equal component are combined
// by an xor butterfly over offsets 16..NV; the 8 warp sums are added in warp
// order; the block partials are summed by one warp, lane l taking blocks
// l, l+32, ..., followed by an xor butterfly over 16..1.
static const int CANON_THREADS = 256;
static const int CANON_BMAX = 1184;

template <typename T, typename Term>
static void canon_reduce(uint64_t n, int NV, int nred, Term term, T *out) {
    for (int i = 0; i < NV * nred; ++i) out[i] = 0;
    if (n == 0) return;
    const uint64_t R = CANON_THREADS / NV;
    const uint64_t ntiles = (n + R - 1) / R;
    const uint64_t B = std::min<uint64_t>(ntiles, CANON_BMAX);
    std::vector<T> partial(B * NV * nred);
    // blocks are independent until their partials are combined below, so
    // they run on the host threads without changing any sum
#pragma omp parallel
    {
    std::vector<T> acc(CANON_THREADS * nred);
    std::vector<T> v(nred);
#pragma omp for schedule(static)
    for (uint64_t b = 0; b < B; ++b) {
        std::fill(acc.begin(), acc.end(), T(0));
        for (int t = 0; t < CANON_THREADS; ++t) {
            const int rt = t / NV, k = t % NV;
            for (uint64_t tile = b; tile < ntiles; tile += B) {
                uint64_t row = tile * R + rt;
                if (row < n) {
                    term(row, k, v.data());
                    for (int r = 0; r < nred; ++r) acc[t * nred + r] = acc[t * nred + r] + v[r];
                }
            }
        }
        std::vector<T> wsum(8 * NV * nred);
        for (int w = 0; w < 8; ++w) {
            for (int r = 0; r < nred; ++r) {
                T lane[32], tmp[32];
                for (int l = 0; l < 32; ++l) lane[l] = acc[(32 * w + l) * nred + r];
                for (int off = 16; off >= NV; off >>= 1) {
                    for (int l = 0; l < 32; ++l) tmp[l] = lane[l];
                    for (int l = 0; l < 32; ++l) lane[l] = tmp[l] + tmp[l ^ off];
                }
                for (int k = 0; k < NV; ++k) wsum[(w * NV + k) * nred + r] = lane[k];
            }
        }
        for (int k = 0; k < NV; ++k)
            for (int r = 0; r < nred; ++r) {
                T s = wsum[(0 * NV + k) * nred + r];
                for (int w = 1; w < 8; ++w) s = s + wsum[(w * NV + k) * nred + r];
                partial[(b * NV + k) * nred + r] = s;
            }
    }
    }
    for (int k = 0; k < NV; ++k)
        for (int r = 0; r < nred; ++r) {
            T lane[32], tmp[32];
            for (int l = 0; l < 32; ++l) {
                T a = 0;
                for (uint64_t bb = l; bb < B; bb += 32) a = a + partial[(bb * NV + k) * nred + r];
                lane[l] = a;
            }
            for (int off = 16; off >= 1; off >>= 1) {
                for (int l = 0; l < 32; ++l) tmp[l] = lane[l];
                for (int l = 0; l < 32; ++l) lane[l] = tmp[l] + tmp[l ^ off];
            }
            out[k * nred + r] = lane[0];
        }
}

// XAMG order: per-core sequential partial sums (blas.inl:504-519,
// blas_merged_bicgstab.inl:60-72), then the partials added in core order
// (the shared-memory allreduce, shm_allreduce.h:112-163).
template <typename T, typename Term>
static void xamg_reduce(uint64_t n, int NV, int nred, Term term, T *out) {
    const int ncores = std::max(1, g_red.ncores);
    std::vector<T> part(ncores * NV * nred, T(0));
    // each core's partial is summed on its own, as XAMG's ranks do
#pragma omp parallel for schedule(static, 1)
    for (int c = 0; c < ncores; ++c) {
        std::vector<T> v(nred);
        uint64_t off, sz;
        core_range(n, ncores, c, off, sz);
        T *p = &part[c * NV * nred];
        for (uint64_t i = off; i < off + sz; ++i)
            for (int k = 0; k < NV; ++k) {
                term(i, k, v.data());
                for (int r = 0; r < nred; ++r) p[k * nred + r] = p[k * nred + r] + v[r];
            }
    }
    for (int i = 0; i < NV * nred; ++i) {
        T s = part[i];
        for (int c = 1; c < ncores; ++c) s = s + part[c * NV * nred + i];
        out[i] = s;
    }
}

template <typename T, typename Term>
static void reduce(uint64_t n, int NV, int nred, Term term, T *out) {
    if (g_red.mode == 1)
        canon_reduce<T>(n, NV, nred, term, out);
    else
        xamg_reduce<T>(n, NV, nred, term, out);
}

// ----------------------------------------------------------------------------
// Vector with XAMG's state flags: vector.h:90-99 (if_zero defaults to true)
// ----------------------------------------------------------------------------
struct Vec {
    uint64_t size = 0;
    int nv = 0;
    bool f32 = false;
    bool init = false;
    bool zero = true;
    std::vector<double> d;
    std::vector<float> f;

    void alloc(uint64_t n, int nv_, bool is_f32) {
        size = n;
        nv = nv_;
        f32 = is_f32;
        if (f32)
            f.assign(n * nv, 0.0f);
        else
            d.assign(n * nv, 0.0);
        init = false;
        zero = true;
    }
    template <typename T>
    T *p();
    template <typename T>
    const T *p() const;
    bool empty() const { return size == 0; }
};
template <>
double *Vec::p<double>() { return d.data(); }
template <>
float *Vec::p<float>() { return f.data(); }
template <>
const double *Vec::p<double>() const { return d.data(); }
template <>
const float *Vec::p<float>() const { return f.data(); }

static Vec scalar_vec(int nv, double val) {
    Vec v;
    v.alloc(1, nv, false);
    for (int k = 0; k < nv; ++k) v.d[k] = val;
    v.init = true;
    v.zero = (std::fabs(val) < 1.e-100);
    return v;
}

template <typename T>
static Vec typed_scalar(int nv, double val) {
    Vec v;
    v.alloc(1, nv, sizeof(T) == 4);
    for (int k = 0; k < nv; ++k) v.p<T>()[k] = (T)val;
    v.init = true;
    v.zero = (std::fabs(val) < 1.e-100);
    return v;
}

// ----------------------------------------------------------------------------
// BLAS1 with the reference's flag short-circuits: blas.inl, blas_ext.inl,
// blas_wrapper.inl. NV is the interleave width of the n-sized vectors.
// ----------------------------------------------------------------------------
namespace blas {

// blas.inl:335-385 (set_const with a vector value)
template <typename T>
void set_const_v(Vec &x, const Vec &val, bool force) {
    if (val.zero && !force) {
        x.init = true;
        x.zero = true;
        return;
    }
    if (x.empty()) {
        x.init = true;
        x.zero = false;
        return;
    }
    T *xp = x.p<T>();
    const T *vp = val.p<T>();
    const int NV = x.nv;
    if (val.size == 1 && val.nv == 1) {
        OR_PAR
        for (uint64_t i = 0; i < x.size * NV; ++i) xp[i] = vp[0];
    } else {
        OR_PAR
        for (uint64_t i = 0; i < x.size * NV; i += NV)
            for (int k = 0; k < NV; ++k) xp[i + k] = vp[k];
    }
    x.init = true;
    x.zero = false;
}

// blas_wrapper.inl:30-43 (a fresh vector is zero-flagged unless |a| > 1e-100)
template <typename T>
void set_const(Vec &x, double a, bool force = false) {
    Vec v;
    v.alloc(1, x.nv, sizeof(T) == 4);
    if (std::fabs(a) > 1.e-100) v.zero = false;
    for (int k = 0; k < x.nv; ++k) v.p<T>()[k] = (T)a;
    v.init = true;
    set_const_v<T>(x, v, force);
}

// blas.inl:640-645 + blas_wrapper.inl:62-75
template <typename T>
void forced_set_const(Vec &x, double a) {
    Vec v;
    v.alloc(1, x.nv, sizeof(T) == 4);
    if (std::fabs(a) > 1.e-100) v.zero = false;
    for (int k = 0; k < x.nv; ++k) v.p<T>()[k] = (T)a;
    v.init = true;
    set_const_v<T>(x, v, true);
}

// blas.inl:30-85
template <typename T>
void ax_y(const Vec &a, const Vec &x, Vec &y) {
    if (a.zero || x.zero) {
        y.init = true;
        y.zero = true;
        return;
    }
    if (x.empty() && y.empty()) {
        y.init = true;
        y.zero = false;
        return;
    }
    const int NV = y.nv;
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    const T *ap = a.p<T>();
    if (a.nv == 1) {
        OR_PAR
        for (uint64_t i = 0; i < NV * y.size; ++i) yp[i] = ap[0] * xp[i];
    } else {
        OR_PAR
        for (uint64_t i = 0; i < NV * y.size; i += NV)
            for (int k = 0; k < NV; ++k) yp[i + k] = ap[k] * xp[i + k];
    }
    y.init = true;
    y.zero = false;
}

template <typename T>
void scal(const Vec &x, Vec &y);

// blas.inl:89-151
template <typename T>
void axpby(const Vec &a, const Vec &x, const Vec &b, Vec &y) {
    if (a.zero || x.zero) {
        scal<T>(b, y);
        return;
    }
    if (b.zero || y.zero) {
        ax_y<T>(a, x, y);
        return;
    }
    if (x.empty() && y.empty()) {
        y.zero = false;
        return;
    }
    const int NV = y.nv;
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    const T *ap = a.p<T>();
    const T *bp = b.p<T>();
    if (a.nv == 1) {
        OR_PAR
        for (uint64_t i = 0; i < NV * y.size; ++i) yp[i] = ap[0] * xp[i] + bp[0] * yp[i];
    } else {
        OR_PAR
        for (uint64_t i = 0; i < NV * y.size; i += NV)
            for (int k = 0; k < NV; ++k) yp[i + k] = ap[k] * xp[i + k] + bp[k] * yp[i + k];
    }
    y.zero = false;
}

// blas_wrapper.inl:79-99
template <typename T>
void axpby_s(double a, const Vec &x, double b, Vec &y) {
    Vec v1, v2;
    v1.alloc(1, y.nv, sizeof(T) == 4);
    v2.alloc(1, y.nv, sizeof(T) == 4);
    if (std::fabs(a) > 1.e-100) v1.zero = false;
    if (std::fabs(b) > 1.e-100) v2.zero = false;
    for (int k = 0; k < y.nv; ++k) {
        v1.p<T>()[k] = (T)a;
        v2.p<T>()[k] = (T)b;
    }
    v1.init = v2.init = true;
    axpby<T>(v1, x, v2, y);
}

// blas.inl:155-219
template <typename T>
void scal(const Vec &x, Vec &y) {
    if (x.zero || y.zero) {
        y.zero = true;
        return;
    }
    if (x.empty() && y.empty()) return;
    if (y.empty() && x.size == 1) return;
    const int NV = y.nv;
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    if (x.nv == 1) {
        if (x.size == 1) {
            OR_PAR
            for (uint64_t i = 0; i < NV * y.size; ++i) yp[i] *= xp[0];
        } else {
            OR_PAR
            for (uint64_t i = 0; i < y.size; ++i)
                for (int k = 0; k < NV; ++k) yp[i * NV + k] *= xp[i];
        }
    } else {
        if (x.size == 1) {
            OR_PAR
            for (uint64_t i = 0; i < NV * y.size; i += NV)
                for (int k = 0; k < NV; ++k) yp[i + k] *= xp[k];
        } else {
            OR_PAR
            for (uint64_t i = 0; i < NV * y.size; ++i) yp[i] *= xp[i];
        }
    }
}

// blas.inl:223-307 (single NUMA domain: same sharing mode)
template <typename T>
void copy(const Vec &x, Vec &y) {
    if (x.zero) {
        y.init = true;
        y.zero = x.zero;
        return;
    }
    if (x.empty()) {
        y.init = true;
        y.zero = x.zero;
        return;
    }
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    OR_PAR
    for (uint64_t i = 0; i < (uint64_t)x.nv * x.size; ++i) yp[i] = xp[i];
    y.init = true;
    y.zero = false;
}

// blas.inl:463-532 (+ the identity allreduce of one rank)
template <typename T>
void dot(const Vec &x, const Vec &y, Vec &res) {
    if (x.zero || y.zero) {
        res.init = true;
        res.zero = true;
        set_const<T>(res, 0, true);
        return;
    }
    if (x.empty() && y.empty()) {
        res.init = true;
        set_const<T>(res, 0, true);
        res.zero = false;
        return;
    }
    const int NV = x.nv;
    const T *xp = x.p<T>();
    const T *yp = y.p<T>();
    T *rp = res.p<T>();
    reduce<T>(x.size, NV, 1,
              [&](uint64_t i, int k, T *v) { v[0] = xp[i * NV + k] * yp[i * NV + k]; }, rp);
    res.init = true;
    res.zero = false;
}

// blas_ext.inl:30-102
template <typename T>
void axpby_z(const Vec &a, const Vec &x, const Vec &b, const Vec &y, Vec &z) {
    if (a.zero || x.zero) {
        ax_y<T>(b, y, z);
        return;
    }
    if (b.zero || y.zero) {
        ax_y<T>(a, x, z);
        return;
    }
    if (x.empty() && y.empty() && z.empty()) {
        z.init = true;
        z.zero = false;
        return;
    }
    const int NV = z.nv;
    const T *xp = x.p<T>();
    const T *yp = y.p<T>();
    T *zp = z.p<T>();
    const T *ap = a.p<T>();
    const T *bp = b.p<T>();
    if (a.nv == 1) {
        OR_PAR
        for (uint64_t i = 0; i < NV * z.size; i += NV)
            for (int k = 0; k < NV; ++k) zp[i + k] = ap[0] * xp[i + k] + bp[0] * yp[i + k];
    } else {
        OR_PAR
        for (uint64_t i = 0; i < NV * z.size; i += NV)
            for (int k = 0; k < NV; ++k) zp[i + k] = ap[k] * xp[i + k] + bp[k] * yp[i + k];
    }
    z.init = true;
    z.zero = false;
}

// blas_ext.inl:106-189
template <typename T>
void axpbypcz(const Vec &a, const Vec &x, const Vec &b, const Vec &y, const Vec &c, Vec &z) {
    if (a.zero || x.zero) {
        axpby<T>(b, y, c, z);
        return;
    }
    if (b.zero || y.zero) {
        axpby<T>(a, x, c, z);
        return;
    }
    if (c.zero || z.zero) {
        axpby_z<T>(a, x, b, y, z);
        return;
    }
    if (x.empty() && y.empty() && z.empty()) {
        z.zero = false;
        return;
    }
    const int NV = z.nv;
    const T *xp = x.p<T>();
    const T *yp = y.p<T>();
    T *zp = z.p<T>();
    const T *ap = a.p<T>();
    const T *bp = b.p<T>();
    const T *cp = c.p<T>();
    if (a.nv == 1) {
        OR_PAR
        for (uint64_t i = 0; i < NV * z.size; i += NV)
            for (int k = 0; k < NV; ++k)
                zp[i + k] = ap[0] * xp[i + k] + bp[0] * yp[i + k] + cp[0] * zp[i + k];
    } else {
        OR_PAR
        for (uint64_t i = 0; i < NV * z.size; i += NV)
            for (int k = 0; k < NV; ++k)
                zp[i + k] = ap[k] * xp[i + k] + bp[k] * yp[i + k] + cp[k] * zp[i + k];
    }
    z.zero = false;
}

// blas_ext.inl:193-239
template <typename T>
void xdivy_z(const Vec &x, const Vec &y, Vec &z) {
    if (x.zero) {
        set_const<T>(z, 0.0);
        return;
    }
    if (y.zero) return;  // the reference asserts here
    const T *xp = x.p<T>();
    const T *yp = y.p<T>();
    T *zp = z.p<T>();
    OR_PAR
    for (uint64_t i = 0; i < (uint64_t)x.nv * x.size; ++i) zp[i] = xp[i] / yp[i];
    z.init = true;
    z.zero = false;
}

// blas_merged_bicgstab.inl:32-87
template <typename T>
void merged_bicgstab_group1(Vec &r0, Vec &b, Vec &p, Vec &r, Vec &rho0) {
    if (b.zero) forced_set_const<T>(b, 0.0);
    if (r0.zero) set_const<T>(r0, 0.0, true);
    const int NV = r0.nv;
    T *r0p = r0.p<T>();
    const T *bp = b.p<T>();
    T *pp = p.p<T>();
    T *rp = r.p<T>();
    // elementwise part first; the sums do not feed back into it
    OR_PAR
    for (uint64_t i = 0; i < NV * r0.size; ++i) {
        r0p[i] = bp[i] - r0p[i];
        pp[i] = r0p[i];
        rp[i] = r0p[i];
    }
    reduce<T>(r0.size, NV, 1,
              [&](uint64_t i, int k, T *v) { v[0] = r0p[i * NV + k] * r0p[i * NV + k]; },
              rho0.p<T>());
    rho0.init = p.init = r.init = true;
    r0.zero = rho0.zero = p.zero = r.zero = false;
}

// blas_merged_bicgstab.inl:89-147
template <typename T>
void merged_bicgstab_group2(Vec &t, Vec &s, Vec &phi, Vec &psi, Vec &theta) {
    if (t.zero) forced_set_const<T>(t, 0.0);
    if (s.zero) forced_set_const<T>(s, 0.0);
    const int NV = s.nv;
    const T *tp = t.p<T>();
    const T *sp = s.p<T>();
    std::vector<T> out(3 * NV);
    reduce<T>(s.size, NV, 3,
              [&](uint64_t i, int k, T *v) {
                  T tv = tp[i * NV + k], sv = sp[i * NV + k];
                  v[0] = tv * sv;
                  v[1] = tv * tv;
                  v[2] = sv * sv;
              },
              out.data());
    for (int k = 0; k < NV; ++k) {
        phi.p<T>()[k] = out[k * 3 + 0];
        psi.p<T>()[k] = out[k * 3 + 1];
        theta.p<T>()[k] = out[k * 3 + 2];
    }
    phi.init = psi.init = theta.init = true;
    phi.zero = psi.zero = theta.zero = false;
}

// blas_merged_bicgstab.inl:149-194
template <typename T>
void merged_bicgstab_group4(Vec &s, Vec &t, Vec &r0, Vec &r, const Vec &omega, Vec &rho) {
    if (s.zero) forced_set_const<T>(s, 0.0);
    if (t.zero) forced_set_const<T>(t, 0.0);
    if (r0.zero) forced_set_const<T>(r0, 0.0);
    const int NV = s.nv;
    const T *sp = s.p<T>();
    const T *tp = t.p<T>();
    const T *r0p = r0.p<T>();
    T *rp = r.p<T>();
    const T *op = omega.p<T>();
    OR_PAR
    for (uint64_t i = 0; i < NV * s.size; i += NV)
        for (int k = 0; k < NV; ++k) rp[i + k] = sp[i + k] - op[k] * tp[i + k];
    reduce<T>(s.size, NV, 1,
              [&](uint64_t i, int k, T *v) { v[0] = rp[i * NV + k] * r0p[i * NV + k]; },
              rho.p<T>());
    r.zero = false;
    rho.zero = false;
    rho.init = true;
}

// blas_merged_bicgstab.inl:198-257
template <typename T>
void merged_bicgstab_group5(Vec &x, Vec &p, Vec &s, Vec &r, Vec &v, const Vec &alpha_conv,
                            const Vec &omega_conv, const Vec &alpha, const Vec &omega,
                            const Vec &beta) {
    (void)alpha;
    if (x.zero) set_const<T>(x, 0.0, true);
    if (p.zero) set_const<T>(p, 0.0, true);
    if (s.zero) forced_set_const<T>(s, 0.0);
    if (r.zero) forced_set_const<T>(r, 0.0);
    if (v.zero) forced_set_const<T>(v, 0.0);
    const int NV = s.nv;
    T *xp = x.p<T>();
    T *pp = p.p<T>();
    const T *sp = s.p<T>();
    const T *rp = r.p<T>();
    const T *vp = v.p<T>();
    const T *ac = alpha_conv.p<T>();
    const T *oc = omega_conv.p<T>();
    const T *bp = beta.p<T>();
    const T *op = omega.p<T>();
    std::vector<T> val(NV);
    for (int k = 0; k < NV; ++k) val[k] = bp[k] * op[k];
    OR_PAR
    for (uint64_t i = 0; i < NV * s.size; i += NV)
        for (int k = 0; k < NV; ++k) {
            xp[i + k] += ac[k] * pp[i + k] + oc[k] * sp[i + k];
            pp[i + k] = rp[i + k] + bp[k] * pp[i + k] - val[k] * vp[i + k];
        }
    x.zero = false;
    p.zero = false;
}

// blas_merged_jacobi.inl:32-90
// blas_merged_rbicgstab.inl:33-116: r = r - alpha v; theta = (t, r),
// phi = (t, t), psi = (t, r0), eta = (r, r)
template <typename T>
void merged_rbicgstab_group1(Vec &r, Vec &v, Vec &t, Vec &r0, const Vec &alpha, Vec &theta,
                             Vec &phi, Vec &psi, Vec &eta) {
    if (r.zero) set_const<T>(r, 0.0, true);
    if (v.zero) forced_set_const<T>(v, 0.0);
    if (t.zero) forced_set_const<T>(t, 0.0);
    if (r0.zero) forced_set_const<T>(r0, 0.0);
    const int NV = r.nv;
    T *rp = r.p<T>();
    const T *vp = v.p<T>(), *tp = t.p<T>(), *r0p = r0.p<T>(), *ap = alpha.p<T>();
    OR_PAR
    for (uint64_t i = 0; i < NV * r.size; i += NV)
        for (int k = 0; k < NV; ++k) rp[i + k] = rp[i + k] - ap[k] * vp[i + k];
    std::vector<T> out(4 * NV);
    reduce<T>(r.size, NV, 4,
              [&](uint64_t i, int k, T *o) {
                  const T tv = tp[i * NV + k], rv = rp[i * NV + k];
                  o[0] = tv * rv;
                  o[1] = tv * tv;
                  o[2] = tv * r0p[i * NV + k];
                  o[3] = rv * rv;
              },
              out.data());
    for (int k = 0; k < NV; ++k) {
        theta.p<T>()[k] = out[k * 4 + 0];
        phi.p<T>()[k] = out[k * 4 + 1];
        psi.p<T>()[k] = out[k * 4 + 2];
        eta.p<T>()[k] = out[k * 4 + 3];
    }
    for (Vec *w : {&theta, &phi, &psi, &eta}) {
        w->init = true;
        w->zero = false;
    }
    r.zero = false;
}

// blas_merged_rbicgstab.inl:120-193: x += alpha_conv v_ + omega_conv t_;
// z = t_ - omega z; v_ = z + beta v_ - beta omega s
template <typename T>
void merged_rbicgstab_group2(Vec &x, Vec &v_, Vec &t_, Vec &z, Vec &s, const Vec &alpha_conv,
                             const Vec &omega_conv, const Vec &omega, const Vec &beta) {
    if (x.zero) set_const<T>(x, 0.0, true);
    if (v_.zero) set_const<T>(v_, 0.0, true);
    if (t_.zero) forced_set_const<T>(t_, 0.0);
    if (z.zero) set_const<T>(z, 0.0, true);
    if (s.zero) forced_set_const<T>(s, 0.0);
    const int NV = x.nv;
    T *xp = x.p<T>(), *vp = v_.p<T>(), *zp = z.p<T>();
    const T *tp = t_.p<T>(), *sp = s.p<T>();
    const T *ac = alpha_conv.p<T>(), *oc = omega_conv.p<T>(), *om = omega.p<T>(),
            *be = beta.p<T>();
    OR_PAR
    for (uint64_t i = 0; i < NV * x.size; i += NV)
        for (int k = 0; k < NV; ++k) {
            xp[i + k] += ac[k] * vp[i + k] + oc[k] * tp[i + k];
            zp[i + k] = tp[i + k] - om[k] * zp[i + k];
            vp[i + k] = zp[i + k] + be[k] * vp[i + k] - be[k] * om[k] * sp[i + k];
        }
    x.zero = z.zero = v_.zero = false;
}

template <typename T>
void merged_jacobi(Vec &x, const Vec &b, const Vec &inv_diag, Vec &r, const Vec &relax) {
    if (x.empty()) {
        x.init = true;
        x.zero = false;
        return;
    }
    const int NV = x.nv;
    T *xp = x.p<T>();
    const T *bp = b.p<T>();
    const T *dp = inv_diag.p<T>();
    const T *rp = r.p<T>();
    const T *wp = relax.p<T>();
    if (x.zero && r.zero) {
        OR_PAR
        for (uint64_t i = 0; i < x.size; i++)
            for (int k = 0; k < NV; ++k) xp[i * NV + k] = wp[k] * dp[i] * bp[i * NV + k];
    } else {
        if (x.zero) forced_set_const<T>(x, 0.0);
        if (r.zero) forced_set_const<T>(r, 0.0);
        rp = r.p<T>();
        OR_PAR
        for (uint64_t i = 0; i < x.size; i++)
            for (int k = 0; k < NV; ++k)
                xp[i * NV + k] += wp[k] * dp[i] * (bp[i * NV + k] - rp[i * NV + k]);
    }
    x.init = true;
    x.zero = false;
}

}  // namespace blas

// ----------------------------------------------------------------------------
// CSR block: csr_matrix.h:47-86 (row pointer, column, value, optional
// row/column index maps after compress()).
// ----------------------------------------------------------------------------
struct Csr {
    uint64_t nrows = 0, ncols = 0, block_nrows = 0, block_ncols = 0, nonzeros = 0;
    uint64_t block_row_offset = 0, block_col_offset = 0;
    bool f32 = false;
    bool indexed = false;
    std::vector<uint32_t> row, col, row_ind, col_ind;
    std::vector<double> vd;
    std::vector<float> vf;
    bool empty() const { return nonzeros == 0; }
    template <typename T>
    const T *val() const;
};
template <>
const double *Csr::val<double>() const { return vd.data(); }
template <>
const float *Csr::val<float>() const { return vf.data(); }

static Csr to_f32(const Csr &a) {
    Csr b = a;
    b.f32 = true;
    b.vf.resize(a.vd.size());
    for (size_t i = 0; i < a.vd.size(); ++i) b.vf[i] = (float)a.vd[i];
    b.vd.clear();
    return b;
}

// B200 extension gpu_level_bf16: a float level operator whose values are
// stored in BF16. Each float value is rounded to the nearest BF16 (ties to
// even: add 0x7FFF plus the lowest kept bit, then drop the low 16 bits; NaN
// stays NaN) and used as that float.
static float round_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) {
        u |= 0x00400000u;  // quiet NaN
    } else {
        u += 0x7FFFu + ((u >> 16) & 1u);
    }
    u &= 0xFFFF0000u;
    std::memcpy(&f, &u, 4);
    return f;
}

static Csr to_bf16_values(const Csr &a) {
    Csr b = a;
    for (float &v : b.vf) v = round_bf16(v);
    return b;
}

// B200 extension gpu_level_fp16 = 1: the same levels store FP16 values
// instead, each float value divided by the level's power-of-two scale s
// (2^(E - 15) for the largest magnitude m * 2^E, m in [0.5, 1), but at
// least 2^-126; 1 for an all-zero level), rounded to the nearest FP16 (ties to even, IEEE
// binary16 through the compiler's _Float16) and read back as h * s; the
// division and the product by s are exact.
static Csr to_fp16_values(const Csr &a) {
    Csr b = a;
    float mx = 0.0f;
    for (float v : b.vf) mx = std::max(mx, std::fabs(v));
    float s = 1.0f;
    if (mx > 0.0f && std::isfinite(mx)) {
        int E = 0;
        std::frexp(mx, &E);
        s = std::ldexp(1.0f, std::max(E - 15, -126));
    }
    for (float &v : b.vf) v = (float)(_Float16)(v / s) * s;
    return b;
}

// csr_matrix.inl:86-170
static void compress(Csr &m) {
    if (m.empty()) return;
    uint64_t non_empty_rows = 0;
    for (uint64_t i = 0; i < m.nrows; ++i)
        if (m.row[i + 1] - m.row[i]) ++non_empty_rows;
    m.row_ind.assign(non_empty_rows, 0);
    non_empty_rows = 0;
    for (uint64_t i = 0; i < m.nrows; ++i)
        if (m.row[i + 1] - m.row[i]) m.row_ind[non_empty_rows++] = (uint32_t)i;

    std::vector<uint64_t> col_label(m.block_ncols, 0);
    for (uint64_t i = 0; i < m.nonzeros; ++i) col_label[m.col[i]] = 1;
    uint64_t non_empty_cols = 0;
    for (uint64_t i = 0; i < m.block_ncols; ++i)
        if (col_label[i]) ++non_empty_cols;
    m.col_ind.assign(non_empty_cols, 0);
    non_empty_cols = 0;
    for (uint64_t i = 0; i < m.block_ncols; ++i)
        if (col_label[i]) {
            m.col_ind[non_empty_cols] = (uint32_t)i;
            col_label[i] = non_empty_cols;
            ++non_empty_cols;
        }

    non_empty_rows = 0;
    for (uint64_t i = 0; i < m.nrows; ++i) {
        if (m.row[i + 1] != m.row[non_empty_rows]) {
            m.row[non_empty_rows + 1] = m.row[i + 1];
            ++non_empty_rows;
        }
    }
    m.nrows = non_empty_rows;
    m.row.resize(m.nrows + 1);
    for (uint64_t i = 0; i < m.nonzeros; ++i) m.col[i] = (uint32_t)col_label[m.col[i]];
    m.ncols = non_empty_cols;
    m.indexed = true;
}

// misc.h:34-44
static uint32_t search_range(uint64_t col, const std::vector<uint64_t> &range) {
    uint32_t val = (uint32_t)range.size() - 1;
    while ((col < range[val]) && (val > 0)) --val;
    return val;
}

// csr_matrix_segment.inl:107-229 (returns (chunk, block id) pairs)
static std::vector<std::pair<Csr, uint32_t>> split_by_columns(
    const Csr &mat, const std::vector<uint64_t> &block_size, const std::vector<uint64_t> &block_indx) {
    std::vector<std::pair<Csr, uint32_t>> chunks;
    if (mat.empty()) return chunks;
    const uint32_t nblocks = (uint32_t)block_size.size();
    std::vector<uint32_t> col_to_block(mat.nonzeros, 0);
    std::vector<uint64_t> nnz_per_block(nblocks, 0);
    for (uint64_t j = 0; j < mat.nonzeros; ++j) {
        col_to_block[j] = search_range(mat.col[j], block_indx);
        nnz_per_block[col_to_block[j]]++;
    }
    std::vector<uint64_t> map(nblocks, 0);
    uint32_t ne = 0;
    for (uint32_t i = 0; i < nblocks; ++i)
        if (nnz_per_block[i]) map[i] = ne++;
    for (auto &c : col_to_block) c = (uint32_t)map[c];
    chunks.resize(ne);
    uint32_t nb = 0;
    for (uint32_t rnb = 0; rnb < nblocks; ++rnb) {
        if (!nnz_per_block[rnb]) continue;
        Csr &c = chunks[nb].first;
        chunks[nb].second = rnb;
        c.nrows = mat.nrows;
        c.ncols = block_size[rnb];
        c.block_nrows = c.nrows;
        c.block_ncols = c.ncols;
        c.block_row_offset = mat.block_row_offset;
        c.block_col_offset = block_indx[rnb];
        c.nonzeros = nnz_per_block[rnb];
        c.f32 = mat.f32;
        c.row.assign(c.nrows + 1, 0);
        c.col.assign(c.nonzeros, 0);
        if (mat.f32)
            c.vf.assign(c.nonzeros, 0.0f);
        else
            c.vd.assign(c.nonzeros, 0.0);
        ++nb;
    }
    for (uint64_t i = 0; i < mat.nrows; ++i) {
        for (nb = 0; nb < ne; ++nb) chunks[nb].first.row[i + 1] = chunks[nb].first.row[i];
        for (uint64_t j = mat.row[i]; j < mat.row[i + 1]; ++j) {
            nb = col_to_block[j];
            Csr &c = chunks[nb].first;
            uint64_t indx = c.row[i + 1];
            c.col[indx] = (uint32_t)(mat.col[j] - c.block_col_offset);
            if (mat.f32)
                c.vf[indx] = mat.vf[j];
            else
                c.vd[indx] = mat.vd[j];
            ++c.row[i + 1];
        }
    }
    for (auto &c : chunks) c.first.block_col_offset += mat.block_col_offset;
    return chunks;
}

// transpose.inl:31-108 (non-indexed case)
static Csr transpose(const Csr &m) {
    Csr t;
    t.nrows = m.ncols;
    t.ncols = m.nrows;
    t.nonzeros = m.nonzeros;
    t.block_nrows = m.block_ncols;
    t.block_ncols = m.block_nrows;
    t.f32 = m.f32;
    std::vector<uint32_t> per_col(m.ncols, 0);
    for (uint64_t j = 0; j < m.nonzeros; ++j) ++per_col[m.col[j]];
    t.row.assign(t.nrows + 1, 0);
    for (uint64_t l = 0; l < t.nrows; ++l) {
        t.row[l + 1] = t.row[l] + per_col[l];
        per_col[l] = 0;
    }
    t.col.assign(t.nonzeros, 0);
    if (m.f32)
        t.vf.assign(t.nonzeros, 0.0f);
    else
        t.vd.assign(t.nonzeros, 0.0);
    for (uint64_t l = 0; l < m.nrows; ++l)
        for (uint64_t j = m.row[l]; j < m.row[l + 1]; ++j) {
            uint32_t rt = m.col[j];
            uint64_t pos = t.row[rt] + per_col[rt];
            t.col[pos] = (uint32_t)l;
            if (m.f32)
                t.vf[pos] = m.vf[j];
            else
                t.vd[pos] = m.vd[j];
            ++per_col[rt];
        }
    return t;
}

// csr_matrix.h:302-334 and 336-368: 1/a_ii computed in double, stored in F
template <typename T>
static std::vector<T> inv_diag(const Csr &m, bool sqrt_) {
    std::vector<T> d(m.nrows, T(0));
    const T *v = m.val<T>();
    for (uint64_t i = 0; i < m.nrows; ++i)
        for (uint64_t j = m.row[i]; j < m.row[i + 1]; ++j)
            if ((uint64_t)m.col[j] == i) d[i] = sqrt_ ? (T)std::sqrt(1.0 / v[j]) : (T)(1.0 / v[j]);
    return d;
}

// inverse.inl:31-106: Gauss-Jordan on [A | I] without pivoting, in type T
template <typename T>
static std::vector<T> gauss_jordan_inverse(const std::vector<T> &a, uint64_t n) {
    const uint64_t nc = 2 * n;
    std::vector<T> e(n * nc, T(0));
    for (uint64_t i = 0; i < n; ++i) {
        e[i * nc + i + n] = 1.0;
        for (uint64_t j = 0; j < n; ++j) e[i * nc + j] = a[i * n + j];
    }
    for (uint64_t i = 0; i < n; ++i) {
        T *ri = &e[i * nc];
        for (uint64_t k = nc - 1; k > i; --k) ri[k] /= ri[i];
        ri[i] = 1.0;
        for (uint64_t j = i + 1; j < n; ++j) {
            T *rj = &e[j * nc];
            for (uint64_t k = nc - 1; k > i; --k) rj[k] -= rj[i] * ri[k];
            rj[i] = 0.0;
        }
    }
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t row = n - 1 - i;
        T *ri = &e[row * nc];
        for (uint64_t j = 0; j < row; ++j) {
            T *rj = &e[j * nc];
            for (uint64_t k = nc / 2; k < nc; ++k) rj[k] -= rj[row] * ri[k];
            rj[row] = 0.0;
        }
    }
    std::vector<T> inv(n * n);
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = 0; j < n; ++j) inv[i * n + j] = e[i * nc + n + j];
    return inv;
}

template <typename T>
static std::vector<T> csr_to_dense(const Csr &m) {
    std::vector<T> a(m.nrows * m.ncols, T(0));
    const T *v = m.val<T>();
    for (uint64_t i = 0; i < m.nrows; ++i)
        for (uint64_t j = m.row[i]; j < m.row[i + 1]; ++j) a[i * m.ncols + m.col[j]] = v[j];
    return a;
}

// ----------------------------------------------------------------------------
// BLAS2: csr_matvec.inl:32-260, csr_gs.inl:32-134, dense_matvec.inl:71-121
// ----------------------------------------------------------------------------
namespace blas2 {

// csr_matvec.inl:148-260 (x.if_zero => y = 0 via set_const, as in :156-159)
template <typename T>
void csr_Ax_y(const Csr &m, const Vec &x, Vec &y) {
    if (x.zero) {
        blas::set_const<T>(y, 0.0, true);
        return;
    }
    if (m.empty()) {
        y.init = true;
        y.zero = false;
        return;
    }
    const int NV = y.nv;
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    const T *v = m.val<T>();
    // rows are independent (each is summed sequentially by one thread), so
    // the threads change no result
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m.nrows; ++i) {
        uint64_t rs = (m.indexed ? m.row_ind[i] : i) * NV;
        for (int k = 0; k < NV; ++k) yp[rs + k] = 0.0;
        for (uint64_t j = m.row[i]; j < m.row[i + 1]; ++j) {
            uint64_t cs = (uint64_t)m.col[j] * NV;
            for (int k = 0; k < NV; ++k) yp[rs + k] += xp[cs + k] * v[j];
        }
    }
    y.init = true;
    y.zero = false;
}

// csr_matvec.inl:32-144 (accumulates directly into y)
template <typename T>
void csr_Axpy(const Csr &m, const Vec &x, Vec &y, uint64_t m_offset = 0) {
    if (x.zero) return;
    if (m.empty()) {
        y.zero = false;
        return;
    }
    const int NV = y.nv;
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    const T *v = m.val<T>();
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m.nrows; ++i) {
        uint64_t rs = ((m.indexed ? m.row_ind[i] : i) + m_offset) * NV;
        for (uint64_t j = m.row[i]; j < m.row[i + 1]; ++j) {
            uint64_t cs = (uint64_t)m.col[j] * NV;
            for (int k = 0; k < NV; ++k) yp[rs + k] += xp[cs + k] * v[j];
        }
    }
    y.zero = false;
}

// blas2.h:305-326: the zero flag short-circuit above the backend
template <typename T>
void Ax_y(const Csr &m, const Vec &x, Vec &y) {
    if (x.zero) {
        y.zero = true;
        return;
    }
    csr_Ax_y<T>(m, x, y);
}

template <typename T>
void Axpy(const Csr &m, const Vec &x, Vec &y) {
    if (x.zero) return;
    csr_Axpy<T>(m, x, y);
}

// dense_matvec.inl:71-121
template <typename T>
void dense_Ax_y(const std::vector<T> &a, uint64_t n, const Vec &x, Vec &y) {
    if (x.zero) {
        y.zero = true;  // blas2.h:310-312 short-circuit above Ax_y_slice
        return;
    }
    const int NV = y.nv;
    const T *xp = x.p<T>();
    T *yp = y.p<T>();
    OR_PAR
    for (uint64_t i = 0; i < n; ++i) {
        for (int k = 0; k < NV; ++k) yp[i * NV + k] = 0.0;
        for (uint64_t j = 0; j < n; ++j)
            for (int k = 0; k < NV; ++k) yp[i * NV + k] += a[i * n + j] * xp[j * NV + k];
    }
    y.init = true;
    y.zero = false;
}

}  // namespace blas2

// ----------------------------------------------------------------------------
// Core layer for HSGS: matrix.inl:382-420 with split_by_columns over the core
// partition and compress() on the off-core chunks.
// ----------------------------------------------------------------------------
struct CoreLayer {
    int ncores = 1;
    std::vector<uint64_t> off, size;
    std::vector<Csr> diag;                                // per core: local columns
    std::vector<std::vector<std::pair<Csr, uint32_t>>> offd;  // per core: compressed chunks
};

static CoreLayer build_core_layer(const Csr &A, int ncores) {
    CoreLayer L;
    L.ncores = ncores;
    L.off.resize(ncores);
    L.size.resize(ncores);
    std::vector<uint64_t> bsize(ncores), bindx(ncores + 1, 0);
    for (int c = 0; c < ncores; ++c) {
        core_range(A.nrows, ncores, c, L.off[c], L.size[c]);
        bsize[c] = L.size[c];
        bindx[c + 1] = bindx[c] + bsize[c];
    }
    L.diag.resize(ncores);
    L.offd.resize(ncores);
    for (int c = 0; c < ncores; ++c) {
        // disassemble rows [off, off+size) (matrix.h:95-127)
        Csr s;
        s.nrows = L.size[c];
        s.block_nrows = L.size[c];
        s.ncols = A.ncols;
        s.block_ncols = A.ncols;
        s.block_row_offset = L.off[c];
        s.f32 = A.f32;
        s.row.assign(s.nrows + 1, 0);
        for (uint64_t i = 0; i < s.nrows; ++i) {
            uint64_t gi = L.off[c] + i;
            for (uint64_t j = A.row[gi]; j < A.row[gi + 1]; ++j) {
                s.col.push_back(A.col[j]);
                if (A.f32)
                    s.vf.push_back(A.vf[j]);
                else
                    s.vd.push_back(A.vd[j]);
            }
            s.row[i + 1] = (uint32_t)s.col.size();
        }
        s.nonzeros = s.col.size();
        auto chunks = split_by_columns(s, bsize, bindx);
        for (auto &ch : chunks) {
            if (ch.second == (uint32_t)c) {
                L.diag[c] = ch.first;
            } else {
                compress(ch.first);
                L.offd[c].push_back(ch);
            }
        }
    }
    return L;
}

// ----------------------------------------------------------------------------
// Solvers: solver.h:121-312 and solvers/detail/*.inl
// ----------------------------------------------------------------------------
struct Params {
    // role -> key -> value; per-level overrides role -> level -> key -> value
    std::map<std::string, std::map<std::string, std::string>> base;
    std::map<std::string, std::map<int, std::map<std::string, std::string>>> lev;
    std::string get(const std::string &role, const std::string &key, int level = -1,
                    const std::string &def = "") const {
        if (level >= 0) {
            auto r = lev.find(role);
            if (r != lev.end()) {
                auto l = r->second.find(level);
                if (l != r->second.end()) {
                    auto k = l->second.find(key);
                    if (k != l->second.end()) return k->second;
                }
            }
        }
        auto r = base.find(role);
        if (r != base.end()) {
            auto k = r->second.find(key);
            if (k != r->second.end()) return k->second;
        }
        return def;
    }
    bool has(const std::string &role) const { return base.count(role) > 0; }
};

// xamg_params_details.h:146-236 (family defaults; list name = role)
struct SolverParams {
    std::string method;
    int convergence_check = 0, convergence_info = 0, max_iters = 1;
    float abs_tol = 0.f, rel_tol = 0.f, relax = 0.99f, spec_fraction = 0.3f;
    int poly_order = 2, mg_cycle = 0;
};

static SolverParams resolve(const Params &P, const std::string &role, int level) {
    SolverParams s;
    s.method = P.get(role, "method", level);
    auto geti = [&](const char *k, int d) {
        std::string v = P.get(role, k, level);
        return v.empty() ? d : (int)std::stol(v);
    };
    auto getf = [&](const char *k, float d) {
        std::string v = P.get(role, k, level);
        return v.empty() ? d : (float)std::stod(v);
    };
    const std::string &f = s.method;
    bool solver = (role == "solver");
    if (f == "Identity" || f == "Direct") return s;
    if (f == "Chebyshev") {
        s.convergence_check = geti("convergence_check", 0);
        s.convergence_info = geti("convergence_info", 0);
        s.poly_order = geti("polynomial_order", 2);
        s.spec_fraction = getf("spectrum_fraction", 0.3f);
        return s;
    }
    int iters = 0;
    float abs_tol = 0.f, rel_tol = 0.f;
    if (solver) {
        abs_tol = 1.e-8f;
        rel_tol = 1.e-8f;
        s.convergence_check = geti("convergence_check", 1);
    } else {
        s.convergence_check = geti("convergence_check", 0);
    }
    s.convergence_info = geti("convergence_info", 0);
    if (f == "Jacobi" || f == "HSGS") {
        iters = solver ? 100 : 2;
        s.relax = getf("relax_factor", 0.99f);
    } else if (f == "MultiGrid") {
        iters = solver ? 30 : 1;
        s.mg_cycle = geti("mg_cycle", 0);
    } else {
        iters = solver ? 50 : 1;
    }
    s.abs_tol = getf("abs_tolerance", abs_tol);
    s.rel_tol = getf("rel_tolerance", rel_tol);
    s.max_iters = geti("max_iters", iters);
    return s;
}

struct Level {
    Csr A;                    // in the level's working precision
    Csr Abf;                  // A with BF16-rounded values (gpu_level_bf16), else empty
    bool bf16 = false;        // the cycle's and smoothers' SpMVs use Abf
    Csr R, P;                 // transfer to level+1 (absent on the coarsest level)
    double min_eig = NAN, max_eig = NAN;
    bool reduced = false;     // working precision is float
};

struct Stats {
    std::vector<int> conv;
    std::vector<double> abs_res, rel_res;
    int iters = 0;
};

struct Solver {
    std::string method;
    SolverParams sp;
    const Csr *A = nullptr;
    bool f32 = false;
    int NV = 1;
    Stats st;
    // smoother data: inverse diagonal and inverse square-root diagonal (nv = 1)
    Vec id, isd;
    std::shared_ptr<CoreLayer> core;
    // Direct: dense inverse of the coarse matrix
    std::vector<double> d_inv;
    std::vector<float> f_inv;
    double min_eig = NAN, max_eig = NAN;
    // solver-owned work vectors (buffer_nvecs of solver.h:152-165)
    std::vector<Vec> buf;
    // MultiGrid
    std::vector<Level> *levels = nullptr;
    std::vector<std::shared_ptr<Solver>> pre, post;
    std::shared_ptr<Solver> coarse;
    std::shared_ptr<Solver> precond;
    std::vector<std::vector<Vec>> mgbuf;  // per level buffers (mg.inl:136-163)
    Vec mg_b32, mg_x32;                   // float input/output (gpu_precond_f32 = 1)
};

template <typename T>
static void print_residuals(int iter, const Vec &res, const Vec &res0, const Vec &conv) {
    printf("%7d | ", iter);
    for (int k = 0; k < res.nv; ++k) {
        if (conv.p<T>()[k] != 0)
            printf("%12e | %12e | ", std::sqrt((double)res.p<T>()[k]),
                   std::sqrt((double)(res.p<T>()[k] / res0.p<T>()[k])));
        else
            printf("%12s | %12s | ", "-", "-");
    }
    printf("\n");
}

// solver.h:173-203
template <typename T>
static bool convergence_check(Solver &S, const Vec &res, const Vec &res0, const Vec &conv) {
    float abs_tol = S.sp.abs_tol, rel_tol = S.sp.rel_tol;
    bool flag = true;
    for (int k = 0; k < res.nv; ++k) {
        if (conv.p<T>()[k] != 0) {
            T abs_res = std::sqrt(res.p<T>()[k]);
            T rel_res = abs_res / std::sqrt(res0.p<T>()[k]);
            if ((abs_res > abs_tol) && (rel_res > rel_tol)) {
                flag = false;
            } else if (!S.st.conv[k]) {
                S.st.abs_res[k] = abs_res;
                S.st.rel_res[k] = rel_res;
                S.st.conv[k] = 1;
            }
        }
    }
    return flag;
}

// solver.h:205-241
template <typename T>
static bool converged(Solver &S, const Vec &res, const Vec &res0, Vec &conv) {
    if (S.sp.convergence_check) {
        if (S.sp.convergence_info) print_residuals<T>(S.st.iters, res, res0, conv);
        if (convergence_check<T>(S, res, res0, conv)) return true;
        for (int k = 0; k < conv.nv; ++k) conv.p<T>()[k] *= (T)(!S.st.conv[k]);
        conv.init = true;
        conv.zero = false;
    }
    return false;
}

static void reset_stats(Solver &S) {
    S.st.iters = 0;
    if (S.sp.convergence_check) {
        S.st.conv.assign(S.NV, 0);
        S.st.abs_res.assign(S.NV, 0.0);
        S.st.rel_res.assign(S.NV, 0.0);
    } else {
        S.st.conv.resize(S.NV, 0);
        S.st.abs_res.resize(S.NV, 0.0);
        S.st.rel_res.resize(S.NV, 0.0);
    }
}

template <typename T>
static void get_residual(Solver &S, const Vec &x, const Vec &b, Vec &r, Vec &res, bool norm) {
    // solver.h:243-256
    blas2::Ax_y<T>(*S.A, x, r);
    blas::axpby_s<T>(1.0, b, -1.0, r);
    if (norm) blas::dot<T>(r, r, res);
}

template <typename T>
static void solve(Solver &S, Vec &x, Vec &b, const Vec &conv);


template <typename T>
static Vec make_vec(uint64_t n, int nv) {
    Vec v;
    v.alloc(n, nv, sizeof(T) == 4);
    return v;
}

template <typename T>
static Vec diag_vec(const Csr &A, bool sqrt_) {
    std::vector<T> d = inv_diag<T>(A, sqrt_);
    Vec v = make_vec<T>(A.nrows, 1);
    std::copy(d.begin(), d.end(), v.p<T>());
    v.init = true;
    v.zero = false;
    return v;
}

// jacobi.inl:49-120
template <typename T>
static void solve_jacobi(Solver &S, Vec &x, Vec &b, const Vec &conv) {
    const int NV = S.NV;
    reset_stats(S);
    Vec iconv = conv;
    Vec a1 = typed_scalar<T>(NV, 1.0);
    Vec relax = make_vec<T>(1, NV);
    blas::set_const<T>(relax, (double)S.sp.relax);
    for (auto &v : S.buf) blas::set_const<T>(v, 0.0);
    Vec &r = S.buf[0];
    Vec rho0 = make_vec<T>(1, NV), res = make_vec<T>(1, NV);
    int &it = S.st.iters;
    if (S.sp.convergence_check) {
        get_residual<T>(S, x, b, r, rho0, true);
        if (converged<T>(S, rho0, rho0, iconv)) return;
        do {
            ++it;
            blas::scal<T>(S.id, r);
            blas::scal<T>(iconv, relax);
            blas::axpby<T>(relax, r, a1, x);
            get_residual<T>(S, x, b, r, res, true);
            if (converged<T>(S, res, rho0, iconv)) return;
        } while (it < S.sp.max_iters);
    } else {
        do {
            ++it;
            blas2::Ax_y<T>(*S.A, x, r);
            blas::merged_jacobi<T>(x, b, S.id, r, relax);
        } while (it < S.sp.max_iters);
    }
}

// blas2.h:184-281 with csr_gs.inl:32-134 for each core block
template <typename T>
static void sgs(Solver &S, const Vec &b, Vec &x, Vec &t, const Vec &relax) {
    const int NV = S.NV;
    CoreLayer &L = *S.core;
    blas::set_const<T>(t, 0.0, true);
    // lagged off-core part: every core gathers the x values its compressed
    // off-core chunks reference, then accumulates them into t
    const T *xp = x.zero ? nullptr : x.p<T>();
    for (int c = 0; c < L.ncores; ++c) {
        for (auto &ch : L.offd[c]) {
            const Csr &m = ch.first;
            Vec recv = make_vec<T>(m.ncols, NV);
            if (!x.zero) {
                for (uint64_t q = 0; q < m.ncols; ++q)
                    for (int k = 0; k < NV; ++k)
                        recv.p<T>()[q * NV + k] = xp[(m.col_ind[q] + m.block_col_offset) * NV + k];
                recv.zero = false;
            }
            recv.init = true;
            blas2::csr_Axpy<T>(m, recv, t, L.off[c]);
        }
    }
    blas::axpby_s<T>(1.0, b, -1.0, t);
    if (x.zero) blas::set_const<T>(x, 0.0, true);
    T *X = x.p<T>();
    const T *tp = t.p<T>();
    const T *dp = S.id.p<T>();
    const T *wp = relax.p<T>();
    // a core block reads and writes only its own rows of x (the off-core
    // terms are in t), so the blocks run on the host threads independently
#pragma omp parallel for schedule(static)
    for (int c = 0; c < L.ncores; ++c) {
        std::vector<T> sum(NV), coeff(NV);
        const Csr &m = L.diag[c];
        if (m.empty()) {
            continue;
        }
        const uint64_t off = L.off[c];
        const T *v = m.val<T>();
        auto row_update = [&](uint64_t i) {
            uint64_t rs = (i + off) * NV;
            for (int k = 0; k < NV; ++k) sum[k] = tp[rs + k];
            for (uint64_t j = m.row[i]; j < m.row[i + 1]; ++j) {
                uint64_t cs = (m.col[j] + off) * NV;
                for (int k = 0; k < NV; ++k) sum[k] -= X[cs + k] * v[j];
            }
            for (int k = 0; k < NV; ++k) coeff[k] = wp[k] * dp[i + off];
            for (int k = 0; k < NV; ++k) X[rs + k] += coeff[k] * sum[k];
        };
        for (uint64_t i = 0; i < m.nrows; ++i) row_update(i);
        for (uint64_t ii = 0; ii < m.nrows; ++ii) row_update(m.nrows - 1 - ii);
    }
    x.zero = false;
}

// hsgs.inl:50-115
template <typename T>
static void solve_hsgs(Solver &S, Vec &x, Vec &b, const Vec &conv) {
    const int NV = S.NV;
    reset_stats(S);
    Vec iconv = conv;
    Vec relax = make_vec<T>(1, NV);
    blas::set_const<T>(relax, (double)S.sp.relax);
    for (auto &v : S.buf) blas::set_const<T>(v, 0.0);
    Vec &r = S.buf[0];
    Vec &t = S.buf[1];
    Vec rho0 = make_vec<T>(1, NV), res = make_vec<T>(1, NV);
    int &it = S.st.iters;
    if (S.sp.convergence_check) {
        get_residual<T>(S, x, b, r, rho0, true);
        if (converged<T>(S, rho0, rho0, iconv)) return;
    }
    do {
        ++it;
        blas::scal<T>(iconv, relax);
        sgs<T>(S, b, x, t, relax);
        if (S.sp.convergence_check) {
            get_residual<T>(S, x, b, r, res, true);
            if (converged<T>(S, res, rho0, iconv)) return;
        }
    } while (it < S.sp.max_iters);
}

// chebyshev.inl:50-127 (coefficients in double, stored in F)
static std::vector<double> cheby_coeffs(double min_eig, double max_eig, int order, double frac) {
    double upper = max_eig * 1.1;
    double lower = (upper - min_eig) * frac + min_eig;
    double theta = (upper + lower) / 2.;
    double delta = (upper - lower) / 2.;
    std::vector<double> c(order);
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

// chebyshev.inl:129-206
template <typename T>
static void solve_chebyshev(Solver &S, Vec &x, Vec &b, const Vec &conv) {
    const int NV = S.NV;
    reset_stats(S);
    Vec a1 = typed_scalar<T>(NV, 1.0);
    for (auto &v : S.buf) blas::set_const<T>(v, 0.0);
    Vec &r = S.buf[0];
    Vec &t1 = S.buf[1];
    Vec &t2 = S.buf[2];
    Vec rho0 = make_vec<T>(1, NV), res = make_vec<T>(1, NV);
    const int order = S.sp.poly_order;
    std::vector<double> cd = cheby_coeffs(S.min_eig, S.max_eig, order, (double)S.sp.spec_fraction);
    std::vector<Vec> c;
    for (int i = 0; i < order; ++i) {
        Vec v = make_vec<T>(1, NV);
        blas::set_const<T>(v, (double)(T)cd[i]);
        v.init = true;
        v.zero = false;
        c.push_back(v);
    }
    get_residual<T>(S, x, b, r, rho0, S.sp.convergence_check != 0);
    if (S.sp.convergence_check && S.sp.convergence_info) print_residuals<T>(0, rho0, rho0, conv);
    blas::scal<T>(S.isd, r);
    blas::ax_y<T>(c[order - 1], r, t1);
    for (int i = order - 2; i >= 0; i--) {
        blas::scal<T>(S.isd, t1);
        blas2::Ax_y<T>(*S.A, t1, t2);
        blas::scal<T>(S.isd, t2);
        blas::axpby_z<T>(c[i], r, a1, t2, t1);
    }
    blas::scal<T>(S.isd, t1);
    blas::axpby<T>(a1, t1, a1, x);
    if (S.sp.convergence_check && S.sp.convergence_info) {
        get_residual<T>(S, x, b, r, res, true);
        print_residuals<T>(0, res, rho0, conv);
    }
}

// direct.inl:49-56
static const std::vector<double> &inverse_of(const Solver &S, double *) { return S.d_inv; }
static const std::vector<float> &inverse_of(const Solver &S, float *) { return S.f_inv; }

template <typename T>
static void solve_direct(Solver &S, Vec &x, Vec &b, const Vec &) {
    blas2::dense_Ax_y<T>(inverse_of(S, (T *)nullptr), S.A->nrows, b, x);
}

template <typename T>
static void convert_vec(const Vec &src, Vec &dst) {
    // vector/operations/convert.inl:31-83
    dst.zero = src.zero;
    if (src.zero) {
        dst.init = true;
        return;
    }
    const uint64_t m = (uint64_t)src.size * src.nv;
    if (src.f32 && !dst.f32) {
        OR_PAR
        for (uint64_t i = 0; i < m; ++i) dst.d[i] = (double)src.f[i];
    } else if (!src.f32 && dst.f32) {
        OR_PAR
        for (uint64_t i = 0; i < m; ++i) dst.f[i] = (float)src.d[i];
    }
    else if (src.f32)
        dst.f = src.f;
    else
        dst.d = src.d;
    dst.init = true;
}

// mg.inl:166-260
template <typename T1, typename T2>
static void mg_cycle(Solver &S, Vec &x, Vec &b, int level, int cycle, const Vec &iconv) {
    std::vector<Level> &L = *S.levels;
    const int NV = S.NV;
    Vec a1 = typed_scalar<T1>(NV, 1.0), a_1 = typed_scalar<T1>(NV, -1.0);
    Vec iconv2 = make_vec<T2>(1, NV);
    Csr &A = L[level].bf16 ? L[level].Abf : L[level].A;
    Csr &R = L[level].R;
    Csr &P = L[level].P;
    Vec &temp = S.mgbuf[level][0];
    Vec &b_H = S.mgbuf[level + 1][1];
    Vec &x_H = S.mgbuf[level + 1][2];
    if (cycle != 1) solve<T1>(*S.pre[level], x, b, iconv);
    blas2::Ax_y<T1>(A, x, temp);
    blas::axpby<T1>(a1, b, a_1, temp);
    const bool mixed = (sizeof(T1) != sizeof(T2));
    if (mixed) {
        Vec &temp32 = S.mgbuf[level][1];
        convert_vec<T1>(temp, temp32);
        blas2::Ax_y<T2>(R, temp32, b_H);
        convert_vec<T1>(iconv, iconv2);
    } else {
        blas2::Ax_y<T2>(R, temp, b_H);
        iconv2 = iconv;
    }
    blas::set_const<T2>(x_H, 0.0);
    if (level + 1 == (int)L.size() - 1) {
        solve<T2>(*S.coarse, x_H, b_H, iconv2);
    } else {
        mg_cycle<T2, T2>(S, x_H, b_H, level + 1, cycle, iconv2);
        if (cycle == 2)
            mg_cycle<T2, T2>(S, x_H, b_H, level + 1, 2, iconv2);
        else if (cycle == 1)
            mg_cycle<T2, T2>(S, x_H, b_H, level + 1, 0, iconv2);
    }
    if (mixed) {
        Vec &temp32 = S.mgbuf[level][1];
        blas2::Ax_y<T2>(P, x_H, temp32);
        convert_vec<T2>(temp32, temp);
        blas::axpby<T1>(a1, temp, a1, x);
    } else {
        blas2::Axpy<T1>(P, x_H, x);
    }
    solve<T1>(*S.post[level], x, b, iconv);
}

// mg.inl:262-334 (F is double)
static void solve_mg(Solver &S, Vec &x, Vec &b, const Vec &conv) {
    const int NV = S.NV;
    reset_stats(S);
    Vec iconv = conv;
    for (auto &v : S.buf) blas::set_const<double>(v, 0.0);
    Vec &r = S.buf[0];
    Vec rho0 = make_vec<double>(1, NV), res = make_vec<double>(1, NV);
    int &it = S.st.iters;
    if (S.sp.convergence_check) {
        get_residual<double>(S, x, b, r, rho0, true);
        if (converged<double>(S, rho0, rho0, iconv)) return;
    }
    const bool reduced = (*S.levels)[1].reduced;
    if ((*S.levels)[0].reduced) {
        // B200 extension (gpu_precond_f32 = 1, preconditioner only): every
        // level in float, the input converted on entry and the result on exit
        // the float copies persist between applications, as the B200
        // library's do (an F-cycle's prolongation reads x32's old contents)
        const uint64_t n = (*S.levels)[0].A.nrows;
        if (S.mg_b32.size != n) {
            S.mg_b32 = make_vec<float>(n, NV);
            S.mg_x32 = make_vec<float>(n, NV);
        }
        Vec &b32 = S.mg_b32, &x32 = S.mg_x32;
        Vec ic32 = make_vec<float>(1, NV);
        convert_vec<double>(b, b32);
        convert_vec<double>(x, x32);
        convert_vec<double>(iconv, ic32);
        do {
            ++it;
            mg_cycle<float, float>(S, x32, b32, 0, S.sp.mg_cycle, ic32);
        } while (it < S.sp.max_iters);
        convert_vec<float>(x32, x);
        return;
    }
    do {
        ++it;
        if (reduced)
            mg_cycle<double, float>(S, x, b, 0, S.sp.mg_cycle, iconv);
        else
            mg_cycle<double, double>(S, x, b, 0, S.sp.mg_cycle, iconv);
        if (S.sp.convergence_check) {
            get_residual<double>(S, x, b, r, res, true);
            if (converged<double>(S, res, rho0, iconv)) return;
        }
    } while (it < S.sp.max_iters);
}

static void precond_apply(Solver &S, Vec &x, Vec &b) {
    if (!S.precond) {  // no preconditioner list: identity, p_ = p
        blas::copy<double>(b, x);
        return;
    }
    Vec ones = typed_scalar<double>(S.NV, 1.0);
    solve<double>(*S.precond, x, b, ones);
}

// merged_bicgstab.inl:44-208 (preconditioned = false) and
// merged_pbicgstab.inl:44-225 (preconditioned = true)
static void solve_merged_bicgstab(Solver &S, Vec &x, Vec &b, const Vec &conv, bool precond) {
    typedef double F;
    const int NV = S.NV;
    reset_stats(S);
    int &it = S.st.iters;
    Vec iconv = conv;
    Vec a1 = typed_scalar<F>(NV, 1.0), a_1 = typed_scalar<F>(NV, -1.0);
    Vec rho = make_vec<F>(1, NV), rho0 = make_vec<F>(1, NV), res = make_vec<F>(1, NV);
    Vec scal1 = make_vec<F>(1, NV), scal2 = make_vec<F>(1, NV), scal3 = make_vec<F>(1, NV);
    Vec alpha = make_vec<F>(1, NV), beta = make_vec<F>(1, NV), omega = make_vec<F>(1, NV);
    Vec theta = make_vec<F>(1, NV), phi = make_vec<F>(1, NV), psi = make_vec<F>(1, NV);
    Vec alpha_conv = make_vec<F>(1, NV), omega_conv = make_vec<F>(1, NV);
    for (auto &v : S.buf) blas::set_const<F>(v, 0.0);
    Vec &r0 = S.buf[0], &r = S.buf[1], &p = S.buf[2], &v = S.buf[3], &s = S.buf[4],
        &t = S.buf[5], &p_ = S.buf[6], &s_ = S.buf[7];
    blas2::Ax_y<F>(*S.A, x, r0);
    blas::merged_bicgstab_group1<F>(r0, b, p, r, rho0);
    if (converged<F>(S, rho0, rho0, iconv)) return;
    blas::copy<F>(rho0, rho);
    do {
        ++it;
        Vec &pa = precond ? p_ : p;
        Vec &sa = precond ? s_ : s;
        if (precond) {
            blas::set_const<F>(p_, 0.0);
            precond_apply(S, p_, p);
        }
        blas2::Ax_y<F>(*S.A, pa, v);
        blas::dot<F>(v, r0, scal1);
        blas::xdivy_z<F>(rho, scal1, alpha);
        blas::scal<F>(a_1, alpha);
        blas::axpby_z<F>(a1, r, alpha, v, s);
        blas::scal<F>(a_1, alpha);
        if (precond) {
            blas::set_const<F>(s_, 0.0);
            precond_apply(S, s_, s);
        }
        blas2::Ax_y<F>(*S.A, sa, t);
        blas::merged_bicgstab_group2<F>(t, s, phi, psi, theta);
        blas::xdivy_z<F>(phi, psi, omega);
        blas::ax_y<F>(omega, phi, res);
        blas::axpby<F>(a1, theta, a_1, res);
        blas::ax_y<F>(iconv, alpha, alpha_conv);
        blas::ax_y<F>(iconv, omega, omega_conv);
        if (precond) {
            blas::axpbypcz<F>(alpha_conv, p_, omega_conv, s_, a1, x);
            if (converged<F>(S, res, rho0, iconv)) return;
        } else {
            if (converged<F>(S, res, rho0, iconv)) {
                blas::axpbypcz<F>(alpha_conv, p, omega_conv, s, a1, x);
                return;
            }
        }
        blas::merged_bicgstab_group4<F>(s, t, r0, r, omega, scal1);
        blas::xdivy_z<F>(scal1, rho, scal2);
        blas::xdivy_z<F>(alpha, omega, scal3);
        blas::ax_y<F>(scal2, scal3, beta);
        blas::copy<F>(scal1, rho);
        if (precond) {
            blas::ax_y<F>(omega, beta, scal1);
            blas::scal<F>(a_1, scal1);
            blas::axpbypcz<F>(a1, r, scal1, v, beta, p);
        } else {
            blas::ax_y<F>(iconv, alpha, alpha_conv);
            blas::ax_y<F>(iconv, omega, omega_conv);
            blas::merged_bicgstab_group5<F>(x, p, s, r, v, alpha_conv, omega_conv, alpha, omega,
                                            beta);
        }
    } while (it < S.sp.max_iters);
}

// bicgstab.inl:43-230 (precond = false) and pbicgstab.inl:43-235 (precond = true)
static void solve_bicgstab(Solver &S, Vec &x, Vec &b, const Vec &conv, bool precond) {
    typedef double F;
    const int NV = S.NV;
    reset_stats(S);
    int &it = S.st.iters;
    Vec iconv = conv;
    Vec a1 = typed_scalar<F>(NV, 1.0), a_1 = typed_scalar<F>(NV, -1.0);
    Vec rho = make_vec<F>(1, NV), rho0 = make_vec<F>(1, NV), res = make_vec<F>(1, NV);
    Vec scal1 = make_vec<F>(1, NV), scal2 = make_vec<F>(1, NV), scal3 = make_vec<F>(1, NV),
        scal4 = make_vec<F>(1, NV);
    Vec alpha = make_vec<F>(1, NV), beta = make_vec<F>(1, NV), omega = make_vec<F>(1, NV);
    Vec alpha_conv = make_vec<F>(1, NV), omega_conv = make_vec<F>(1, NV);
    for (auto &v : S.buf) blas::set_const<F>(v, 0.0);
    Vec &r0 = S.buf[0], &r = S.buf[1], &p = S.buf[2], &v = S.buf[3], &s = S.buf[4],
        &t = S.buf[5];
    get_residual<F>(S, x, b, r0, rho0, true);
    blas::copy<F>(r0, r);
    if (converged<F>(S, rho0, rho0, iconv)) return;
    blas::copy<F>(rho0, rho);
    blas::copy<F>(r0, p);
    do {
        ++it;
        Vec *pa = &p, *sa = &s;
        if (precond) {
            Vec &p_ = S.buf[6];
            blas::set_const<F>(p_, 0.0);
            precond_apply(S, p_, p);
            pa = &p_;
        }
        blas2::Ax_y<F>(*S.A, *pa, v);
        blas::dot<F>(v, r0, scal1);
        blas::xdivy_z<F>(rho, scal1, alpha);
        blas::scal<F>(a_1, alpha);
        blas::axpby_z<F>(a1, r, alpha, v, s);
        blas::scal<F>(a_1, alpha);
        if (precond) {
            Vec &s_ = S.buf[7];
            blas::set_const<F>(s_, 0.0);
            precond_apply(S, s_, s);
            sa = &s_;
        }
        blas2::Ax_y<F>(*S.A, *sa, t);
        blas::dot<F>(t, s, scal2);
        blas::dot<F>(t, t, scal3);
        blas::dot<F>(s, s, scal4);
        blas::xdivy_z<F>(scal2, scal3, omega);
        blas::ax_y<F>(iconv, alpha, alpha_conv);
        blas::ax_y<F>(iconv, omega, omega_conv);
        blas::axpbypcz<F>(alpha_conv, *pa, omega_conv, *sa, a1, x);
        blas::ax_y<F>(omega, scal2, res);
        blas::axpby<F>(a1, scal4, a_1, res);
        if (converged<F>(S, res, rho0, iconv)) return;
        blas::scal<F>(a_1, omega);
        blas::axpby_z<F>(a1, s, omega, t, r);
        blas::scal<F>(a_1, omega);
        blas::dot<F>(r, r0, scal1);
        blas::xdivy_z<F>(scal1, rho, scal2);
        blas::xdivy_z<F>(alpha, omega, scal3);
        blas::ax_y<F>(scal2, scal3, beta);
        blas::copy<F>(scal1, rho);
        blas::ax_y<F>(omega, beta, scal1);
        blas::scal<F>(a_1, scal1);
        blas::axpbypcz<F>(a1, r, scal1, v, beta, p);
    } while (it < S.sp.max_iters);
}

// pcg.inl:44-162: preconditioned conjugate gradients (the preconditioner is
// the identity when no preconditioner list is given)
static void solve_pcg(Solver &S, Vec &x, Vec &b, const Vec &conv) {
    typedef double F;
    const int NV = S.NV;
    reset_stats(S);
    int &it = S.st.iters;
    Vec iconv = conv;
    Vec a1 = typed_scalar<F>(NV, 1.0), a_1 = typed_scalar<F>(NV, -1.0);
    Vec rho0 = make_vec<F>(1, NV), res = make_vec<F>(1, NV);
    Vec scal1 = make_vec<F>(1, NV), scal2 = make_vec<F>(1, NV), scal3 = make_vec<F>(1, NV);
    Vec alpha = make_vec<F>(1, NV), beta = make_vec<F>(1, NV), alpha_conv = make_vec<F>(1, NV);
    for (auto &v : S.buf) blas::set_const<F>(v, 0.0);
    Vec &r = S.buf[0], &z = S.buf[1], &p = S.buf[2], &Ap = S.buf[3];
    get_residual<F>(S, x, b, r, rho0, S.sp.convergence_check != 0);
    if (converged<F>(S, rho0, rho0, iconv)) return;
    blas::set_const<F>(z, 0.0);
    precond_apply(S, z, r);
    blas::copy<F>(z, p);
    do {
        ++it;
        blas2::Ax_y<F>(*S.A, p, Ap);
        blas::dot<F>(r, z, scal1);
        blas::dot<F>(p, Ap, scal2);
        blas::xdivy_z<F>(scal1, scal2, alpha);
        blas::ax_y<F>(iconv, alpha, alpha_conv);
        blas::axpby<F>(alpha_conv, p, a1, x);
        blas::scal<F>(a_1, alpha);
        blas::axpby<F>(alpha, Ap, a1, r);
        blas::set_const<F>(z, 0.0);
        precond_apply(S, z, r);
        blas::dot<F>(r, z, scal3);
        blas::xdivy_z<F>(scal3, scal1, beta);
        blas::axpby<F>(a1, z, beta, p);
        blas::dot<F>(r, r, res);
        if (converged<F>(S, res, rho0, iconv)) return;
    } while (it < S.sp.max_iters);
}

// rbicgstab.inl:44-243 (merged = false) and merged_rbicgstab.inl:44-230
// (merged = true): BiCGStab reordered so that each preconditioner application
// can overlap a reduction
static void solve_rbicgstab(Solver &S, Vec &x, Vec &b, const Vec &conv, bool merged) {
    typedef double F;
    const int NV = S.NV;
    reset_stats(S);
    int &it = S.st.iters;
    Vec iconv = conv;
    Vec a1 = typed_scalar<F>(NV, 1.0), a_1 = typed_scalar<F>(NV, -1.0);
    Vec rho = make_vec<F>(1, NV), rho0 = make_vec<F>(1, NV), res = make_vec<F>(1, NV);
    Vec theta = make_vec<F>(1, NV), phi = make_vec<F>(1, NV), psi = make_vec<F>(1, NV),
        delta = make_vec<F>(1, NV), alpha = make_vec<F>(1, NV), beta = make_vec<F>(1, NV),
        omega = make_vec<F>(1, NV), eta = make_vec<F>(1, NV), temp = make_vec<F>(1, NV);
    Vec alpha_conv = make_vec<F>(1, NV), omega_conv = make_vec<F>(1, NV);
    for (auto &v : S.buf) blas::set_const<F>(v, 0.0);
    Vec &r0 = S.buf[0], &r = S.buf[1], &z = S.buf[2], &v_ = S.buf[3], &v = S.buf[4],
        &s = S.buf[5], &t_ = S.buf[6], &t = S.buf[7];
    get_residual<F>(S, x, b, r0, rho0, true);
    blas::copy<F>(r0, r);
    if (converged<F>(S, rho0, rho0, iconv)) return;
    blas::copy<F>(rho0, rho);
    blas::set_const<F>(z, 0.0);
    precond_apply(S, z, r0);
    blas::copy<F>(z, v_);
    do {
        ++it;
        blas2::Ax_y<F>(*S.A, v_, v);
        blas::dot<F>(v, r0, delta);
        blas::set_const<F>(s, 0.0);
        precond_apply(S, s, v);
        blas::xdivy_z<F>(rho, delta, alpha);
        blas::scal<F>(a_1, alpha);
        blas::axpby_z<F>(a1, z, alpha, s, t_);
        blas::scal<F>(a_1, alpha);
        blas2::Ax_y<F>(*S.A, t_, t);
        if (merged) {
            blas::merged_rbicgstab_group1<F>(r, v, t, r0, alpha, theta, phi, psi, eta);
        } else {
            blas::scal<F>(a_1, alpha);
            blas::axpby<F>(alpha, v, a1, r);
            blas::scal<F>(a_1, alpha);
            blas::dot<F>(t, r, theta);
            blas::dot<F>(t, t, phi);
            blas::dot<F>(t, r0, psi);
            blas::dot<F>(r, r, eta);
        }
        blas::set_const<F>(z, 0.0);
        precond_apply(S, z, t);
        blas::xdivy_z<F>(theta, phi, omega);
        blas::scal<F>(a_1, omega);
        blas::axpby<F>(omega, t, a1, r);
        blas::scal<F>(a_1, omega);
        blas::ax_y<F>(omega, theta, res);
        blas::axpby<F>(a1, eta, a_1, res);
        blas::ax_y<F>(iconv, alpha, alpha_conv);
        blas::ax_y<F>(iconv, omega, omega_conv);
        if (!merged) blas::axpbypcz<F>(alpha_conv, v_, omega_conv, t_, a1, x);
        if (converged<F>(S, res, rho0, iconv)) {
            if (merged) blas::axpbypcz<F>(alpha_conv, v_, omega_conv, t_, a1, x);
            return;
        }
        blas::ax_y<F>(omega, psi, rho);
        blas::scal<F>(a_1, rho);
        blas::ax_y<F>(delta, omega, temp);
        blas::xdivy_z<F>(rho, temp, beta);
        if (merged) {
            blas::ax_y<F>(iconv, alpha, alpha_conv);
            blas::ax_y<F>(iconv, omega, omega_conv);
            blas::merged_rbicgstab_group2<F>(x, v_, t_, z, s, alpha_conv, omega_conv, omega,
                                             beta);
        } else {
            blas::scal<F>(a_1, omega);
            blas::axpby<F>(a1, t_, omega, z);
            blas::ax_y<F>(omega, beta, delta);
            blas::scal<F>(a_1, omega);
            blas::axpbypcz<F>(a1, z, delta, s, beta, v_);
        }
    } while (it < S.sp.max_iters);
}

template <typename T>
static void solve(Solver &S, Vec &x, Vec &b, const Vec &conv) {
    const std::string &m = S.method;
    if (m == "Jacobi")
        solve_jacobi<T>(S, x, b, conv);
    else if (m == "HSGS")
        solve_hsgs<T>(S, x, b, conv);
    else if (m == "Chebyshev")
        solve_chebyshev<T>(S, x, b, conv);
    else if (m == "Direct")
        solve_direct<T>(S, x, b, conv);
    else if (m == "Identity")
        blas::copy<T>(b, x);
    else if (m == "MultiGrid")
        solve_mg(S, x, b, conv);
    else if (m == "MergedBiCGStab")
        solve_merged_bicgstab(S, x, b, conv, false);
    else if (m == "MergedPBiCGStab")
        solve_merged_bicgstab(S, x, b, conv, true);
    else if (m == "BiCGStab")
        solve_bicgstab(S, x, b, conv, false);
    else if (m == "PBiCGStab")
        solve_bicgstab(S, x, b, conv, true);
    else if (m == "PCG")
        solve_pcg(S, x, b, conv);
    else if (m == "RBiCGStab")
        solve_rbicgstab(S, x, b, conv, false);
    else if (m == "MergedRBiCGStab")
        solve_rbicgstab(S, x, b, conv, true);
}

// ----------------------------------------------------------------------------
// Solver construction: solver.h:259-276 (assemble), mg.inl:97-164 (setup)
// ----------------------------------------------------------------------------
struct System {
    Params P;
    std::vector<Csr> A64;  // level matrices as delivered by the hierarchy (double)
    std::vector<Csr> P64;  // interpolation P_l (n_l x n_{l+1}, double)
    std::vector<double> min_eig, max_eig;
    std::vector<Level> levels;
    std::shared_ptr<Solver> root;
    int NV = 1;
    int hsgs_ncores = 1;
};

static int buffer_nvecs(const std::string &m) {
    if (m == "Jacobi" || m == "HSGS") return 2;
    if (m == "Chebyshev") return 3;
    if (m == "MultiGrid") return 1;
    if (m == "BiCGStab") return 6;
    if (m == "PCG") return 4;
    if (m == "RBiCGStab" || m == "MergedRBiCGStab") return 8;
    if (m == "PBiCGStab" || m == "MergedBiCGStab" || m == "MergedPBiCGStab") return 8;
    return 0;
}

// op: the matrix the solver's SpMVs use when it differs from A (a BF16-valued
// level operator); diagonals and the other setup read A.
static std::shared_ptr<Solver> make_basic(System &sys, const std::string &role, int level,
                                          const Csr &A, bool f32, double min_eig,
                                          double max_eig, const Csr *op = nullptr) {
    auto S = std::make_shared<Solver>();
    S->sp = resolve(sys.P, role, level);
    S->method = S->sp.method;
    S->A = op ? op : &A;
    S->f32 = f32;
    S->NV = sys.NV;
    S->min_eig = min_eig;
    S->max_eig = max_eig;
    const std::string &m = S->method;
    if (m == "Jacobi" || m == "HSGS") S->id = f32 ? diag_vec<float>(A, false) : diag_vec<double>(A, false);
    if (m == "Chebyshev") S->isd = f32 ? diag_vec<float>(A, true) : diag_vec<double>(A, true);
    if (m == "HSGS") {
        // hsgs_ncores > 0: that many cores on every level; < 0: blocks of
        // about -hsgs_ncores rows, i.e. max(1, n / rows) cores on each level
        int nc = sys.hsgs_ncores;
        if (nc < 0) nc = (int)std::max<uint64_t>(1, A.nrows / (uint64_t)(-nc));
        S->core = std::make_shared<CoreLayer>(build_core_layer(A, nc));
    }
    if (m == "Direct") {
        if (f32)
            S->f_inv = gauss_jordan_inverse<float>(csr_to_dense<float>(A), A.nrows);
        else
            S->d_inv = gauss_jordan_inverse<double>(csr_to_dense<double>(A), A.nrows);
    }
    int nb = buffer_nvecs(m);
    for (int i = 0; i < nb; ++i) {
        Vec v;
        v.alloc(A.nrows, sys.NV, f32);
        S->buf.push_back(v);
    }
    S->st.conv.assign(sys.NV, 0);
    S->st.abs_res.assign(sys.NV, 0.0);
    S->st.rel_res.assign(sys.NV, 0.0);
    return S;
}

static int setup(System &sys) {
    if (sys.A64.empty()) return -1;
    // dictionary defaults (xamg_params_details.h:131-144): with a MultiGrid
    // list present, missing smoother lists are Jacobi and the coarse grid
    // solver is Direct
    bool any_mg = false;
    for (auto &l : sys.P.base) {
        auto m = l.second.find("method");
        if (m != l.second.end() && m->second == "MultiGrid") any_mg = true;
    }
    if (any_mg) {
        if (!sys.P.has("pre_smoother")) sys.P.base["pre_smoother"]["method"] = "Jacobi";
        if (!sys.P.has("post_smoother")) sys.P.base["post_smoother"]["method"] = "Jacobi";
        if (!sys.P.has("coarse_grid_solver")) sys.P.base["coarse_grid_solver"]["method"] = "Direct";
    }
    const std::string pre = sys.P.get("preconditioner", "method");
    const std::string sol = sys.P.get("solver", "method");
    const bool mg_solver = (sol == "MultiGrid");
    const bool mg_prec = (pre == "MultiGrid");
    const std::string mg_role = mg_solver ? "solver" : "preconditioner";
    bool reduced = false, full32 = false;
    int bf16_levels = 0;
    bool fp16 = false;
    if (mg_solver || mg_prec) {
        std::string bf = sys.P.get(mg_role, "gpu_level_bf16");
        if (!bf.empty()) bf16_levels = (int)std::stol(bf);
        std::string hf = sys.P.get(mg_role, "gpu_level_fp16");
        fp16 = !hf.empty() && std::stol(hf) == 1;
        std::string v = sys.P.get(mg_role, "mg_reduced_precision");
        reduced = !v.empty() && std::stol(v) != 0;
        // B200 extension: gpu_precond_f32 = 1 puts the finest level of the
        // multigrid preconditioner in float too (0: none, unset: XAMG's rule)
        std::string g = sys.P.get(mg_role, "gpu_precond_f32");
        if (!g.empty()) {
            reduced = std::stol(g) != 0;
            full32 = mg_prec && std::stol(g) == 1;
        }
    }
    // hierarchy parse: hypre_base.inl:337-403 (A_l, eigenvalue estimates,
    // P_l and R_l = transpose(P_l), converted to float when reduced)
    const size_t L = (mg_solver || mg_prec) ? sys.A64.size() : 1;
    sys.levels.assign(L, Level());
    for (size_t l = 0; l < L; ++l) {
        Level &lv = sys.levels[l];
        lv.reduced = (l >= 1 || full32) && reduced;
        lv.A = lv.reduced ? to_f32(sys.A64[l]) : sys.A64[l];
        // gpu_level_bf16: the finest float cycle operators store BF16 values
        // (the smoothers' diagonals and the transfers keep the float values)
        lv.bf16 = lv.reduced && (int)l < bf16_levels;
        if (lv.bf16) lv.Abf = fp16 ? to_fp16_values(lv.A) : to_bf16_values(lv.A);
        lv.min_eig = sys.min_eig[l];
        lv.max_eig = sys.max_eig[l];
        if (l + 1 < L) {
            Csr Pm = sys.P64[l];
            Csr Rm = transpose(Pm);
            lv.P = reduced ? to_f32(Pm) : Pm;
            lv.R = reduced ? to_f32(Rm) : Rm;
        }
    }
    auto build_mg = [&](const std::string &role) {
        auto M = std::make_shared<Solver>();
        M->sp = resolve(sys.P, role, -1);
        M->method = "MultiGrid";
        M->A = &sys.levels[0].A;
        M->NV = sys.NV;
        M->levels = &sys.levels;
        for (size_t nl = 0; nl + 1 < L; ++nl) {
            Level &lv = sys.levels[nl];
            const Csr *op = lv.bf16 ? &lv.Abf : nullptr;
            M->pre.push_back(make_basic(sys, "pre_smoother", (int)nl, lv.A, lv.reduced,
                                        lv.min_eig, lv.max_eig, op));
            M->post.push_back(make_basic(sys, "post_smoother", (int)nl, lv.A, lv.reduced,
                                         lv.min_eig, lv.max_eig, op));
        }
        Level &cl = sys.levels[L - 1];
        M->coarse = make_basic(sys, "coarse_grid_solver", -1, cl.A, cl.reduced, cl.min_eig,
                               cl.max_eig, cl.bf16 ? &cl.Abf : nullptr);
        M->mgbuf.resize(L);
        for (size_t nl = 0; nl < L; ++nl) {
            const uint64_t n = sys.levels[nl].A.nrows;
            if (nl == 0) {
                if (sys.levels[0].reduced) {
                    // every level in float: the level-0 residual is float too
                    M->mgbuf[0].push_back(make_vec<float>(n, sys.NV));
                } else {
                    M->mgbuf[0].push_back(make_vec<double>(n, sys.NV));
                    if (reduced) M->mgbuf[0].push_back(make_vec<float>(n, sys.NV));
                }
            } else {
                for (int i = 0; i < 3; ++i) {
                    Vec v;
                    v.alloc(n, sys.NV, sys.levels[nl].reduced);
                    M->mgbuf[nl].push_back(v);
                }
            }
        }
        M->buf.push_back(make_vec<double>(sys.levels[0].A.nrows, sys.NV));
        M->st.conv.assign(sys.NV, 0);
        M->st.abs_res.assign(sys.NV, 0.0);
        M->st.rel_res.assign(sys.NV, 0.0);
        return M;
    };
    if (mg_solver) {
        sys.root = build_mg("solver");
    } else {
        sys.root = make_basic(sys, "solver", -1, sys.A64[0], false, sys.levels[0].min_eig,
                              sys.levels[0].max_eig);
        if (sys.P.has("preconditioner")) {
            if (mg_prec)
                sys.root->precond = build_mg("preconditioner");
            else
                sys.root->precond = make_basic(sys, "preconditioner", -1, sys.A64[0], false,
                                               sys.levels[0].min_eig, sys.levels[0].max_eig);
        }
    }
    return 0;
}

static Csr csr_from(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint32_t *row,
                    const uint32_t *col, const double *val) {
    Csr c;
    c.nrows = c.block_nrows = nrows;
    c.ncols = c.block_ncols = ncols;
    c.nonzeros = nnz;
    c.row.assign(row, row + nrows + 1);
    c.col.assign(col, col + nnz);
    c.vd.assign(val, val + nnz);
    return c;
}

}  // namespace orc

// ============================================================================
// C ABI for the tests (ctypes)
// ============================================================================
using namespace orc;

extern "C" {

int or_version() { return 1; }

// Threads the SpMV row loops use (OMP_NUM_THREADS, default: all cores).
int or_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_reduction(int mode, int ncores) {
    g_red.mode = mode;
    g_red.ncores = ncores < 1 ? 1 : ncores;
}

uint16_t or_define_int_type(uint64_t range) { return define_int_type(range); }

uint16_t or_encode_hash(uint64_t nnz, uint64_t ncols, uint64_t bnrows, uint64_t bncols, int f32,
                        int reduced) {
    return encode_hash(nnz, ncols, bnrows, bncols, f32 != 0, reduced != 0);
}

void or_core_range(uint64_t n, int ncores, int core, uint64_t *off, uint64_t *size) {
    core_range(n, ncores, core, *off, *size);
}

// y = A x (f32 = 0: double values/vectors; 1: float)
void or_csr_ax_y(int f32, uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint32_t *row,
                 const uint32_t *col, const void *val, const void *x, void *y, int nv) {
    Csr m;
    m.nrows = m.block_nrows = nrows;
    m.ncols = m.block_ncols = ncols;
    m.nonzeros = nnz;
    m.row.assign(row, row + nrows + 1);
    m.col.assign(col, col + nnz);
    m.f32 = f32 != 0;
    Vec X, Y;
    X.alloc(ncols, nv, m.f32);
    Y.alloc(nrows, nv, m.f32);
    X.zero = false;
    X.init = true;
    if (m.f32) {
        m.vf.assign((const float *)val, (const float *)val + nnz);
        std::memcpy(X.f.data(), x, ncols * nv * sizeof(float));
        blas2::csr_Ax_y<float>(m, X, Y);
        std::memcpy(y, Y.f.data(), nrows * nv * sizeof(float));
    } else {
        m.vd.assign((const double *)val, (const double *)val + nnz);
        std::memcpy(X.d.data(), x, ncols * nv * sizeof(double));
        blas2::csr_Ax_y<double>(m, X, Y);
        std::memcpy(y, Y.d.data(), nrows * nv * sizeof(double));
    }
}

// y += A x
void or_csr_axpy(int f32, uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint32_t *row,
                 const uint32_t *col, const void *val, const void *x, void *y, int nv) {
    Csr m;
    m.nrows = m.block_nrows = nrows;
    m.ncols = m.block_ncols = ncols;
    m.nonzeros = nnz;
    m.row.assign(row, row + nrows + 1);
    m.col.assign(col, col + nnz);
    m.f32 = f32 != 0;
    Vec X, Y;
    X.alloc(ncols, nv, m.f32);
    Y.alloc(nrows, nv, m.f32);
    X.zero = Y.zero = false;
    X.init = Y.init = true;
    if (m.f32) {
        m.vf.assign((const float *)val, (const float *)val + nnz);
        std::memcpy(X.f.data(), x, ncols * nv * sizeof(float));
        std::memcpy(Y.f.data(), y, nrows * nv * sizeof(float));
        blas2::csr_Axpy<float>(m, X, Y);
        std::memcpy(y, Y.f.data(), nrows * nv * sizeof(float));
    } else {
        m.vd.assign((const double *)val, (const double *)val + nnz);
        std::memcpy(X.d.data(), x, ncols * nv * sizeof(double));
        std::memcpy(Y.d.data(), y, nrows * nv * sizeof(double));
        blas2::csr_Axpy<double>(m, X, Y);
        std::memcpy(y, Y.d.data(), nrows * nv * sizeof(double));
    }
}

// compress() of an off-diagonal block. Outputs: new row pointer (first
// *nrows_out+1 entries of row), renumbered col, row_ind (<= nrows), col_ind
// (<= block_ncols).
void or_compress(uint64_t nrows, uint64_t block_ncols, uint64_t nnz, uint32_t *row, uint32_t *col,
                 uint32_t *row_ind, uint32_t *col_ind, uint64_t *nrows_out, uint64_t *ncols_out) {
    Csr m;
    m.nrows = m.block_nrows = nrows;
    m.ncols = m.block_ncols = block_ncols;
    m.nonzeros = nnz;
    m.row.assign(row, row + nrows + 1);
    m.col.assign(col, col + nnz);
    m.vd.assign(nnz, 1.0);
    compress(m);
    std::copy(m.row.begin(), m.row.end(), row);
    std::copy(m.col.begin(), m.col.end(), col);
    std::copy(m.row_ind.begin(), m.row_ind.end(), row_ind);
    std::copy(m.col_ind.begin(), m.col_ind.end(), col_ind);
    *nrows_out = m.nrows;
    *ncols_out = m.ncols;
}

// transpose of a double CSR (R = P^T)
void or_transpose(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint32_t *row,
                  const uint32_t *col, const double *val, uint32_t *trow, uint32_t *tcol,
                  double *tval) {
    Csr m = csr_from(nrows, ncols, nnz, row, col, val);
    Csr t = transpose(m);
    std::copy(t.row.begin(), t.row.end(), trow);
    std::copy(t.col.begin(), t.col.end(), tcol);
    std::copy(t.vd.begin(), t.vd.end(), tval);
}

// Gauss-Jordan inverse of a dense n x n matrix (f32: float arrays)
void or_inverse(int f32, uint64_t n, const void *a, void *ainv) {
    if (f32) {
        std::vector<float> m((const float *)a, (const float *)a + n * n);
        auto r = gauss_jordan_inverse<float>(m, n);
        std::memcpy(ainv, r.data(), n * n * sizeof(float));
    } else {
        std::vector<double> m((const double *)a, (const double *)a + n * n);
        auto r = gauss_jordan_inverse<double>(m, n);
        std::memcpy(ainv, r.data(), n * n * sizeof(double));
    }
}

void or_inv_diag(int f32, int sqrt_, uint64_t nrows, uint64_t nnz, const uint32_t *row,
                 const uint32_t *col, const double *val, void *out) {
    Csr m = csr_from(nrows, nrows, nnz, row, col, val);
    if (f32) {
        Csr mf = to_f32(m);
        auto d = inv_diag<float>(mf, sqrt_ != 0);
        std::memcpy(out, d.data(), nrows * sizeof(float));
    } else {
        auto d = inv_diag<double>(m, sqrt_ != 0);
        std::memcpy(out, d.data(), nrows * sizeof(double));
    }
}

void or_cheby_coeffs(double min_eig, double max_eig, int order, float frac, double *out) {
    auto c = cheby_coeffs(min_eig, max_eig, order, (double)frac);
    for (int i = 0; i < order; ++i) out[i] = c[i];
}

// BF16 rounding of float values (gpu_level_bf16 operators)
void or_round_bf16(uint64_t n, const float *in, float *out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = round_bf16(in[i]);
}

// dot products in the configured reduction order (double)
void or_dot(uint64_t n, int nv, const double *x, const double *y, double *out) {
    Vec X, Y, R;
    X.alloc(n, nv, false);
    Y.alloc(n, nv, false);
    R.alloc(1, nv, false);
    std::memcpy(X.d.data(), x, n * nv * sizeof(double));
    std::memcpy(Y.d.data(), y, n * nv * sizeof(double));
    X.zero = Y.zero = false;
    blas::dot<double>(X, Y, R);
    std::memcpy(out, R.d.data(), nv * sizeof(double));
}

// merged BiCGStab groups (double), arrays [n][nv]
void or_group1(uint64_t n, int nv, double *r0, const double *b, double *p, double *r,
               double *rho0) {
    Vec R0, Bv, Pv, Rv, Rho;
    R0.alloc(n, nv, false);
    Bv.alloc(n, nv, false);
    Pv.alloc(n, nv, false);
    Rv.alloc(n, nv, false);
    Rho.alloc(1, nv, false);
    std::memcpy(R0.d.data(), r0, n * nv * 8);
    std::memcpy(Bv.d.data(), b, n * nv * 8);
    R0.zero = Bv.zero = false;
    blas::merged_bicgstab_group1<double>(R0, Bv, Pv, Rv, Rho);
    std::memcpy(r0, R0.d.data(), n * nv * 8);
    std::memcpy(p, Pv.d.data(), n * nv * 8);
    std::memcpy(r, Rv.d.data(), n * nv * 8);
    std::memcpy(rho0, Rho.d.data(), nv * 8);
}

void or_group2(uint64_t n, int nv, const double *t, const double *s, double *phi, double *psi,
               double *theta) {
    Vec Tv, Sv, a, b2, c;
    Tv.alloc(n, nv, false);
    Sv.alloc(n, nv, false);
    a.alloc(1, nv, false);
    b2.alloc(1, nv, false);
    c.alloc(1, nv, false);
    std::memcpy(Tv.d.data(), t, n * nv * 8);
    std::memcpy(Sv.d.data(), s, n * nv * 8);
    Tv.zero = Sv.zero = false;
    blas::merged_bicgstab_group2<double>(Tv, Sv, a, b2, c);
    std::memcpy(phi, a.d.data(), nv * 8);
    std::memcpy(psi, b2.d.data(), nv * 8);
    std::memcpy(theta, c.d.data(), nv * 8);
}

void or_group4(uint64_t n, int nv, const double *s, const double *t, const double *r0, double *r,
               const double *omega, double *rho) {
    Vec Sv, Tv, R0, Rv, Om, Rho;
    Sv.alloc(n, nv, false);
    Tv.alloc(n, nv, false);
    R0.alloc(n, nv, false);
    Rv.alloc(n, nv, false);
    Om.alloc(1, nv, false);
    Rho.alloc(1, nv, false);
    std::memcpy(Sv.d.data(), s, n * nv * 8);
    std::memcpy(Tv.d.data(), t, n * nv * 8);
    std::memcpy(R0.d.data(), r0, n * nv * 8);
    std::memcpy(Om.d.data(), omega, nv * 8);
    Sv.zero = Tv.zero = R0.zero = Om.zero = false;
    blas::merged_bicgstab_group4<double>(Sv, Tv, R0, Rv, Om, Rho);
    std::memcpy(r, Rv.d.data(), n * nv * 8);
    std::memcpy(rho, Rho.d.data(), nv * 8);
}

// cube.inl:28-174 restated: 7-point Laplacian on nx*ny*nz (one rank)
uint64_t or_generate_cube(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t *row, uint32_t *col,
                          double *val) {
    const uint64_t n = nx * ny * nz;
    double hx = 1.0 / nx, hy = 1.0 / ny, hz = 1.0 / nz;
    double q1 = 1.0 / hx / hx, q2 = 1.0 / hy / hy, q3 = 1.0 / hz / hz;
    uint64_t cntr = 0;
    row[0] = 0;
    for (uint64_t indx = 0; indx < n; ++indx) {
        uint64_t ii = indx % nx, jj = (indx / nx) % ny, kk = indx / (nx * ny);
        uint64_t d = cntr;
        col[cntr] = (uint32_t)indx;
        val[cntr++] = 0.0;
        if (kk > 0) { val[d] += q3; col[cntr] = (uint32_t)(indx - nx * ny); val[cntr++] = -q3; }
        else if (nz > 1) val[d] += 2.0 * q3;
        if (jj > 0) { val[d] += q2; col[cntr] = (uint32_t)(indx - nx); val[cntr++] = -q2; }
        else if (ny > 1) val[d] += 2.0 * q2;
        if (ii > 0) { val[d] += q1; col[cntr] = (uint32_t)(indx - 1); val[cntr++] = -q1; }
        else if (nx > 1) val[d] += 2.0 * q1;
        if (ii < nx - 1) { val[d] += q1; col[cntr] = (uint32_t)(indx + 1); val[cntr++] = -q1; }
        else if (nx > 1) val[d] += 2.0 * q1;
        if (jj < ny - 1) { val[d] += q2; col[cntr] = (uint32_t)(indx + nx); val[cntr++] = -q2; }
        else if (ny > 1) val[d] += 2.0 * q2;
        if (kk < nz - 1) { val[d] += q3; col[cntr] = (uint32_t)(indx + nx * ny); val[cntr++] = -q3; }
        else if (nz > 1) val[d] += 2.0 * q3;
        row[indx + 1] = (uint32_t)cntr;
    }
    return cntr;
}

// ---- whole-system solve --------------------------------------------------
void *or_sys_create(int nv) {
    System *s = new System();
    s->NV = nv;
    return s;
}
void or_sys_destroy(void *h) { delete (System *)h; }

void or_sys_set_param(void *h, const char *role, const char *key, const char *value, int level) {
    System *s = (System *)h;
    if (level < 0)
        s->P.base[role][key] = value;
    else
        s->P.lev[role][level][key] = value;
}

void or_sys_set_hsgs_cores(void *h, int ncores) { ((System *)h)->hsgs_ncores = ncores; }

void or_sys_add_level(void *h, uint64_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col,
                      const double *val, double min_eig, double max_eig) {
    System *s = (System *)h;
    s->A64.push_back(csr_from(n, n, nnz, row, col, val));
    s->min_eig.push_back(min_eig);
    s->max_eig.push_back(max_eig);
}

void or_sys_add_interp(void *h, uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint32_t *row,
                       const uint32_t *col, const double *val) {
    System *s = (System *)h;
    s->P64.push_back(csr_from(nrows, ncols, nnz, row, col, val));
}

int or_sys_setup(void *h) { return setup(*(System *)h); }

// x: in = initial guess, out = solution; conv/abs/rel: nv entries; returns iters
int or_sys_solve(void *h, double *x, const double *b, int *conv, double *abs_res,
                 double *rel_res) {
    System *s = (System *)h;
    const uint64_t n = s->levels[0].A.nrows;
    const int nv = s->NV;
    Vec X, B;
    X.alloc(n, nv, false);
    B.alloc(n, nv, false);
    std::memcpy(X.d.data(), x, n * nv * 8);
    std::memcpy(B.d.data(), b, n * nv * 8);
    X.zero = B.zero = false;
    X.init = B.init = true;
    Vec ones = typed_scalar<double>(nv, 1.0);
    solve<double>(*s->root, X, B, ones);
    std::memcpy(x, X.d.data(), n * nv * 8);
    for (int k = 0; k < nv; ++k) {
        conv[k] = s->root->st.conv[k];
        abs_res[k] = s->root->st.abs_res[k];
        rel_res[k] = s->root->st.rel_res[k];
    }
    return s->root->st.iters;
}

// Export the working-precision level data the oracle derived, for
// bit-exact comparison with what the product uploaded: which = 0 A, 1 R, 2 P.
// Returns nnz; fills row/col and val as float or double by the level precision.
uint64_t or_sys_level_matrix(void *h, int level, int which, uint32_t *row, uint32_t *col,
                             void *val, int *is_f32, uint64_t *nrows, uint64_t *ncols) {
    System *s = (System *)h;
    Level &lv = s->levels[level];
    const Csr &m = which == 0 ? lv.A : (which == 1 ? lv.R : lv.P);
    *is_f32 = m.f32;
    *nrows = m.nrows;
    *ncols = m.ncols;
    if (row) std::copy(m.row.begin(), m.row.end(), row);
    if (col) std::copy(m.col.begin(), m.col.end(), col);
    if (val) {
        if (m.f32)
            std::memcpy(val, m.vf.data(), m.nonzeros * 4);
        else
            std::memcpy(val, m.vd.data(), m.nonzeros * 8);
    }
    return m.nonzeros;
}

}  // extern "C"
