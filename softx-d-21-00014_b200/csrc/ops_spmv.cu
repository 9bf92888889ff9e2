// Launchers of the CSR kernels: runtime (nv, column width) -> template
// instantiation of k_spmv with the matching epilogue.
#include <algorithm>
#include <map>
#include <tuple>
#include <type_traits>

#include "ops.h"

namespace xg {
namespace ops {

template <int V>
using NVc = std::integral_constant<int, V>;

template <class Fn>
static void dispatch_nv(int nv, Fn &&fn) {
    switch (nv) {
    case 1: fn(NVc<1>()); break;
    case 2: fn(NVc<2>()); break;
    case 4: fn(NVc<4>()); break;
    case 8: fn(NVc<8>()); break;
    case 16: fn(NVc<16>()); break;
    case 32: fn(NVc<32>()); break;
    default: throw Error(XAMG_ERR_INVALID_ARG, "nv must be one of 1,2,4,8,16,32");
    }
}

template <class Fn>
static void dispatch_col(int cb, Fn &&fn) {
    switch (cb) {
    case 1: fn((uint8_t *)nullptr); break;
    case 2: fn((uint16_t *)nullptr); break;
    case 4: fn((uint32_t *)nullptr); break;
    case -2: fn((int16_t *)nullptr); break;
    default: throw Error(XAMG_ERR_INVALID_ARG, "column width must be 1, 2, 4 or -2 bytes");
    }
}

// Largest tile entry count for nv: known from the upload for library-owned
// matrices; for caller-owned device descriptors computed once on the device
// and remembered per (row pointer, rows). A stale value can only change which
// tiles are staged, never a result.
static uint32_t tile_max(const DCsr &A, int nv, cudaStream_t s) {
    int l = 0;
    while ((1 << l) < nv) ++l;
    if (A.tile_max[l] || A.nnz == 0) return A.tile_max[l];
    static std::map<std::tuple<const void *, uint64_t, int>, uint32_t> cache;
    auto key = std::make_tuple((const void *)A.row.p, A.nrows, l);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const uint64_t R = (uint64_t)k::CT >> l;
    const uint64_t ntiles = (A.nrows + R - 1) / R;
    unsigned *d = ctx().red_ticket.as<unsigned>() + 1;
    XG_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned), s));
    k::k_tile_max<<<(unsigned)((ntiles + 255) / 256), 256, 0, s>>>(A.row.as<uint32_t>(), A.nrows,
                                                                     R, d);
    XG_CUDA(cudaGetLastError());
    unsigned h = 0;
    XG_CUDA(cudaMemcpyAsync(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    XG_CUDA(cudaStreamSynchronize(s));
    cache[key] = h;
    return h;
}

// Staging buffers: one buffer holds cap entries of values and columns (plus
// alignment slack); two buffers (the copy of the next tile overlapping the
// current one) while they fit in 48 KB, at least four blocks per SM; else one
// buffer of up to 96 KB.
template <typename F, typename I>
static uint32_t stage_buffer_bytes(uint32_t cap) {
    auto r16 = [](uint64_t b) { return (uint32_t)((b + 15) & ~(uint64_t)15); };
    return r16((uint64_t)cap * sizeof(F) + 32) + r16((uint64_t)cap * sizeof(I) + 32);
}

template <typename F, typename FX, typename I, int NV, int VK, int NRED, class Epi>
static void launch_vk(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s) {
    const int B = k::canon_blocks(A.nrows, NV);
    constexpr uint32_t LIMIT1 = (96u * 1024u - 64u) / (uint32_t)(sizeof(F) + sizeof(I));
    const uint32_t tm = tile_max(A, NV, s);
    uint32_t cap = tm, nbuf = 2;
    if (2 * stage_buffer_bytes<F, I>(tm) > 48u * 1024u) {
        nbuf = 1;
        cap = std::min(tm, LIMIT1);
    }
    const size_t smem = (size_t)nbuf * stage_buffer_bytes<F, I>(cap);
    auto kern = k::k_spmv<F, FX, I, NV, VK, NRED, Epi>;
    static bool big_smem = false;  // one flag per instantiation
    if (smem > 48u * 1024u && !big_smem) {
        XG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)stage_buffer_bytes<F, I>(LIMIT1)));
        big_smem = true;
    }
    kern<<<B, k::CT / VK, smem, s>>>(A.args<F>(), x, epi, ctx().red(), cap, nbuf);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

// Vector loads of x need x aligned to VK elements; library vectors always are
// (cudaMalloc). The entry points that take a caller's x (CALLER_X) fall back
// to one right-hand side per thread for an x that is not (same results, same
// reduction order).
template <typename F, typename FX, typename I, int NV, int NRED, bool CALLER_X = false,
          class Epi>
static void launch(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s) {
    if (A.nrows == 0) return;
    constexpr int VK = k::spmv_vk<FX, NV>();
    constexpr uintptr_t ALIGN = VK * sizeof(FX);
    if (VK == 1 || (uintptr_t)x % ALIGN == 0) {
        launch_vk<F, FX, I, NV, VK, NRED>(A, x, epi, s);
    } else if constexpr (CALLER_X) {
        launch_vk<F, FX, I, NV, 1, NRED>(A, x, epi, s);
    } else {
        throw Error(XAMG_ERR_INTERNAL, "library vector not aligned for the SpMV gather");
    }
}

template <typename F, int NV, int NRED, class Epi>
static void launch_rows(uint64_t n, const Epi &epi, cudaStream_t s) {
    if (n == 0) return;
    const int B = k::canon_blocks(n, NV);
    k::k_rows<F, NV, NRED, Epi><<<B, k::CT, 0, s>>>(n, epi, ctx().red());
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

#define XG_DISPATCH(A, nv, ...)                                             \
    dispatch_nv(nv, [&](auto nvc) {                                         \
        constexpr int NV = decltype(nvc)::value;                            \
        dispatch_col((A).col_bytes, [&](auto ip) {                          \
            using I = std::remove_pointer_t<decltype(ip)>;                  \
            __VA_ARGS__;                                                    \
        });                                                                 \
    })

void wait_selftest(uint64_t limit_ns, cudaStream_t s) {
    k::k_wait_selftest<<<1, 32, 0, s>>>(limit_ns, ctx().red().flag);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

template <typename F>
void spmv(const DCsr &A, const F *x, F *y, int nv, bool axpy, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        if (axpy)
            launch<F, F, I, NV, 0, true>(A, x, k::EAxpy<F, NV>{{}, y}, s);
        else
            launch<F, F, I, NV, 0, true>(A, x, k::EStore<F, NV>{{}, y}, s);
    });
}
template void spmv<double>(const DCsr &, const double *, double *, int, bool, cudaStream_t);
template void spmv<float>(const DCsr &, const float *, float *, int, bool, cudaStream_t);

void spmv_f32_from_f64(const DCsr &A, const double *x, float *y, int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, { launch<float, double, I, NV, 0>(A, x, k::EStore<float, NV>{{}, y}, s); });
}

template <typename F>
void residual(const DCsr &A, const F *x, const F *b, F *r, int nv, double *norm_out,
              cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        if (norm_out)
            launch<F, F, I, NV, 1>(A, x, k::EResid<F, NV, true>{r, b, norm_out}, s);
        else
            launch<F, F, I, NV, 0>(A, x, k::EResid<F, NV, false>{r, b, nullptr}, s);
    });
}
template void residual<double>(const DCsr &, const double *, const double *, double *, int,
                               double *, cudaStream_t);
template void residual<float>(const DCsr &, const float *, const float *, float *, int, double *,
                              cudaStream_t);

void group1(const DCsr &A, const double *x, const double *b, double *r0, double *p, double *r,
            double *sc, int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        launch<double, double, I, NV, 1>(A, x, k::EGroup1<NV>{r0, p, r, b, sc}, s);
    });
}

// group1 with a zero-flagged x: Ax_y leaves r0 zero-flagged and group1 then
// computes r0 = b - 0 (blas_merged_bicgstab.inl:45-46 writes the zeros).
template <int NV>
struct EGroup1Zero {
    double *r0, *p, *r;
    const double *b;
    double *sc;
    template <int NR>
    __device__ void elem(uint64_t i, int kk, double (&acc)[NR]) const {
        const uint64_t e = i * NV + kk;
        const double rv = k::sub(b[e], 0.0);
        r0[e] = rv;
        p[e] = rv;
        r[e] = rv;
        acc[0] = k::add(acc[0], k::mul(rv, rv));
    }
    __device__ void operator()(int kk, const double *s1) const {
        sc[k::SC_RHO0 * k::SC_STRIDE + kk] = s1[0];
        sc[k::SC_RHO * k::SC_STRIDE + kk] = s1[0];
    }
};

void group1_zero(uint64_t n, const double *b, double *r0, double *p, double *r, double *sc,
                 int nv, cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        launch_rows<double, NV, 1>(n, EGroup1Zero<NV>{r0, p, r, b, sc}, s);
    });
}

void spmv_dot_alpha(const DCsr &A, const double *pa, double *v, const double *r0, double *sc,
                    int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        launch<double, double, I, NV, 1, true>(A, pa, k::EDotAlpha<NV>{v, r0, sc}, s);
    });
}

void spmv_dot3(const DCsr &A, const double *sa, double *t, const double *s_, double *sc, int nv,
               cudaStream_t s) {
    XG_DISPATCH(A, nv, { launch<double, double, I, NV, 3>(A, sa, k::EDot3<NV>{t, s_, sc}, s); });
}

template <typename F>
void jacobi_sweep(const DCsr &A, const F *xin, F *xout, const F *b, const F *d, F relax, int nv,
                  cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        launch<F, F, I, NV, 0>(A, xin, k::EJacobi<F, NV>{{}, xout, xin, b, d, relax}, s);
    });
}
template void jacobi_sweep<double>(const DCsr &, const double *, double *, const double *,
                                   const double *, double, int, cudaStream_t);
template void jacobi_sweep<float>(const DCsr &, const float *, float *, const float *,
                                  const float *, float, int, cudaStream_t);

template <typename F>
void cheby_first(const DCsr &A, const F *x, bool x_zero, const F *b, const F *isd, F c, F *rs,
                 F *t1s, int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        k::ECheby0<F, NV> e{{}, rs, t1s, b, isd, c};
        if (x_zero)
            launch_rows<F, NV, 0>(A.nrows, e, s);
        else
            launch<F, F, I, NV, 0>(A, x, e, s);
    });
}
template void cheby_first<double>(const DCsr &, const double *, bool, const double *,
                                  const double *, double, double *, double *, int, cudaStream_t);
template void cheby_first<float>(const DCsr &, const float *, bool, const float *, const float *,
                                 float, float *, float *, int, cudaStream_t);

template <typename F>
void cheby_step(const DCsr &A, const F *t1s, const F *rs, const F *isd, F c, F *out, bool last,
                bool x_zero, int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        launch<F, F, I, NV, 0>(
            A, t1s, k::ECheby1<F, NV>{{}, out, rs, isd, c, (int)last, (int)x_zero}, s);
    });
}
template void cheby_step<double>(const DCsr &, const double *, const double *, const double *,
                                 double, double *, bool, bool, int, cudaStream_t);
template void cheby_step<float>(const DCsr &, const float *, const float *, const float *, float,
                                float *, bool, bool, int, cudaStream_t);

void prolong_mixed(const DCsr &P, const float *xH, double *x, bool x_zero, int nv,
                   cudaStream_t s) {
    XG_DISPATCH(P, nv, {
        launch<float, float, I, NV, 0>(P, xH, k::EProlongMixed<NV>{{}, x, (int)x_zero}, s);
    });
}

template <typename F>
void hsgs_sweep(const DCsr &A, const uint64_t *boff, int nblocks, const F *t, F *x, const F *d,
                const double *relax_sc, int nv, cudaStream_t s) {
    if (nblocks == 0) return;
    XG_DISPATCH(A, nv, {
        const uint64_t threads = (uint64_t)nblocks * NV;
        const int B = (int)((threads + k::CT - 1) / k::CT);
        k::k_hsgs_sweep<F, I, NV><<<B, k::CT, 0, s>>>(A.row.as<uint32_t>(), (const I *)A.col.p,
                                                      A.val.as<F>(), boff, nblocks, t, x, d,
                                                      relax_sc);
        XG_CUDA(cudaGetLastError());
        ++g_kernel_launches;
    });
}
template void hsgs_sweep<double>(const DCsr &, const uint64_t *, int, const double *, double *,
                                 const double *, const double *, int, cudaStream_t);
template void hsgs_sweep<float>(const DCsr &, const uint64_t *, int, const float *, float *,
                                const float *, const double *, int, cudaStream_t);

template <typename F>
void dense_apply(const F *a, uint64_t n, const F *x, F *y, int nv, cudaStream_t s) {
    if (n == 0) return;
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        const uint64_t m = n * NV;
        k::k_dense<F, NV><<<(unsigned)((m + k::CT - 1) / k::CT), k::CT, 0, s>>>(a, n, x, y);
        XG_CUDA(cudaGetLastError());
        ++g_kernel_launches;
    });
}
template void dense_apply<double>(const double *, uint64_t, const double *, double *, int,
                                  cudaStream_t);
template void dense_apply<float>(const float *, uint64_t, const float *, float *, int,
                                 cudaStream_t);

// --- canonical-order vector reductions ------------------------------------
template <typename F>
void dot(uint64_t n, const F *x, const F *y, double *out, int nv, cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        launch_rows<F, NV, 1>(n, k::EDot<F, NV>{x, y, out}, s);
    });
}
template void dot<double>(uint64_t, const double *, const double *, double *, int, cudaStream_t);
template void dot<float>(uint64_t, const float *, const float *, double *, int, cudaStream_t);

void group2(uint64_t n, const double *t, const double *s_, double *out96, int nv,
            cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        launch_rows<double, NV, 3>(n, k::EGroup2<NV>{t, s_, out96}, s);
    });
}

void group4(uint64_t n, const double *s_, const double *t, const double *r0, double *r,
            double *x, const double *pa, const double *sa, bool with_x, double *sc, int nv,
            cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        if (with_x)
            launch_rows<double, NV, 1>(n, k::EGroup4<NV, true>{s_, t, r0, r, x, pa, sa, sc}, s);
        else
            launch_rows<double, NV, 1>(n, k::EGroup4<NV, false>{s_, t, r0, r, x, pa, sa, sc}, s);
    });
}

}  // namespace ops
}  // namespace xg
