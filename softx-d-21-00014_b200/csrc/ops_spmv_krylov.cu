// SpMV kernels of the Krylov solvers (merged BiCGStab groups with
// their dot products) and the canonical-order vector reductions.
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

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

void spmv_dot_alpha(const DCsr &A, const float *pa, double *v, const double *r0, double *sc,
                    int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        launch<double, float, I, NV, 1>(A, pa, k::EDotAlpha<NV>{v, r0, sc}, s);
    });
}

void spmv_dot3(const DCsr &A, const float *sa, double *t, const double *s_, double *sc, int nv,
               cudaStream_t s) {
    XG_DISPATCH(A, nv, { launch<double, float, I, NV, 3>(A, sa, k::EDot3<NV>{t, s_, sc}, s); });
}

void pcg_ap(const DCsr &A, const double *p, double *Ap, double *sc, int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, { launch<double, double, I, NV, 1>(A, p, k::EPcgAp<NV>{Ap, p, sc}, s); });
}

void pcg_dots(uint64_t n, const double *r, const double *z, double *sc, bool first, int nv,
              cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        launch_rows<double, NV, 2>(n, k::EPcgDots<NV>{r, z, sc, first}, s);
    });
}

void rb_group1(uint64_t n, double *r, const double *v, const double *t, const double *r0,
               double *sc, int nv, cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        launch_rows<double, NV, 4>(n, k::ERbGroup1<NV>{r, v, t, r0, sc}, s);
    });
}

void spmv_dot3(const DCsr &A, const double *sa, double *t, const double *s_, double *sc, int nv,
               cudaStream_t s) {
    XG_DISPATCH(A, nv, { launch<double, double, I, NV, 3>(A, sa, k::EDot3<NV>{t, s_, sc}, s); });
}

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
            double *x, const float *pa, const float *sa, double *sc, int nv, cudaStream_t s) {
    dispatch_nv(nv, [&](auto nvc) {
        constexpr int NV = decltype(nvc)::value;
        launch_rows<double, NV, 1>(n, k::EGroup4<NV, true, float>{s_, t, r0, r, x, pa, sa, sc}, s);
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
