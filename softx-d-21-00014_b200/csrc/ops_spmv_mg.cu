// SpMV kernels of the other smoothers, the mixed-precision prolongation and
// the dense coarse solve.
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

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
        constexpr uint64_t RB = k::DT / NV;
        k::k_dense<F, NV><<<(unsigned)((n + RB - 1) / RB), k::DT, 0, s>>>(a, n, x, y);
        XG_CUDA(cudaGetLastError());
        ++g_kernel_launches;
    });
}
template void dense_apply<double>(const double *, uint64_t, const double *, double *, int,
                                  cudaStream_t);
template void dense_apply<float>(const float *, uint64_t, const float *, float *, int,
                                 cudaStream_t);


}  // namespace ops
}  // namespace xg
