// SpMV kernels of the Chebyshev smoother.
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

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

}  // namespace ops
}  // namespace xg
