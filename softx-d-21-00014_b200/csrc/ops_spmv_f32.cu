// SpMV entry points for FP32: y = Ax, y += Ax, and the FP64 -> FP32 restriction.
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

template <typename F>
void spmv(const DCsr &A, const F *x, F *y, int nv, bool axpy, cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        if (axpy)
            launch<F, F, I, NV, 0, true>(A, x, k::EAxpy<F, NV>{{}, y}, s);
        else
            launch<F, F, I, NV, 0, true>(A, x, k::EStore<F, NV>{{}, y}, s);
    });
}
template void spmv<float>(const DCsr &, const float *, float *, int, bool, cudaStream_t);

void spmv_f32_from_f64(const DCsr &A, const double *x, float *y, int nv, cudaStream_t s) {
    XG_DISPATCH(A, nv, { launch<float, double, I, NV, 0>(A, x, k::EStore<float, NV>{{}, y}, s); });
}

}  // namespace ops
}  // namespace xg
