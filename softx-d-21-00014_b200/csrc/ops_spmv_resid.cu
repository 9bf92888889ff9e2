// SpMV kernels of the residual r = b - A x (with its norm for the Krylov
// level, without for the multigrid levels).
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

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

}  // namespace ops
}  // namespace xg
