// SpMV entry points for FP64: y = Ax, y += Ax; and the bounded-wait check.
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

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

}  // namespace ops
}  // namespace xg
