// Launchers of the persistent preconditioned BiCGStab (k_pbicgstab_persist,
// csrc/kernels.cuh) and of its grid barrier's self-test.
#include "spmv_launch.cuh"

namespace xg {
namespace ops {

// The whole iteration runs as one cooperative launch: B = canon_blocks(n,
// nv) canonical blocks played by ceil(B / share) physical blocks (share =
// gpu_persistent: canonical blocks a physical block plays), which must be
// resident at once; the two halves of the partial-sum buffer must hold B x
// nv x 4 values each.
static int grid_of(int B, int share) { return (B + share - 1) / (share < 1 ? 1 : share); }

template <int NV, typename I>
static bool fits_nv(uint64_t n, int share) {
    const int B = k::canon_blocks(n, NV);
    if ((uint64_t)B * NV * 8 > (uint64_t)k::BMAX * 32 * 4) return false;
    const int res = resident_blocks(k::k_pbicgstab_persist<NV, I>, k::CT, 0);
    return (uint64_t)res * (uint64_t)ctx().sms >= (uint64_t)grid_of(B, share);
}

bool pbicgstab_persist_fits(const DCsr &A, int nv, int share) {
    bool ok = false;
    XG_DISPATCH(A, nv, { ok = fits_nv<NV, I>(A.nrows, share); });
    return ok;
}

void pbicgstab_persist(const DCsr &A, const k::PersistArgs &P, int nv, int share,
                       cudaStream_t s) {
    XG_DISPATCH(A, nv, {
        const int B = k::canon_blocks(A.nrows, NV);
        k::CsrArgs<double> a = A.args<double>();
        k::PersistArgs p = P;
        p.B = (uint32_t)B;
        void *args[] = {(void *)&a, (void *)&p};
        XG_CUDA(cudaLaunchCooperativeKernel((const void *)k::k_pbicgstab_persist<NV, I>,
                                            dim3((unsigned)grid_of(B, share)), dim3(k::CT), args,
                                            0, s));
        ++g_kernel_launches;
    });
}

void grid_selftest(unsigned *count_gen, unsigned *flag, uint64_t limit_ns, cudaStream_t s) {
    XG_CUDA(cudaMemsetAsync(count_gen, 0, 2 * sizeof(unsigned), s));
    k::GridSync g{reinterpret_cast<unsigned long long *>(count_gen), flag, limit_ns};
    const int blocks = 4;  // resident together on any GPU this library runs on
    void *args[] = {(void *)&g};
    XG_CUDA(cudaLaunchCooperativeKernel((const void *)k::k_grid_selftest, dim3(blocks), dim3(32),
                                        args, 0, s));
    ++g_kernel_launches;
}

}  // namespace ops
}  // namespace xg
