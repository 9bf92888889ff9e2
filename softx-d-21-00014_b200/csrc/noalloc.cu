// XAMG_b200_dot_noalloc: the multi-RHS dot product of XAMG_b200_dot without
// any memory allocation.
//
// Who needs it: callers that cannot allocate device memory at the point where
// they need a reduction. Examples are host applications that hand all device
// memory to their own pool allocator up front, and latency-bound loops in
// which a cudaMalloc is not acceptable because it may synchronise the whole
// device or fail under memory pressure. The regular entry points allocate the
// library's working memory on first use; this one never does.
//
// How: the reduction's scratch (per-block partial sums and the completion
// counter) lives in one file-scope __device__ array below, present on every GPU
// that loads this library, for as long as the process runs. Host code never
// passes the array's name to a kernel (in host code that name is only a
// stand-in); the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current. XAMG_init does this for the
// library's device, and also loads the kernels this entry point launches, so
// that under CUDA's lazy module loading no call on that device loads code or
// maps the array. On any other device the first call does the lookup and the
// loading itself (which may allocate and synchronise), so make that first call
// before any stream capture and outside the region that must not allocate.
// Inputs and the output are the caller's device arrays.
//
// Limits: nv must be 1, 2, 4, 8, 16 or 32; the array holds 1184 x 32 partial
// sums (303,104 bytes) plus the counter, enough for every row count since the
// reduction uses at most 1184 blocks. Every call uses the same array, and the
// counter is cleared at the start of each call: two calls whose kernels overlap
// on the GPU (for example on two streams) race and give wrong results.
#include <type_traits>

#include "ops.h"

namespace xg {
namespace {

constexpr int NOALLOC_PARTIALS = k::BMAX * 32;         // doubles of partial sums
constexpr int NOALLOC_WORDS = NOALLOC_PARTIALS + 32;   // + counter area

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_WORDS];

constexpr int MAX_DEVICES = 64;
static double *g_scratch_addr[MAX_DEVICES];  // device address per device, set once

// Looks up the device address of g_noalloc_scratch for the current device.
int scratch_for_current_device(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return XAMG_ERR_CUDA;
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return XAMG_ERR_CUDA;
        g_scratch_addr[dev] = (double *)p;
    }
    *out = g_scratch_addr[dev];
    return XAMG_OK;
}

template <int NV>
cudaError_t load_dot_kernel() {
    cudaFuncAttributes a;
    return cudaFuncGetAttributes(&a, k::k_rows<double, NV, 1, k::EDot<double, NV>>);
}

template <int NV>
int launch_dot(uint64_t n, const double *x, const double *y, double *out, double *scratch,
               cudaStream_t s) {
    unsigned *ticket = (unsigned *)(scratch + NOALLOC_PARTIALS);
    if (cudaMemsetAsync(ticket, 0, sizeof(unsigned), s) != cudaSuccess) return XAMG_ERR_CUDA;
    const int B = k::canon_blocks(n, NV);
    k::k_rows<double, NV, 1, k::EDot<double, NV>>
        <<<B, k::CT, 0, s>>>(n, k::EDot<double, NV>{x, y, out}, k::RedArgs{scratch, ticket});
    return cudaGetLastError() == cudaSuccess ? XAMG_OK : XAMG_ERR_CUDA;
}

}  // namespace

// Called by the library's initialisation with its device current: resolves
// the array's address and loads every kernel the entry point can launch.
namespace ops {
int noalloc_prepare_current_device() {
    double *p = nullptr;
    int rc = scratch_for_current_device(&p);
    if (rc != XAMG_OK) return rc;
    const cudaError_t e[] = {load_dot_kernel<1>(), load_dot_kernel<2>(), load_dot_kernel<4>(),
                             load_dot_kernel<8>(), load_dot_kernel<16>(), load_dot_kernel<32>()};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return XAMG_ERR_CUDA;
    return XAMG_OK;
}
}  // namespace ops

}  // namespace xg

extern "C" int XAMG_b200_dot_noalloc(uint64_t n, int nv, const double *x, const double *y,
                                     double *dot_out, void *stream) {
    using namespace xg;
    if (!x || !y || !dot_out) return XAMG_ERR_INVALID_ARG;
    if (!nv_supported(nv)) return XAMG_ERR_INVALID_ARG;  // beyond the 32-RHS scratch
    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != XAMG_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        return cudaMemsetAsync(dot_out, 0, nv * sizeof(double), s) == cudaSuccess ? XAMG_OK
                                                                                  : XAMG_ERR_CUDA;
    }
    switch (nv) {
    case 1: return launch_dot<1>(n, x, y, dot_out, scratch, s);
    case 2: return launch_dot<2>(n, x, y, dot_out, scratch, s);
    case 4: return launch_dot<4>(n, x, y, dot_out, scratch, s);
    case 8: return launch_dot<8>(n, x, y, dot_out, scratch, s);
    case 16: return launch_dot<16>(n, x, y, dot_out, scratch, s);
    default: return launch_dot<32>(n, x, y, dot_out, scratch, s);
    }
}
