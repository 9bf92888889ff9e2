// x-staged CSR SpMV for irregular levels (gpu_index_compress >= 2).
//
// On a coarse level of an unstructured hierarchy the rows of a warp have
// unrelated columns, so every entry's gather of nv values of x lands in a
// 128-byte line of its own and the L1 data pipe serves one wavefront per
// entry and right-hand-side group; it is the limit there. Consecutive rows of
// a tile share most of their columns, though. This form keeps, per canonical
// tile of 256/nv rows, the tile's sorted unique columns (ucol) and for every
// entry its slot among them (slot, 16 bits). A block copies the tile's x rows
// once into shared memory (cp.async, contiguous runs of unique columns read
// contiguously), stages the tile's values and slots by bulk copy as k_spmv
// does, and sums each row from shared memory, in entry order: every output
// element is the CSR kernel's, bit for bit. Reading 16 bytes of a random x
// row from shared memory costs about a third of the wavefronts of a
// scattered 32-byte global gather.
#pragma once

#include "kernels.cuh"

namespace xg {
namespace k {

__device__ __forceinline__ void cp_async(void *dst, const void *src, int bytes) {
    const uint32_t d = smem_addr(dst);
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// VK consecutive x values of a staged row from shared memory (16-byte loads
// where VK values fill them).
template <typename FX, int VK>
__device__ __forceinline__ void ld_xs(const FX *p, FX (&o)[VK]) {
    if constexpr (std::is_same<FX, double>::value && VK % 2 == 0) {
#pragma unroll
        for (int h = 0; h < VK; h += 2) {
            const double2 t = *reinterpret_cast<const double2 *>(p + h);
            o[h] = t.x;
            o[h + 1] = t.y;
        }
    } else if constexpr (std::is_same<FX, float>::value && VK % 4 == 0) {
#pragma unroll
        for (int h = 0; h < VK; h += 4) {
            const float4 t = *reinterpret_cast<const float4 *>(p + h);
            o[h] = t.x;
            o[h + 1] = t.y;
            o[h + 2] = t.z;
            o[h + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int v = 0; v < VK; ++v) o[v] = p[v];
    }
}

struct XsArgs {
    const uint32_t *uptr;  // [ntiles + 1] offsets into ucol
    const uint32_t *ucol;  // unique columns of each tile, sorted
    const uint16_t *slot;  // [nnz] slot of each entry among its tile's columns
    uint32_t umax, emax;   // largest unique-column and entry counts of a tile
};

// Shared memory of one block: x rows (umax * NV of FX), then the staged
// values and slots (emax each, plus alignment slack).
template <typename FX, typename V, int NV>
__host__ __device__ inline uint32_t xs_smem_bytes(uint32_t umax, uint32_t emax) {
    auto r16 = [](uint32_t b) { return (b + 15u) & ~15u; };
    return r16(umax * NV * (uint32_t)sizeof(FX)) + r16(emax * (uint32_t)sizeof(V) + 32u) +
           r16(emax * 2u + 32u);
}

template <typename F, typename FX, int NV, int VK, class Epi, typename V = F>
__global__ void __launch_bounds__(CT / VK)
    k_spmv_xs(CsrArgs<F> A, XsArgs X, const FX *__restrict__ x, Epi epi, unsigned *flag) {
    constexpr int G = NV / VK;
    constexpr int R = CT / NV;
    constexpr int NT = CT / VK;
    constexpr int XB = NV * (int)sizeof(FX);     // bytes of one x row
    constexpr int CS = XB < 16 ? XB : 16;        // bytes a cp.async moves
    constexpr int CH = XB / CS;                  // copies per x row
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    const uint32_t XSB = (X.umax * (uint32_t)XB + 15u) & ~15u;
    const uint32_t VSB = (X.emax * (uint32_t)sizeof(V) + 32u + 15u) & ~15u;
    FX *xs = (FX *)smem_raw;
    V *vbuf = (V *)(smem_raw + XSB);
    uint16_t *sbuf = (uint16_t *)(smem_raw + XSB + VSB);
    const int rt = threadIdx.x / G, k0 = (threadIdx.x % G) * VK;
    const uint32_t *__restrict__ row = A.row;
    const V *__restrict__ val = (const V *)A.val;
    const uint64_t n = A.n;
    const uint64_t nnz = n ? row[n] : 0;
    const uint64_t ntiles = (n + R - 1) / R;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t phase = 0;
    bool timed_out = false;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t r0 = tile * R, r1 = r0 + R < n ? r0 + R : n;
        const uint32_t tj0 = __ldg(&row[r0]), tj1 = __ldg(&row[r1]);
        const uint32_t u0 = __ldg(&X.uptr[tile]), nu = __ldg(&X.uptr[tile + 1]) - u0;
        if (threadIdx.x == 0) {
            const V *vsrc;
            V *vdst;
            const uint16_t *ssrc;
            uint16_t *sdst;
            const uint32_t vb = stage_range<V>(vbuf, val, nnz, tj0, tj1, vsrc, vdst);
            const uint32_t sb = stage_range<uint16_t>(sbuf, X.slot, nnz, tj0, tj1, ssrc, sdst);
            mbar_arrive_expect(&mbar, vb + sb);  // releases the plain-load writes above
            fence_proxy_async_smem();
            if (vb) bulk_g2s(vdst, vsrc, vb, &mbar);
            if (sb) bulk_g2s(sdst, ssrc, sb, &mbar);
        }
        // the tile's x rows, unique columns in order
        for (uint32_t c = threadIdx.x; c < nu * CH; c += NT) {
            const uint32_t u = c / CH, part = c % CH;
            const uint32_t col = __ldg(&X.ucol[u0 + u]);
            cp_async((unsigned char *)xs + (size_t)u * XB + part * CS,
                     (const unsigned char *)x + (size_t)col * XB + part * CS, CS);
        }
        cp_async_wait_all();
        const bool ok = mbar_wait(&mbar, phase);
        // a copy that never landed: every thread of the block stops here
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        phase ^= 1u;
        const uint64_t i = r0 + rt;
        if (i < n) {
            F y[VK];
#pragma unroll
            for (int v = 0; v < VK; ++v) y[v] = epi.init(i, k0 + v);
            const uint32_t j0 = __ldg(&row[i]), j1 = __ldg(&row[i + 1]);
            const V *sv = vbuf + stage_shift<V>(val, tj0) + (j0 - tj0);
            const uint16_t *ss = sbuf + stage_shift<uint16_t>(X.slot, tj0) + (j0 - tj0);
#pragma unroll 4
            for (uint32_t j = 0; j < j1 - j0; ++j) {
                const F av = val_as<F, V>(sv[j]);
                FX xv[VK];
                ld_xs<FX, VK>(xs + (uint32_t)ss[j] * NV + k0, xv);
#pragma unroll
                for (int v = 0; v < VK; ++v) y[v] = add(y[v], mul((F)xv[v], av));
            }
            F none[1] = {F(0)};
#pragma unroll
            for (int v = 0; v < VK; ++v) epi.store(i, k0 + v, y[v], none);
        }
        __syncthreads();  // every reader is done with the tile's shared memory
    }
    if (timed_out && threadIdx.x == 0) {
        // raise the flag; no block exits with a copy into its shared memory
        // still in flight (bounded wait)
        atomicOr(flag, 1u);
        mbar_wait(&mbar, phase);
    }
}

}  // namespace k
}  // namespace xg
