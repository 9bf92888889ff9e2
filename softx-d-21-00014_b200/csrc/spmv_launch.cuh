// Launch helpers of the CSR kernels, shared by the ops_spmv*.cu files:
// runtime (nv, column width) -> template instantiation of k_spmv with the
// matching epilogue.
#pragma once

#include <algorithm>
#include <map>
#include <tuple>
#include <type_traits>

#include "ops.h"
#include "stencil.cuh"
#include "xstage.cuh"

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
// alignment slack). Two buffers let the copy of a block's next tile overlap
// its current one, one buffer lets more blocks share an SM: the launcher
// takes two unless that lowers the number of resident blocks (measured on the
// 27-point 128^3 matrix: nv = 4 runs 10 % faster on one buffer and twice the
// blocks, nv = 8 and 16 about 10 % faster on two at equal blocks). Buffers
// hold at most 96 KB.
template <typename F, typename I>
static uint32_t stage_buffer_bytes(uint32_t cap) {
    auto r16 = [](uint64_t b) { return (uint32_t)((b + 15) & ~(uint64_t)15); };
    return r16((uint64_t)cap * sizeof(F) + 32) + r16((uint64_t)cap * sizeof(I) + 32);
}

// Resident blocks per SM of a kernel for a dynamic shared-memory size
// (remembered per kernel and size).
template <class Kern>
static int resident_blocks(Kern kern, int threads, size_t smem) {
    static std::map<std::pair<const void *, size_t>, int> cache;
    const auto key = std::make_pair((const void *)kern, smem);
    auto it = cache.find(key);
    if (it == cache.end()) {
        int nb = 0;
        XG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem));
        it = cache.emplace(key, std::max(nb, 1)).first;
    }
    return it->second;
}

// Grid: as many blocks as fit the GPU at once (one wave). With dot products
// the tiles still go to the canonical B = min(ntiles, 1184) blocks, which the
// grid's blocks run in turn; without, the grid's blocks take the tiles.
// run RUN_WALK (no dot products): the plane walk, each block taking one
// run of consecutive walk positions, the runs as even as the grid allows.
constexpr uint32_t RUN_WALK = 0xFFFFFFFFu;
// The plane walk's stride in tiles of R rows (0: the matrix has none, or
// too few tiles for two planes).
inline uint32_t walk_stride(const DCsr &A, uint64_t R) {
    if (!A.walk_rows) return 0;
    const uint64_t S = (A.walk_rows + R / 2) / R;
    const uint64_t ntiles = (A.nrows + R - 1) / R;
    return S >= 2 && ntiles >= 2 * S ? (uint32_t)S : 0u;
}

template <typename F, typename FX, typename I, int NV, int VK, int NRED, typename V = F,
          class Epi>
static void launch_vk(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s,
                      uint32_t nbuf_force = 0, uint32_t run = 1) {
    constexpr uint32_t LIMIT1 = (96u * 1024u - 64u) / (uint32_t)(sizeof(V) + sizeof(I));
    constexpr int NT = k::CT / VK;
    // the kernel forms x offsets c*NV + k and row indices in 32 bits
    XG_REQUIRE(std::max(A.ncols, A.nrows) * (uint64_t)NV < (1ull << 32), XAMG_ERR_UNSUPPORTED,
               "SpMV: x of 2^32 or more values");
    auto kern = k::k_spmv<F, FX, I, NV, VK, NRED, Epi, V>;
    static bool big_smem = false;  // one flag per instantiation
    if (!big_smem) {
        XG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)stage_buffer_bytes<V, I>(LIMIT1)));
        big_smem = true;
    }
    // nbuf_force 3: no staging (every tile reads global memory)
    const uint32_t cap = nbuf_force == 3 ? 0u : std::min(tile_max(A, NV, s), LIMIT1);
    const size_t one = stage_buffer_bytes<V, I>(cap);
    const int res1 = resident_blocks(kern, NT, one);
    uint32_t nbuf = 1;
    int res = res1;
    if (2 * one <= (size_t)stage_buffer_bytes<V, I>(LIMIT1)) {
        const int res2 = resident_blocks(kern, NT, 2 * one);
        if ((nbuf_force == 0 && res2 >= res1) || nbuf_force == 2) {
            nbuf = 2;
            res = res2;
        }
    }
    const size_t smem = nbuf * one;
    const uint64_t R = k::CT / NV;
    const uint64_t ntiles = (A.nrows + R - 1) / R;
    const uint64_t wave = (uint64_t)res * (uint64_t)ctx().sms;
    uint32_t stride = 0;
    if (NRED == 0 && run == RUN_WALK) {
        stride = walk_stride(A, R);
        run = (uint32_t)std::max<uint64_t>(1, (ntiles + wave - 1) / wave);
    }
    if (NRED > 0 || run < 1) run = 1;
    const uint32_t B = NRED > 0 ? (uint32_t)k::canon_blocks(A.nrows, NV)
                                : (uint32_t)std::min<uint64_t>((ntiles + run - 1) / run, wave);
    const uint32_t P = (uint32_t)std::min<uint64_t>(B, wave);
    kern<<<P, NT, smem, s>>>(A.args<F>(), x, epi, ctx().red(), cap, nbuf, B, run, stride);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

// The warp-per-row kernel (k_spmv_wide): one wave of 256-thread blocks.
template <typename F, typename FX, typename I, int NV, typename V, class Epi>
static void launch_wide(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s) {
    XG_REQUIRE(std::max(A.ncols, A.nrows) * (uint64_t)NV < (1ull << 32), XAMG_ERR_UNSUPPORTED,
               "SpMV: x of 2^32 or more values");
    auto kern = k::k_spmv_wide<F, FX, I, NV, Epi, V>;
    const int res = resident_blocks(kern, k::WT, 0);
    const uint64_t need = (A.nrows + k::WT / 32 - 1) / (k::WT / 32);
    const uint32_t P = (uint32_t)std::min<uint64_t>(need, (uint64_t)res * ctx().sms);
    kern<<<P, k::WT, 0, s>>>(A.args<F>(), x, epi);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}
// The x-staged kernel (k_spmv_xs) on a matrix's x-staged copy for NV: one
// wave of persistent blocks over the canonical tiles.
template <typename F, typename FX, int NV, typename V, class Epi>
static void launch_xs(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s) {
    constexpr int VK = k::spmv_vk<FX, NV>();
    constexpr int NT = k::CT / VK;
    XG_REQUIRE(std::max(A.ncols, A.nrows) * (uint64_t)NV < (1ull << 32), XAMG_ERR_UNSUPPORTED,
               "SpMV: x of 2^32 or more values");
    auto kern = k::k_spmv_xs<F, FX, NV, VK, Epi, V>;
    const uint32_t smem = k::xs_smem_bytes<FX, V, NV>(A.xs_umax, A.xs_emax);
    static uint32_t attr = 48 * 1024;  // dynamic shared memory allowed so far (per instantiation)
    if (smem > attr) {
        XG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     96 * 1024));
        attr = 96 * 1024;
    }
    const int res = resident_blocks(kern, NT, smem);
    const uint64_t R = k::CT / NV;
    const uint64_t ntiles = (A.nrows + R - 1) / R;
    const uint32_t P = (uint32_t)std::min<uint64_t>(ntiles, (uint64_t)res * ctx().sms);
    const k::XsArgs xa{A.xs_uptr.as<uint32_t>(), A.xs_ucol.as<uint32_t>(),
                       A.xs_slot.as<uint16_t>(), A.xs_umax, A.xs_emax};
    kern<<<P, NT, smem, s>>>(A.args<F>(), xa, x, epi, ctx().red().flag);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

// Whether the x-staged kernel can take this SpMV: a copy built for NV, x
// aligned for its vector loads, the block's shared memory within 96 KB (an
// x type wider than the level's, as in the FP64-to-FP32 restriction, needs
// more than the upload checked).
template <typename FX, typename V, int NV>
static bool xs_usable(const DCsr &A, const FX *x) {
    return A.xs_nv == NV && (uintptr_t)x % (k::spmv_vk<FX, NV>() * sizeof(FX)) == 0 &&
           k::xs_smem_bytes<FX, V, NV>(A.xs_umax, A.xs_emax) <= 96u * 1024u;
}

constexpr uint8_t TUNE_WIDE = 28;         // autotuner code of the warp-per-row kernel
constexpr uint64_t WIDE_MAX_VALUES = 1u << 20;  // rows * nv up to which it is a candidate

// Autotuner of the SpMVs without dot products: the right-hand sides a thread
// carries (2 or 4; the alternative of spmv_vk's choice; 8 for FP32 x at
// nv >= 8), the staging buffers
// (1, 2, or none: tiles read from global memory, for small matrices where the
// copy's round trip is not hidden) and the run of consecutive tiles a block
// takes (1, 4 or 16, or the plane walk where the matrix has a walk stride) are
// timed with CUDA events on the caller's x into a scratch y (EStore), once
// per matrix, precision and nv, outside any graph capture; the fastest is
// kept in the matrix (DCsr::tuned). Matrices of at most WIDE_MAX_VALUES rows
// times nv also time the warp-per-row kernel (code TUNE_WIDE). Every candidate
// sums each (row, right-hand side) in the same CSR order, so the choice never
// changes a result.
constexpr uint32_t TUNE_RUNS[3] = {1, 4, 16};
struct Tuned {
    int alt;
    uint32_t nbuf, run;
};
constexpr uint8_t TUNE_WALK0 = 29;  // first code of the plane walk (29..37)
inline Tuned tuned_shape(uint8_t code) {
    if (code >= TUNE_WALK0) {
        const int c = code - TUNE_WALK0;
        return Tuned{c / 3, (uint32_t)(c % 3 + 1), RUN_WALK};
    }
    const int c = code - 1;
    return Tuned{c / 9, (uint32_t)((c / 3) % 3 + 1), TUNE_RUNS[c % 3]};
}
// Eight right-hand sides a thread (one thread a row at nv = 8): a third
// shape the autotuner times for FP32 x and nv >= 8, halving the shared-memory
// reads of each staged (column, value) pair against four a thread.
template <typename FX, int NV, int NRED>
constexpr bool spmv_has_vk8() {
    return std::is_same<FX, float>::value && NV >= 8 && NRED == 0;
}

template <typename FX, int NV>
constexpr int spmv_vk_alt() {
    constexpr int d = k::spmv_vk<FX, NV>();
    constexpr int a = d == 2 ? 4 : d == 4 ? 2 : d;
    return a <= NV ? a : d;
}

template <typename F, typename FX, typename I, int NV, typename V>
static uint8_t autotune(const DCsr &A, const FX *x, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    XG_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return 0;
    constexpr int VD = k::spmv_vk<FX, NV>();
    constexpr int VA = spmv_vk_alt<FX, NV>();
    DevBuf y(A.nrows * (uint64_t)NV * sizeof(F));
    k::EStore<F, NV> e{{}, y.as<F>()};
    cudaEvent_t e0, e1;
    XG_CUDA(cudaEventCreate(&e0));
    XG_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    uint8_t code = 1;
    constexpr bool V8 = spmv_has_vk8<FX, NV, 0>() && VD != 8 && VA != 8;
    // run index 3: the plane walk, where the matrix has one at this nv
    const int nruns = walk_stride(A, (uint64_t)(k::CT / NV)) ? 4 : 3;
    for (int alt = 0; alt < 3; ++alt)
        for (uint32_t nb = 1; nb <= 3; ++nb)
            for (int ri = 0; ri < nruns; ++ri) {
                if ((alt == 1 && VA == VD) || (alt == 2 && !V8)) continue;
                const uint32_t run = ri == 3 ? RUN_WALK : TUNE_RUNS[ri];
                auto go = [&] {
                    if (alt == 2) {
                        if constexpr (V8) launch_vk<F, FX, I, NV, 8, 0, V>(A, x, e, s, nb, run);
                    } else if (alt) {
                        launch_vk<F, FX, I, NV, VA, 0, V>(A, x, e, s, nb, run);
                    } else {
                        launch_vk<F, FX, I, NV, VD, 0, V>(A, x, e, s, nb, run);
                    }
                };
                // the faster of two rounds of three launches, after one untimed
                float ms = 1e30f;
                go();
                for (int round = 0; round < 2; ++round) {
                    XG_CUDA(cudaEventRecord(e0, s));
                    for (int r = 0; r < 3; ++r) go();
                    XG_CUDA(cudaEventRecord(e1, s));
                    XG_CUDA(cudaEventSynchronize(e1));
                    float t = 0;
                    XG_CUDA(cudaEventElapsedTime(&t, e0, e1));
                    ms = std::min(ms, t);
                }
                if (ms < best) {
                    best = ms;
                    code = ri == 3 ? (uint8_t)(TUNE_WALK0 + alt * 3 + (nb - 1))
                                   : (uint8_t)(1 + alt * 9 + (nb - 1) * 3 + ri);
                }
            }
    if (A.nrows * (uint64_t)NV <= WIDE_MAX_VALUES) {
        auto go = [&] { launch_wide<F, FX, I, NV, V>(A, x, e, s); };
        float ms = 1e30f;
        go();
        for (int round = 0; round < 2; ++round) {
            XG_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < 3; ++r) go();
            XG_CUDA(cudaEventRecord(e1, s));
            XG_CUDA(cudaEventSynchronize(e1));
            float t = 0;
            XG_CUDA(cudaEventElapsedTime(&t, e0, e1));
            ms = std::min(ms, t);
        }
        if (ms < best) {
            best = ms;
            code = TUNE_WIDE;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    XG_CUDA(cudaStreamSynchronize(s));
    return code;
}

// Vector loads of x need x aligned to VK elements; library vectors always are
// (cudaMalloc). The entry points that take a caller's x (CALLER_X) fall back
// to one right-hand side per thread for an x that is not (same results, same
// reduction order).
// FP64 x on short rows (fewer than 16 entries on average: 7-point stencils
// and the like) takes four right-hand sides per thread: the staging buffers
// are small enough for sixteen 64-thread blocks an SM, and the wider gathers
// win; longer rows keep two.
template <typename F, typename FX, typename I, int NV, int NRED, bool CALLER_X, typename V,
          class Epi>
static void launch_v(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s) {
    // With dot products the grid is the canonical 1,184 blocks (one wave at
    // eight an SM), so the threads a block has are the warps an SM keeps in
    // flight: such kernels carry at most two right-hand sides a thread (FP32 x
    // at four a thread measured 35 % slower on the 27-point 128^3 matrix).
    constexpr int VK = NRED > 0 ? std::min(k::spmv_vk<FX, NV>(), 2) : k::spmv_vk<FX, NV>();
    if constexpr (NRED == 0) {
        if (A.wide_force && A.nrows * (uint64_t)NV <= WIDE_MAX_VALUES) {
            launch_wide<F, FX, I, NV, V>(A, x, epi, s);
            return;
        }
        if constexpr (!std::is_same<V, __half>::value)
            if (A.xs_force && xs_usable<FX, V, NV>(A, x)) {
                launch_xs<F, FX, NV, V>(A, x, epi, s);
                return;
            }
        if (A.walk_force && walk_stride(A, (uint64_t)(k::CT / NV)) &&
            (VK == 1 || (uintptr_t)x % (VK * sizeof(FX)) == 0)) {
            launch_vk<F, FX, I, NV, VK, NRED, V>(A, x, epi, s, 0, RUN_WALK);
            return;
        }
    }
    if constexpr (NRED == 0 && NV > 1) {
        if (A.tune_on && (uintptr_t)x % (4 * sizeof(FX)) == 0) {
            int l = 0;
            while ((1 << l) < NV) ++l;
            uint8_t &t = A.tuned[sizeof(F) == 4][sizeof(FX) == 4][l];
            if (!t) t = autotune<F, FX, I, NV, V>(A, x, s);
            if (t == TUNE_WIDE) {
                launch_wide<F, FX, I, NV, V>(A, x, epi, s);
                return;
            }
            if (t) {
                const Tuned c = tuned_shape(t);
                if constexpr (spmv_has_vk8<FX, NV, NRED>() && VK != 8 &&
                              spmv_vk_alt<FX, NV>() != 8) {
                    if (c.alt == 2) {
                        launch_vk<F, FX, I, NV, 8, NRED, V>(A, x, epi, s, c.nbuf, c.run);
                        return;
                    }
                }
                if (c.alt)
                    launch_vk<F, FX, I, NV, spmv_vk_alt<FX, NV>(), NRED, V>(A, x, epi, s,
                                                                           c.nbuf, c.run);
                else
                    launch_vk<F, FX, I, NV, VK, NRED, V>(A, x, epi, s, c.nbuf, c.run);
                return;
            }
        }
    }
    constexpr uintptr_t ALIGN = VK * sizeof(FX);
    constexpr bool SHORT4 = sizeof(FX) == 8 && VK == 2 && NV >= 4 && NRED == 0;
    if (SHORT4 && A.nnz < 16 * A.nrows && (uintptr_t)x % (4 * sizeof(FX)) == 0) {
        if constexpr (SHORT4) launch_vk<F, FX, I, NV, 4, NRED, V>(A, x, epi, s);
    } else if (VK == 1 || (uintptr_t)x % ALIGN == 0) {
        launch_vk<F, FX, I, NV, VK, NRED, V>(A, x, epi, s);
    } else if constexpr (CALLER_X) {
        launch_vk<F, FX, I, NV, 1, NRED, V>(A, x, epi, s);
    } else {
        throw Error(XAMG_ERR_INTERNAL, "library vector not aligned for the SpMV gather");
    }
}

// The grid-stencil kernel (csrc/stencil.cuh) on a matrix's stencil copy: M
// grid lines a thread, as many right-hand sides a thread as the CSR kernel
// carries; one wave of persistent blocks over the tiles, two staging buffers
// a block unless that lowers the resident blocks or does not fit.
template <typename F, int NV, typename V, int PAT, int MINB, class Epi>
static void launch_stencil_p(const DCsr &A, const F *x, const Epi &epi, cudaStream_t s) {
    constexpr int VK = k::spmv_vk<F, NV>();
    constexpr int G = NV / VK;
    constexpr int M = k::ST_LINES;
    constexpr uint32_t TX = k::st_tx<G>();
    constexpr uint32_t BUF = k::st_buffer_bytes<V, G, M, PAT>();
    constexpr uint32_t SMEM_MAX = 227u * 1024u;
    static_assert(BUF <= SMEM_MAX, "stencil staging buffer exceeds shared memory");
    constexpr bool TWO = 2 * BUF <= SMEM_MAX;
    XG_REQUIRE(A.nrows * (uint64_t)NV < (1ull << 32), XAMG_ERR_UNSUPPORTED,
               "SpMV: x of 2^32 or more values");
    auto kern = k::k_spmv_stencil<F, F, NV, VK, M, PAT, MINB, Epi, V>;
    static bool big_smem = false;  // one flag per instantiation
    if (!big_smem) {
        XG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(TWO ? 2 * BUF : BUF)));
        big_smem = true;
    }
    const int res1 = resident_blocks(kern, k::ST_THREADS, BUF);
    const int res2 = TWO ? resident_blocks(kern, k::ST_THREADS, 2 * BUF) : 0;
    const uint32_t nbuf = res2 >= res1 ? 2 : 1;
    const int res = nbuf == 2 ? res2 : res1;
    const uint64_t chunks = (A.st_S + TX - 1) / TX;
    const uint64_t groups = (A.nrows + (uint64_t)M * A.st_S - 1) / ((uint64_t)M * A.st_S);
    const uint64_t ntiles = groups * chunks;
    const uint32_t P = (uint32_t)std::min<uint64_t>(ntiles, (uint64_t)res * ctx().sms);
    const k::StencilArgs a{A.st_val.p,  A.st_mask.as<uint32_t>(), (uint32_t)A.nrows, A.st_S,
                           A.st_S2,     A.st_SP,                  A.st_slot,
                           A.st_diag_first ? 1 : 0};
    kern<<<P, k::ST_THREADS, nbuf * BUF, s>>>(a, x, epi, nbuf, ctx().red().flag);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}
// regs: 0 the 64-register form, 1 the 128-register form
template <typename F, int NV, typename V, class Epi>
static void launch_stencil(const DCsr &A, const F *x, const Epi &epi, cudaStream_t s, int regs) {
    if (A.st_pat == k::ST_BOX27) {
        if (regs)
            launch_stencil_p<F, NV, V, k::ST_BOX27, 4>(A, x, epi, s);
        else
            launch_stencil_p<F, NV, V, k::ST_BOX27, 8>(A, x, epi, s);
    } else {
        if (regs)
            launch_stencil_p<F, NV, V, k::ST_STAR7, 4>(A, x, epi, s);
        else
            launch_stencil_p<F, NV, V, k::ST_STAR7, 8>(A, x, epi, s);
    }
}

// Stencil or CSR (DCsr::st_choice): on matrices with a grid-stencil copy and
// tuning on, the first SpMV without dot products for each precision and nv
// times y = A x (EStore into a scratch y, the caller's x) with the stencil
// kernel's two register budgets and with the CSR kernel's tuned shape (the
// faster of two rounds of three launches each, outside any graph capture).
// A stencil form is kept only when it is at least ST_MARGIN faster than the
// CSR kernel: the smoothers' epilogues read and write more vectors than the
// timed y = A x, which costs the register-heavy stencil kernel more
// (measured in the 128^3 solve: its Chebyshev steps 13 % slower than CSR at
// equal y = A x times). All give the same results bit for bit.
constexpr float ST_MARGIN = 0.9f;
constexpr uint8_t ST_USE64 = 1, ST_USE128 = 2, ST_USE_CSR = 3;
template <typename F, typename I, int NV, bool CALLER_X>
static uint8_t tune_stencil(const DCsr &A, const F *x, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    XG_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return 0;
    DevBuf y(A.nrows * (uint64_t)NV * sizeof(F));
    k::EStore<F, NV> e{{}, y.as<F>()};
    cudaEvent_t e0, e1;
    XG_CUDA(cudaEventCreate(&e0));
    XG_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    uint8_t code = ST_USE64;
    for (uint8_t c = ST_USE64; c <= ST_USE_CSR; ++c) {
        auto go = [&] {
            if (c == ST_USE_CSR) {
                if constexpr (std::is_same<F, float>::value)
                    if (A.bf16) {
                        launch_v<F, F, I, NV, 0, CALLER_X, __nv_bfloat16>(A, x, e, s);
                        return;
                    }
                launch_v<F, F, I, NV, 0, CALLER_X, F>(A, x, e, s);
            } else if constexpr (std::is_same<F, float>::value) {
                if (A.bf16)
                    launch_stencil<F, NV, __nv_bfloat16>(A, x, e, s, c == ST_USE128);
                else
                    launch_stencil<F, NV, F>(A, x, e, s, c == ST_USE128);
            } else {
                launch_stencil<F, NV, F>(A, x, e, s, c == ST_USE128);
            }
        };
        float ms = 1e30f;
        go();  // untimed (tunes the CSR shape on its first call)
        for (int round = 0; round < 2; ++round) {
            XG_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < 3; ++r) go();
            XG_CUDA(cudaEventRecord(e1, s));
            XG_CUDA(cudaEventSynchronize(e1));
            float t = 0;
            XG_CUDA(cudaEventElapsedTime(&t, e0, e1));
            ms = std::min(ms, t);
        }
        if (ms < best) {
            best = ms;
            code = c;
        }
        if (c == ST_USE_CSR && code != ST_USE_CSR && best > ST_MARGIN * ms) code = ST_USE_CSR;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    XG_CUDA(cudaStreamSynchronize(s));
    return code;
}

// FP32 matrices may store their values in BF16 (DCsr::bf16; gpu_level_bf16):
// the kernel then widens each value to float as it reads it. SpMVs without
// dot products on a matrix with a grid-stencil copy run the stencil kernel
// (the same sums) unless the autotuner measured the CSR kernel faster.
template <typename F, typename FX, typename I, int NV, int NRED, bool CALLER_X = false,
          class Epi>
static void launch(const DCsr &A, const FX *x, const Epi &epi, cudaStream_t s) {
    if (A.nrows == 0) return;
    if constexpr (NRED == 0 && std::is_same<F, FX>::value) {
        constexpr uintptr_t SA = k::spmv_vk<F, NV>() * sizeof(F);
        if (A.st_pat >= 0 && (!CALLER_X || (uintptr_t)x % SA == 0)) {
            int choice = A.st_force ? A.st_force : ST_USE64;
            if (A.tune_on) {
                int l = 0;
                while ((1 << l) < NV) ++l;
                uint8_t &c = A.st_choice[sizeof(F) == 4][l];
                if (!c) c = tune_stencil<F, I, NV, CALLER_X>(A, x, s);
                if (c) choice = c;
            }
            if (choice != ST_USE_CSR) {
                if constexpr (std::is_same<F, float>::value)
                    if (A.bf16) {
                        launch_stencil<F, NV, __nv_bfloat16>(A, x, epi, s, choice == ST_USE128);
                        return;
                    }
                launch_stencil<F, NV, F>(A, x, epi, s, choice == ST_USE128);
                return;
            }
        }
    }
    if constexpr (std::is_same<F, float>::value && std::is_same<FX, float>::value) {
        if (A.bf16) {
            launch_v<F, FX, I, NV, NRED, CALLER_X, __nv_bfloat16>(A, x, epi, s);
            return;
        }
        if (A.fp16) {
            launch_v<F, FX, I, NV, NRED, CALLER_X, __half>(A, x, epi, s);
            return;
        }
    }
    XG_REQUIRE(!A.bf16 && !A.fp16, XAMG_ERR_UNSUPPORTED,
               "16-bit matrix values need float values and a float x");
    launch_v<F, FX, I, NV, NRED, CALLER_X, F>(A, x, epi, s);
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
}  // namespace ops
}  // namespace xg
