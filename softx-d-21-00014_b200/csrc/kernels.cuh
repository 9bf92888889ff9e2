// Device kernels of the solve phase (sm_100a).
//
// Layout: every n-vector with nv right-hand sides is stored row-major
// interleaved, element (i, k) at i*NV + k, as XAMG stores it
// (src/primitives/vector/vector.h:509-525). CSR blocks keep 32-bit row
// pointers, XAMG-narrowed column indices (u8/u16/u32) and float or double
// values.
//
// Arithmetic: products and sums use the round-to-nearest intrinsics
// (__dmul_rn, __dadd_rn, ...), which the compiler never contracts into FMA,
// and each row is accumulated in the reference's order (entry by entry, from
// 0 for y = Ax, from y for y += Ax). Every element a kernel writes therefore
// equals, bit for bit, what the reference's -ffp-contract=off CPU loop
// computes.
//
// Row schedule ("canonical order"): a block has 256 threads; thread t works on
// row slot t/NV and right-hand side t%NV, so a tile covers 256/NV consecutive
// rows and consecutive threads read consecutive x entries of a row. (The SpMV
// runs these 256 canonical threads on 256/VK physical ones, each carrying VK
// consecutive right-hand sides; see canon_finish.) Tiles are
// dealt round-robin to B = min(ntiles, 1184) blocks (8 per SM on 148 SMs).
// Dot products are accumulated per thread in tile order, combined within a
// warp by an xor butterfly (offsets 16..NV), across the 8 warps in warp
// order, and across blocks by the last block to finish: lane l sums blocks
// l, l+32, ... and a full butterfly finishes. The order depends only on
// (n, NV), so results are reproducible run to run and the CPU oracle can
// replay it exactly.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

namespace xg {
namespace k {

constexpr int CT = 256;     // threads per block
constexpr int BMAX = 1184;  // block cap of the canonical schedule

// ---------------------------------------------------------------------------
// Separately rounded arithmetic
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int off) {
    return __shfl_xor_sync(0xffffffffu, v, off);
}

template <typename T>
__device__ __forceinline__ T ld_cg(const T *p) {
    return __ldcg(p);
}

// ---------------------------------------------------------------------------
// Per-solver scalar block: NV-wide FP64 scalars of the Krylov recurrences,
// kept in device memory so that no kernel waits on the host for them.
// ---------------------------------------------------------------------------
enum Sc : int {
    SC_RHO = 0,
    SC_RHO0,
    SC_RES,
    SC_ALPHA,
    SC_OMEGA,
    SC_BETA,
    SC_PHI,
    SC_PSI,
    SC_THETA,
    SC_SCAL1,
    SC_SCAL2,
    SC_SCAL3,
    SC_SCAL4,
    SC_ICONV,
    SC_ALPHA_C,
    SC_OMEGA_C,
    SC_NSCAL,  // -(omega*beta), the v coefficient of the p update
    SC_RELAX,
    SC_ETA,    // (r, r) of the reordered BiCGStab
    SC_COUNT
};
constexpr int SC_STRIDE = 32;

__host__ __device__ inline int canon_rows_per_tile(int nv) { return CT / nv; }

inline int canon_blocks(uint64_t n, int nv) {
    const uint64_t R = CT / nv;
    const uint64_t nt = (n + R - 1) / R;
    return (int)(nt < (uint64_t)BMAX ? (nt == 0 ? 1 : nt) : (uint64_t)BMAX);
}

// ---------------------------------------------------------------------------
// Canonical reduction: block partials, then the last block finishes.
// ---------------------------------------------------------------------------
struct RedArgs {
    void *part;              // [BMAX][32][4] partial sums (element type of the kernel)
    unsigned *ticket;        // zero between launches
    unsigned *flag = nullptr;  // bit 0: a bounded wait ran out (read by the host)
};

// A block may run the 256 canonical threads with CT/VK physical threads:
// physical thread p plays canonical threads p*VK .. p*VK+VK-1 (right-hand
// sides k0 .. k0+VK-1 of one row slot) and keeps one accumulator per
// canonical thread. Canonical warp w is then physical threads
// [w*32/VK, (w+1)*32/VK), and a canonical butterfly offset `off` (a multiple
// of VK, since off >= NV >= VK) is the physical offset off/VK, so every sum is
// formed from the same operands in the same order as with VK = 1.
//
// canon_partial: the block's sum of canonical block cb's accumulators into
// part[cb] (called by every thread; zeroes acc). A physical block may run
// several canonical blocks one after the other.
template <typename T, int NV, int NRED, int VK>
__device__ __forceinline__ void canon_partial(T (&acc)[VK][NRED], const RedArgs &ra, uint32_t cb) {
    constexpr int NT = CT / VK;   // physical threads of the block
    constexpr int SUB = 32 / VK;  // physical threads of one canonical warp
    constexpr int G = NV / VK;    // physical threads of one row slot
    __shared__ T wsum[8 * NV * NRED];
    T *part = (T *)ra.part;
    const int cw = threadIdx.x / SUB, cl = threadIdx.x % SUB;  // canonical lane = cl*VK + v
#pragma unroll
    for (int v = 0; v < VK; ++v) {
#pragma unroll
        for (int r = 0; r < NRED; ++r) {
            T s = acc[v][r];
#pragma unroll
            for (int off = 16; off >= NV; off >>= 1) s = add(s, shfl_xor(s, off / VK));
            if (cl < G) wsum[(cw * NV + cl * VK + v) * NRED + r] = s;
            acc[v][r] = T(0);
        }
    }
    __syncthreads();
    for (int o = threadIdx.x; o < NV * NRED; o += NT) {  // o = k*NRED + r
        T s = wsum[o];
#pragma unroll
        for (int w = 1; w < 8; ++w) s = add(s, wsum[w * NV * NRED + o]);
        part[(size_t)cb * NV * NRED + o] = s;
    }
    __syncthreads();  // wsum is free for the next canonical block
}

// canon_final: after all of a launch's partials are written, the last
// physical block to arrive sums the B partials (lane l sums l, l+32, ...,
// then a full butterfly) and calls fin(k, sums of k).
template <typename T, int NV, int NRED, int NT, class Fin>
__device__ __forceinline__ void canon_final(const RedArgs &ra, uint32_t B, const Fin &fin) {
    constexpr int NW = NT / 32;
    __shared__ T sums[NV * NRED];
    __shared__ int is_last;
    const T *part = (const T *)ra.part;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(ra.ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    for (int o = warp; o < NV * NRED; o += NW) {
        T a = T(0);
        for (unsigned bb = lane; bb < B; bb += 32)
            a = add(a, ld_cg(&part[(size_t)bb * NV * NRED + o]));
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) a = add(a, shfl_xor(a, off));
        if (lane == 0) sums[o] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ra.ticket = 0u;
    for (int kk = threadIdx.x; kk < NV; kk += NT) fin(kk, &sums[kk * NRED]);
}

// One canonical block per physical block (256 threads).
template <typename T, int NV, int NRED, class Fin>
__device__ __forceinline__ void canon_finish(T (&acc)[NRED], const RedArgs &ra, const Fin &fin) {
    canon_partial<T, NV, NRED, 1>(reinterpret_cast<T(&)[1][NRED]>(acc), ra, blockIdx.x);
    canon_final<T, NV, NRED, CT>(ra, gridDim.x, fin);
}

// ---------------------------------------------------------------------------
// CSR SpMV with a compile-time epilogue.
//   acc = epi.init(i,k); for j in row i: acc = acc + x[col[j]*NV+k] * val[j]
//   epi.store(i, k, acc, terms[NRED])
// FX is the element type x is stored in; it is converted to F on load (the
// fused form of vector::convert before a reduced-precision restriction).
// ---------------------------------------------------------------------------
template <typename F>
struct CsrArgs {
    const uint32_t *row;
    const void *col;
    const F *val;
    uint64_t n;
    float vscale = 1.0f;  // FP16-stored values: the level's power-of-two scale
};

// Shared-memory staging: a tile's entries [row[r0], row[r0+R]) (values and
// columns in their stored types) are copied into shared memory by the bulk
// copy engine (cp.async.bulk, completion on an mbarrier), double-buffered so
// that the copy of a block's next tile overlaps the work on the current one;
// every thread then walks its own row from shared memory. The copy takes the
// 16-byte-aligned part of each array range; the few entries outside it (at an
// array's unaligned start or end) are copied with plain loads by the issuing
// thread before it arrives on the barrier. Tiles with more entries than the
// staging capacity read global memory directly.

// Column index of entry j: narrowed absolute index (I unsigned) or, for
// I = int16_t, a signed offset from the row index (the 2-byte relative form
// used where every |col - row| < 32768).
template <typename I>
__device__ __forceinline__ uint64_t col_at(I c, uint64_t i) {
    if constexpr (std::is_same<I, int16_t>::value)
        return (uint64_t)((int64_t)i + (int64_t)c);
    else
        return (uint64_t)c;
}

// Right-hand sides one SpMV thread carries: x[c*NV + k0 .. k0+VK-1] is
// loaded with 16-byte (or 8-byte) vector loads, so a warp issues 1/VK of the
// shared-memory reads of (column, value) and of the gather instructions that
// a thread per right-hand side would. The canonical order does not change
// (canon_finish).
#ifndef XG_SPMV_VK64
#define XG_SPMV_VK64 2  // FP64 x
#endif
#ifndef XG_SPMV_VK32
#define XG_SPMV_VK32 4  // FP32 x
#endif
// (The launcher may also pick 4 for FP64 x on short rows.)
template <typename FX, int NV>
__host__ __device__ constexpr int spmv_vk() {
    constexpr int w = sizeof(FX) == 8 ? XG_SPMV_VK64 : XG_SPMV_VK32;
    return NV < w ? NV : w;
}

template <typename FX, int VK>
__device__ __forceinline__ void ld_x(const FX *p, FX (&o)[VK]) {
    if constexpr (VK == 1) {
        o[0] = __ldg(p);
    } else if constexpr (std::is_same<FX, double>::value) {
#pragma unroll
        for (int h = 0; h < VK; h += 2) {
            const double2 t = __ldg(reinterpret_cast<const double2 *>(p + h));
            o[h] = t.x;
            o[h + 1] = t.y;
        }
    } else if constexpr (VK == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
        o[0] = t.x;
        o[1] = t.y;
    } else {
#pragma unroll
        for (int h = 0; h < VK; h += 4) {
            const float4 t = __ldg(reinterpret_cast<const float4 *>(p + h));
            o[h] = t.x;
            o[h + 1] = t.y;
            o[h + 2] = t.z;
            o[h + 3] = t.w;
        }
    }
}

// Row accumulation, entry by entry in row order (the loop is unrolled so that
// gathers of later entries can issue before earlier sums complete; the
// additions stay in order). cl/vl point at the row's first entry.
// Resident blocks the register budget is set for: 1024 threads an SM at 64
// registers a thread, whatever the block size.
template <int VK>
constexpr int spmv_min_blocks() { return 4 * VK; }

#ifndef XG_SPMV_UNROLL
#define XG_SPMV_UNROLL 4
#endif
constexpr int SPMV_UNROLL = XG_SPMV_UNROLL;

// A stored matrix value in the arithmetic type F: the value itself, or a
// BF16 value widened exactly to float.
template <typename F, typename V>
__device__ __forceinline__ F val_as(V v) {
    if constexpr (std::is_same<V, __nv_bfloat16>::value)
        return (F)__bfloat162float(v);
    else
        return (F)v;
}
// The same with a scale: an FP16-stored value times its level's power-of-two
// scale (an exact product), every other storage type as above.
template <typename F, typename V>
__device__ __forceinline__ F val_as(V v, float sc) {
    if constexpr (std::is_same<V, __half>::value)
        return (F)__fmul_rn(__half2float(v), sc);
    else
        return val_as<F, V>(v);
}

// Column index in 32 bits (the launcher checks that every x offset c*NV + k
// fits): the gather address is one 32-bit multiply-add and one widening add.
template <typename I>
__device__ __forceinline__ uint32_t col_at32(I c, uint32_t i) {
    if constexpr (std::is_same<I, int16_t>::value)
        return (uint32_t)((int32_t)i + (int32_t)c);
    else
        return (uint32_t)c;
}

template <typename F, typename FX, typename I, int NV, int VK, typename V = F>
__device__ __forceinline__ void row_sum(F (&y)[VK], uint32_t len, uint64_t i, int k0, const I *cl,
                                        const V *vl, const FX *x, float vsc = 1.0f) {
    const uint32_t i32 = (uint32_t)i;
#pragma unroll SPMV_UNROLL
    for (uint32_t j = 0; j < len; ++j) {
        const uint32_t c = col_at32<I>(cl[j], i32);
        const F av = val_as<F, V>(vl[j], vsc);
        FX xv[VK];
        ld_x<FX, VK>(x + (c * (uint32_t)NV + (uint32_t)k0), xv);
#pragma unroll
        for (int v = 0; v < VK; ++v) y[v] = add(y[v], mul((F)xv[v], av));
    }
}

// --- mbarrier and bulk-copy primitives (PTX) -------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(m)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for phase `parity` of the barrier for at most limit_ns nanoseconds
// of the global timer (and a bounded number of polls); false if the limit ran
// out.
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t *m, uint32_t parity,
                                          uint64_t limit_ns = WAIT_LIMIT_NS) {
    if (mbar_try_wait(m, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < (1u << 30); ++it) {
        if (mbar_try_wait(m, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
    return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *m) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(m))
        : "memory");
}

// Staging plan of entries [j0, j1) of an array of n elements of T: the
// 16-byte-aligned global range [c0, c1) goes by bulk copy (src/dst/return
// value: its source, destination and byte count) and entry j lands at
// sbuf[j - j0 + stage_shift(arr, j0)]; entries outside [c0, c1) are copied
// here with plain loads.
template <typename T>
__device__ __forceinline__ uint32_t stage_range(T *sbuf, const T *arr, uint64_t n, uint32_t j0,
                                                uint32_t j1, const T *&src, T *&dst) {
    constexpr uintptr_t A16 = 15;
    const uintptr_t base = (uintptr_t)arr, end = (uintptr_t)(arr + n);
    const uintptr_t lo = (uintptr_t)(arr + j0), hi = (uintptr_t)(arr + j1);
    const uintptr_t g0 = lo & ~A16;
    const uintptr_t b16 = (base + A16) & ~A16, e16 = end & ~A16, h16 = (hi + A16) & ~A16;
    uintptr_t c0 = g0 > b16 ? g0 : b16;
    uintptr_t c1 = h16 < e16 ? h16 : e16;
    if (c1 <= c0) c0 = c1 = lo;  // nothing aligned to copy in bulk
    T *s0 = sbuf + (lo - g0) / sizeof(T);  // s0[j - j0] is entry j's slot
    const uint32_t cnt = j1 - j0;
    uint32_t head = c0 > lo ? (uint32_t)((c0 - lo) / sizeof(T)) : 0u;  // entries before c0
    if (head > cnt) head = cnt;
    for (uint32_t e = 0; e < head; ++e) s0[e] = arr[j0 + e];
    uint32_t tail = c1 > lo ? (uint32_t)((c1 - lo) / sizeof(T)) : 0u;  // first entry at/after c1
    if (tail < head) tail = head;
    for (uint32_t e = tail; e < cnt; ++e) s0[e] = arr[j0 + e];
    src = (const T *)c0;
    dst = sbuf + (c0 - g0) / sizeof(T);
    return (uint32_t)(c1 - c0);
}

template <typename T>
__device__ __forceinline__ uint32_t stage_shift(const T *arr, uint32_t j0) {
    return (uint32_t)(((uintptr_t)(arr + j0) & 15) / sizeof(T));
}

// Kernel with dynamic shared memory: nbuf (1 or 2) buffers, each of cap
// entries of values and columns plus 32 bytes of alignment slack per array;
// tiles with more entries read global memory directly. V is the type the
// values are stored in: F, or BF16 for an FP32 level stored in BF16 (the
// arithmetic stays in F).
// CT/VK threads; thread p carries row slot p/(NV/VK) and right-hand sides
// k0 = (p % (NV/VK))*VK .. k0+VK-1 (x aligned to VK elements).
// Tiles are dealt round-robin to B canonical blocks (tile t to block t % B);
// physical block p runs canonical blocks p, p + gridDim.x, ... in turn, so a
// grid of the blocks that fit the GPU at once covers any B. Without dot
// products B is simply the grid size, and the tiles may be dealt in runs of
// `run` consecutive tiles (run q to block q % gridDim.x), so that a block's
// successive tiles share columns in its SM's L1.
template <typename F, typename FX, typename I, int NV, int VK, int NRED, class Epi,
          typename V = F>
__global__ void __launch_bounds__(CT / VK, spmv_min_blocks<VK>())
    k_spmv(CsrArgs<F> A, const FX *__restrict__ x, Epi epi, RedArgs ra, uint32_t cap,
           uint32_t nbuf, uint32_t B, uint32_t run = 1, uint32_t stride = 0) {
    constexpr int G = NV / VK;
    constexpr int R = CT / NV;
    constexpr int NR = NRED > 0 ? NRED : 1;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar[2];
    const uint32_t VB = ((cap * (uint32_t)sizeof(V) + 32u) + 15u) & ~15u;
    const uint32_t BB = VB + (((cap * (uint32_t)sizeof(I) + 32u) + 15u) & ~15u);
    const uint32_t CAP = cap;
    const int rt = threadIdx.x / G, k0 = (threadIdx.x % G) * VK;
    const uint32_t *__restrict__ row = A.row;
    const I *__restrict__ col = (const I *)A.col;
    const V *__restrict__ val = (const V *)A.val;
    const uint64_t n = A.n;
    const uint64_t nnz = n ? row[n] : 0;
    const uint64_t ntiles = (n + R - 1) / R;
    // position after t in this physical block's sequence (ntiles: none);
    // positions are tiles except in the plane walk below
    auto next_tile = [&](uint64_t t) -> uint64_t {
        if constexpr (NRED == 0) {
            if ((t + 1) % run != 0 && t + 1 < ntiles) return t + 1;
            const uint64_t q = (t / run + gridDim.x) * run;
            return q < ntiles ? q : ntiles;
        }
        if (t + B < ntiles) return t + B;
        const uint64_t c = t % B + gridDim.x;
        return c < B ? c : ntiles;
    };
    // Plane walk (no dot products, stride > 0): the blocks run through walk
    // positions u as above, position u being tile (u % M) * stride + u / M for
    // u < M * stride (M = ntiles / stride) and tile u after that: a
    // bijection, under which consecutive positions are tiles stride apart.
    const uint64_t wM = (NRED == 0 && stride) ? ntiles / stride : 0;
    const uint64_t wmain = wM * stride;
    auto tile_at = [&](uint64_t u) -> uint64_t {
        if constexpr (NRED == 0)
            if (u < wmain) return (u % wM) * stride + u / wM;
        return u;
    };
    const uint64_t first = NRED == 0 ? (uint64_t)blockIdx.x * run : (uint64_t)blockIdx.x;
    F acc[VK][NR];
#pragma unroll
    for (int v = 0; v < VK; ++v)
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[v][r] = F(0);

    if (threadIdx.x == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t n_issued = 0, n_used = 0;  // staged tiles issued (thread 0) / consumed
    bool timed_out = false;
    // thread 0: copy tile t into the next buffer if it fits
    auto issue = [&](uint64_t t) {
        if (t >= ntiles) return;
        const uint64_t a0 = t * R, a1 = a0 + R < n ? a0 + R : n;
        const uint32_t j0 = row[a0], j1 = row[a1];
        if (j1 - j0 > CAP) return;
        unsigned char *buf = smem_raw + (size_t)(n_issued % nbuf) * BB;
        uint64_t *m = &mbar[n_issued % nbuf];
        ++n_issued;
        const V *vsrc;
        V *vdst;
        const I *csrc;
        I *cdst;
        const uint32_t vb = stage_range<V>((V *)buf, val, nnz, j0, j1, vsrc, vdst);
        const uint32_t cb = stage_range<I>((I *)(buf + VB), col, nnz, j0, j1, csrc, cdst);
        mbar_arrive_expect(m, vb + cb);  // releases the plain-load writes above
        fence_proxy_async_smem();
        if (vb) bulk_g2s(vdst, vsrc, vb, m);
        if (cb) bulk_g2s(cdst, csrc, cb, m);
    };
    if (threadIdx.x == 0) issue(tile_at(first));

    for (uint64_t u = first; u < ntiles;) {
        const uint64_t unext = next_tile(u);
        const uint64_t tile = tile_at(u);
        const uint64_t tnext = unext < ntiles ? tile_at(unext) : ntiles;
        const uint64_t r0 = tile * R;
        const uint64_t r1 = r0 + R < n ? r0 + R : n;
        const uint32_t tj0 = __ldg(&row[r0]), tj1 = __ldg(&row[r1]);
        bool staged = tj1 - tj0 <= CAP;
        if (nbuf == 2 && threadIdx.x == 0) issue(tnext);
        const V *sv = nullptr;
        const I *sc = nullptr;
        if (staged) {
            const uint32_t b = n_used % nbuf;
            // a copy that never landed: raise the flag, read global memory
            if (!mbar_wait(&mbar[b], (n_used / nbuf) & 1u)) timed_out = true;
            ++n_used;
            const unsigned char *buf = smem_raw + (size_t)b * BB;
            sv = (const V *)buf + stage_shift<V>(val, tj0);
            sc = (const I *)(buf + VB) + stage_shift<I>(col, tj0);
            staged = !timed_out;
        }
        const uint64_t i = r0 + rt;
        if (i < n) {
            F y[VK];
#pragma unroll
            for (int v = 0; v < VK; ++v) y[v] = epi.init(i, k0 + v);
            const uint32_t j0 = __ldg(&row[i]), j1 = __ldg(&row[i + 1]);
            if (staged)
                row_sum<F, FX, I, NV, VK, V>(y, j1 - j0, i, k0, sc + (j0 - tj0), sv + (j0 - tj0),
                                             x, A.vscale);
            else
                row_sum<F, FX, I, NV, VK, V>(y, j1 - j0, i, k0, col + j0, val + j0, x, A.vscale);
#pragma unroll
            for (int v = 0; v < VK; ++v) epi.store(i, k0 + v, y[v], acc[v]);
        }
        __syncthreads();  // every reader is done with this tile's buffer
        if (nbuf == 1 && threadIdx.x == 0) issue(tnext);
        if constexpr (NRED > 0)
            if (tnext == ntiles || tnext % B != tile % B)
                canon_partial<F, NV, NRED, VK>(acc, ra, (uint32_t)(tile % B));
        u = unext;
    }
    if (timed_out) {
        atomicOr(ra.flag, 1u);
        // no block exits with a copy into its shared memory still in flight
        if (threadIdx.x == 0)
            for (uint32_t u = n_used; u < n_issued; ++u) mbar_wait(&mbar[u % nbuf], (u / nbuf) & 1u);
    }
    if constexpr (NRED > 0) canon_final<F, NV, NRED, CT / VK>(ra, B, epi);
}

// Warp-per-row SpMV for matrices with few rows (the coarse levels and their
// transfers), where k_spmv's time is one thread's chain of gathers down a
// whole row. A warp takes one row at a time: its lanes gather the products
// of 32/NV entries at once (lane = entry slot * NV + right-hand side), each
// product rounded on its own (mul(x, a), as row_sum rounds it), into a
// shared-memory chunk of WCH entries; then lane k < NV adds the chunk's
// products to its sum in entry order. So every output element is the same
// sequence of separately rounded products and sums as in k_spmv, while a
// row's gathers are in flight together.
constexpr int WT = 256;  // threads per block (8 warps)
template <int NV>
constexpr int wide_chunk() { return 512 / NV; }  // entries per warp-chunk
template <typename F, typename FX, typename I, int NV, class Epi, typename V = F>
__global__ void __launch_bounds__(WT) k_spmv_wide(CsrArgs<F> A, const FX *__restrict__ x, Epi epi) {
    constexpr int E = NV >= 32 ? 1 : 32 / NV;  // entries a warp gathers per round
    constexpr int CH = wide_chunk<NV>();
    __shared__ F prod[WT / 32][CH * NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = lane % NV, es = lane / NV;  // es < E for NV <= 32
    const uint32_t *__restrict__ row = A.row;
    const I *__restrict__ col = (const I *)A.col;
    const V *__restrict__ val = (const V *)A.val;
    F *pw = prod[warp];
    const uint64_t nw = (uint64_t)gridDim.x * (WT / 32);
    for (uint64_t i = (uint64_t)blockIdx.x * (WT / 32) + warp; i < A.n; i += nw) {
        const uint32_t j0 = __ldg(&row[i]), j1 = __ldg(&row[i + 1]);
        const uint32_t i32 = (uint32_t)i;
        F y = k < NV && lane < NV ? epi.init(i, k) : F(0);
        for (uint32_t c0 = j0; c0 < j1; c0 += CH) {
            const uint32_t len = j1 - c0 < (uint32_t)CH ? j1 - c0 : (uint32_t)CH;
#pragma unroll 4
            for (uint32_t e = es; e < len; e += E) {
                const uint32_t c = col_at32<I>(__ldg(&col[c0 + e]), i32);
                const F av = val_as<F, V>(__ldg(&val[c0 + e]), A.vscale);
                pw[e * NV + k] = mul((F)__ldg(&x[c * (uint32_t)NV + (uint32_t)k]), av);
            }
            __syncwarp();
            if (lane < NV) {
#pragma unroll 8
                for (uint32_t e = 0; e < len; ++e) y = add(y, pw[e * NV + lane]);
            }
            __syncwarp();
        }
        F none[1] = {F(0)};
        if (lane < NV) epi.store(i, lane, y, none);
    }
}

// Bounded-wait check: one block waits on an mbarrier that nothing arrives
// at, gives up after limit_ns and raises the timeout flag, as a staging wait
// of k_spmv does when its copy never lands. Nothing is in flight when it
// returns.
static __global__ void k_wait_selftest(uint64_t limit_ns, unsigned *flag) {
    __shared__ __align__(8) uint64_t m;
    if (threadIdx.x == 0) {
        mbar_init(&m, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (!mbar_wait(&m, 0, limit_ns) && threadIdx.x == 0) atomicOr(flag, 1u);
}

// Largest entry count of a tile of R rows (for matrices whose row pointers
// live only on the device).
static __global__ void k_tile_max(const uint32_t *__restrict__ row, uint64_t n, uint64_t R,
                                  unsigned *out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t r0 = t * R;
    if (r0 < n) {
        const uint64_t r1 = r0 + R < n ? r0 + R : n;
        atomicMax(out, row[r1] - row[r0]);
    }
}

// Element-wise canonical kernel (same schedule, no matrix). At most 64
// registers a thread, so that four 256-thread blocks share an SM (the merged
// group kernels with nv <= 8 take 76 registers left alone, three blocks);
// these streaming kernels are bound by the loads in flight.
template <typename F, int NV, int NRED, class Epi>
__global__ void __launch_bounds__(CT, 4) k_rows(uint64_t n, Epi epi, RedArgs ra) {
    constexpr int R = CT / NV;
    const int rt = threadIdx.x / NV, k = threadIdx.x % NV;
    const uint64_t ntiles = (n + R - 1) / R;
    F acc[NRED > 0 ? NRED : 1];
#pragma unroll
    for (int r = 0; r < (NRED > 0 ? NRED : 1); ++r) acc[r] = F(0);
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t i = tile * R + rt;
        if (i < n) epi.elem(i, k, acc);
    }
    if constexpr (NRED > 0) canon_finish<F, NV, NRED>(acc, ra, epi);
}

// Scalar-only kernel: one thread per right-hand side.
template <class Op>
__global__ void k_scalar(int nv, Op op) {
    if ((int)threadIdx.x < nv) op(threadIdx.x);
}

// ---------------------------------------------------------------------------
// Epilogues. `NoFin` is used when the epilogue has no reduction.
// ---------------------------------------------------------------------------
struct NoFin {
    template <typename T>
    __device__ void operator()(int, const T *) const {}
};

// y = A x  (csr_matvec.inl:213-231)
template <typename F, int NV>
struct EStore : NoFin {
    F *y;
    __device__ F init(uint64_t, int) const { return F(0); }
    template <int NR>
    __device__ void store(uint64_t i, int k, F v, F (&)[NR]) const { y[i * NV + k] = v; }
};

// y += A x  (csr_matvec.inl:106-120: accumulate directly into y)
template <typename F, int NV>
struct EAxpy : NoFin {
    F *y;
    __device__ F init(uint64_t i, int k) const { return y[i * NV + k]; }
    template <int NR>
    __device__ void store(uint64_t i, int k, F v, F (&)[NR]) const { y[i * NV + k] = v; }
};

// r = 1*b + (-1)*(A x)  (solver.h:249-250: Ax_y then axpby(1, b, -1, r)),
// optionally with (r, r) (vector_norm, blas.inl:537-555).
template <typename F, int NV, bool NORM>
struct EResid {
    F *r;
    const F *b;
    double *out;  // NORM: sums land here (nv values)
    __device__ F init(uint64_t, int) const { return F(0); }
    template <int NR>
    __device__ void store(uint64_t i, int k, F v, F (&acc)[NR]) const {
        const F rv = add(mul(F(1), b[i * NV + k]), mul(F(-1), v));
        r[i * NV + k] = rv;
        if constexpr (NORM) acc[0] = add(acc[0], mul(rv, rv));
    }
    __device__ void operator()(int k, const F *s) const {
        if constexpr (NORM) out[k] = (double)s[0];
    }
};

// merged_bicgstab_group1 after r0 = A x (blas_merged_bicgstab.inl:60-72):
// r0 = b - r0; rho0 += r0*r0; p = r = r0. The finaliser also copies
// rho0 into rho (merged_bicgstab.inl:119).
template <int NV>
struct EGroup1 {
    double *r0, *p, *r;
    const double *b;
    double *sc;
    __device__ double init(uint64_t, int) const { return 0.0; }
    template <int NR>
    __device__ void store(uint64_t i, int k, double v, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        const double rv = sub(b[e], v);
        r0[e] = rv;
        p[e] = rv;
        r[e] = rv;
        acc[0] = add(acc[0], mul(rv, rv));
    }
    __device__ void operator()(int k, const double *s) const {
        sc[SC_RHO0 * SC_STRIDE + k] = s[0];
        sc[SC_RHO * SC_STRIDE + k] = s[0];
    }
};

// v = A p_ ; scal1 = (v, r0) ; alpha = rho / scal1
// (merged_pbicgstab.inl:140-155)
template <int NV>
struct EDotAlpha {
    double *v;
    const double *r0;
    double *sc;
    __device__ double init(uint64_t, int) const { return 0.0; }
    template <int NR>
    __device__ void store(uint64_t i, int k, double y, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        v[e] = y;
        acc[0] = add(acc[0], mul(y, r0[e]));
    }
    __device__ void operator()(int k, const double *s) const {
        sc[SC_SCAL1 * SC_STRIDE + k] = s[0];
        sc[SC_ALPHA * SC_STRIDE + k] = dvd(sc[SC_RHO * SC_STRIDE + k], s[0]);
    }
};

// t = A s_ ; phi = (t,s), psi = (t,t), theta = (s,s); omega = phi/psi;
// res = theta - omega*phi; alpha_c = iconv*alpha; omega_c = iconv*omega
// (merged_pbicgstab.inl:168-192)
template <int NV>
struct EDot3 {
    double *t;
    const double *s;
    double *sc;
    __device__ double init(uint64_t, int) const { return 0.0; }
    template <int NR>
    __device__ void store(uint64_t i, int k, double y, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        t[e] = y;
        const double sv = s[e];
        acc[0] = add(acc[0], mul(y, sv));
        acc[1] = add(acc[1], mul(y, y));
        acc[2] = add(acc[2], mul(sv, sv));
    }
    __device__ void operator()(int k, const double *s3) const {
        double *S = sc;
        const double phi = s3[0], psi = s3[1], theta = s3[2];
        S[SC_PHI * SC_STRIDE + k] = phi;
        S[SC_PSI * SC_STRIDE + k] = psi;
        S[SC_THETA * SC_STRIDE + k] = theta;
        const double omega = dvd(phi, psi);
        S[SC_OMEGA * SC_STRIDE + k] = omega;
        double res = mul(omega, phi);
        res = add(mul(1.0, theta), mul(-1.0, res));
        S[SC_RES * SC_STRIDE + k] = res;
        const double ic = S[SC_ICONV * SC_STRIDE + k];
        S[SC_ALPHA_C * SC_STRIDE + k] = mul(ic, S[SC_ALPHA * SC_STRIDE + k]);
        S[SC_OMEGA_C * SC_STRIDE + k] = mul(ic, omega);
    }
};

// One Jacobi sweep with x not zero (blas_merged_jacobi.inl:74-80):
// x_out = x_in + relax*d*(b - A x_in)
template <typename F, int NV>
struct EJacobi : NoFin {
    F *xout;
    const F *xin, *b, *d;
    F relax;
    __device__ F init(uint64_t, int) const { return F(0); }
    template <int NR>
    __device__ void store(uint64_t i, int k, F v, F (&)[NR]) const {
        const uint64_t e = i * NV + k;
        xout[e] = add(xin[e], mul(mul(relax, d[i]), sub(b[e], v)));
    }
};

// Chebyshev, first polynomial step (chebyshev.inl:179-190):
// r = b - A x; r := r*isd; t1 = c_top * r; t1 := t1*isd (input of the next
// SpMV). x_zero: r = 1*b without the SpMV (used by k_rows through elem()).
template <typename F, int NV>
struct ECheby0 : NoFin {
    F *rs, *t1s;
    const F *b, *isd;
    F c;
    __device__ F init(uint64_t, int) const { return F(0); }
    __device__ void finish(uint64_t i, int k, F r) const {
        const uint64_t e = i * NV + k;
        const F d = isd[i];
        const F rr = mul(r, d);
        rs[e] = rr;
        t1s[e] = mul(mul(c, rr), d);
    }
    template <int NR>
    __device__ void store(uint64_t i, int k, F v, F (&)[NR]) const {
        const uint64_t e = i * NV + k;
        finish(i, k, add(mul(F(1), b[e]), mul(F(-1), v)));
    }
    template <int NR>
    __device__ void elem(uint64_t i, int k, F (&)[NR]) const {
        finish(i, k, mul(F(1), b[i * NV + k]));
    }
};

// Chebyshev inner step i (chebyshev.inl:189-199):
// t2 = A t1s; t2 := t2*isd; t1 = c_i*rs + 1*t2; then either t1s_out = t1*isd
// (more steps) or x = 1*(t1*isd) + 1*x (last step; x_zero: x = 1*(t1*isd)).
template <typename F, int NV>
struct ECheby1 : NoFin {
    F *out;  // next t1s, or x on the last step
    const F *rs, *isd;
    F c;
    int last, x_zero;
    __device__ F init(uint64_t, int) const { return F(0); }
    template <int NR>
    __device__ void store(uint64_t i, int k, F v, F (&)[NR]) const {
        const uint64_t e = i * NV + k;
        const F d = isd[i];
        const F t2 = mul(v, d);
        const F t1 = add(mul(c, rs[e]), mul(F(1), t2));
        const F t1d = mul(t1, d);
        if (!last)
            out[e] = t1d;
        else if (x_zero)
            out[e] = mul(F(1), t1d);
        else
            out[e] = add(mul(F(1), t1d), mul(F(1), out[e]));
    }
};

// Prolongation with a reduced-precision P (mg.inl:241-249): the product is
// accumulated in float, converted to double, then x = 1*t + 1*x
// (x_zero: x = 1*t, the ax_y branch of axpby).
template <int NV>
struct EProlongMixed : NoFin {
    double *x;
    int x_zero;
    __device__ float init(uint64_t, int) const { return 0.0f; }
    template <int NR>
    __device__ void store(uint64_t i, int k, float v, float (&)[NR]) const {
        const uint64_t e = i * NV + k;
        const double t = (double)v;
        x[e] = x_zero ? mul(1.0, t) : add(mul(1.0, t), mul(1.0, x[e]));
    }
};

// ---------------------------------------------------------------------------
// Element-wise epilogues for k_rows
// ---------------------------------------------------------------------------

// dot[k] = (x, y)_k  (blas.inl:504-519)
template <typename F, int NV>
struct EDot {
    const F *x, *y;
    double *out;
    template <int NR>
    __device__ void elem(uint64_t i, int k, F (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        acc[0] = add(acc[0], mul(x[e], y[e]));
    }
    __device__ void operator()(int k, const F *s) const { out[k] = (double)s[0]; }
};

// merged_bicgstab_group2 (blas_merged_bicgstab.inl:127-134)
template <int NV>
struct EGroup2 {
    const double *t, *s;
    double *out;  // phi, psi, theta at out[0..nv), out[32..), out[64..)
    template <int NR>
    __device__ void elem(uint64_t i, int k, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        const double tv = t[e], sv = s[e];
        acc[0] = add(acc[0], mul(tv, sv));
        acc[1] = add(acc[1], mul(tv, tv));
        acc[2] = add(acc[2], mul(sv, sv));
    }
    __device__ void operator()(int k, const double *s3) const {
        out[k] = s3[0];
        out[32 + k] = s3[1];
        out[64 + k] = s3[2];
    }
};

// group4 (blas_merged_bicgstab.inl:179-185): r = s - omega*t; rho += r*r0,
// optionally preceded by the x update of merged_pbicgstab.inl:193
// (x = alpha_c*p_ + omega_c*s_ + 1*x). The finaliser does lines 207-217:
// beta = (scal1/rho)*(alpha/omega); rho = scal1; nscal = -(omega*beta);
// and, for the unpreconditioned form, alpha_c/omega_c from the current iconv
// (merged_bicgstab.inl:192-199).
// PT: the type the preconditioned vectors pa, sa are stored in (float when
// an FP32 preconditioner leaves its result in float; widened exactly).
template <int NV, bool XUPD, typename PT = double>
struct EGroup4 {
    const double *s, *t, *r0;
    double *r;
    double *x;
    const PT *pa, *sa;
    double *sc;
    template <int NR>
    __device__ void elem(uint64_t i, int k, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        if constexpr (XUPD) {
            const double ac = sc[SC_ALPHA_C * SC_STRIDE + k], oc = sc[SC_OMEGA_C * SC_STRIDE + k];
            x[e] = add(add(mul(ac, (double)pa[e]), mul(oc, (double)sa[e])), mul(1.0, x[e]));
        }
        const double om = sc[SC_OMEGA * SC_STRIDE + k];
        const double rv = sub(s[e], mul(om, t[e]));
        r[e] = rv;
        acc[0] = add(acc[0], mul(rv, r0[e]));
    }
    __device__ void operator()(int k, const double *s1) const {
        double *S = sc;
        const double scal1 = s1[0];
        S[SC_SCAL1 * SC_STRIDE + k] = scal1;
        const double scal2 = dvd(scal1, S[SC_RHO * SC_STRIDE + k]);
        const double scal3 = dvd(S[SC_ALPHA * SC_STRIDE + k], S[SC_OMEGA * SC_STRIDE + k]);
        const double beta = mul(scal2, scal3);
        S[SC_SCAL2 * SC_STRIDE + k] = scal2;
        S[SC_SCAL3 * SC_STRIDE + k] = scal3;
        S[SC_BETA * SC_STRIDE + k] = beta;
        S[SC_RHO * SC_STRIDE + k] = scal1;
        S[SC_NSCAL * SC_STRIDE + k] = mul(mul(S[SC_OMEGA * SC_STRIDE + k], beta), -1.0);
        const double ic = S[SC_ICONV * SC_STRIDE + k];
        S[SC_ALPHA_C * SC_STRIDE + k] = mul(ic, S[SC_ALPHA * SC_STRIDE + k]);
        S[SC_OMEGA_C * SC_STRIDE + k] = mul(ic, S[SC_OMEGA * SC_STRIDE + k]);
    }
};

// ---------------------------------------------------------------------------
// Flat element-wise kernels (no reduction): one thread per element e of the
// [n][NV] array, grid-stride.
// ---------------------------------------------------------------------------
template <class Op>
__global__ void __launch_bounds__(CT) k_flat(uint64_t m, Op op) {
    for (uint64_t e = (uint64_t)blockIdx.x * CT + threadIdx.x; e < m;
         e += (uint64_t)gridDim.x * CT)
        op(e);
}

// s = 1*r + (-alpha)*v  (merged_pbicgstab.inl:159-161)
struct OpSUpdate {
    double *s;
    const double *r, *v, *sc;
    int nv;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double na = mul(sc[SC_ALPHA * SC_STRIDE + k], -1.0);
        s[e] = add(mul(1.0, r[e]), mul(na, v[e]));
    }
};

// x = alpha_c*pa + omega_c*sa + 1*x  (merged_pbicgstab.inl:193, blas_ext.inl:173-177)
template <typename PT = double>
struct OpXUpdateT {
    double *x;
    const PT *pa, *sa;
    const double *sc;
    int nv;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double ac = sc[SC_ALPHA_C * SC_STRIDE + k], oc = sc[SC_OMEGA_C * SC_STRIDE + k];
        x[e] = add(add(mul(ac, (double)pa[e]), mul(oc, (double)sa[e])), mul(1.0, x[e]));
    }
};
using OpXUpdate = OpXUpdateT<double>;

// PCG (pcg.inl:103-150). Ap = A p with scal2 = (p, Ap); finaliser:
// alpha = scal1 / scal2, alpha_conv = iconv * alpha, then alpha = -1 * alpha
// (kept in SC_NSCAL). scal1 = (r, z) is the previous (r, z) (EPcgDots).
template <int NV>
struct EPcgAp {
    double *Ap;
    const double *p;
    double *sc;
    __device__ double init(uint64_t, int) const { return 0.0; }
    template <int NR>
    __device__ void store(uint64_t i, int k, double y, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        Ap[e] = y;
        acc[0] = add(acc[0], mul(p[e], y));
    }
    __device__ void operator()(int k, const double *s) const {
        double *S = sc;
        S[SC_SCAL2 * SC_STRIDE + k] = s[0];
        const double alpha = dvd(S[SC_SCAL1 * SC_STRIDE + k], s[0]);
        S[SC_ALPHA * SC_STRIDE + k] = alpha;
        S[SC_ALPHA_C * SC_STRIDE + k] = mul(S[SC_ICONV * SC_STRIDE + k], alpha);
        S[SC_NSCAL * SC_STRIDE + k] = mul(-1.0, alpha);
    }
};

// (r, z) and (r, r) in one pass; finaliser: first call scal1 = (r, z);
// afterwards scal3 = (r, z), beta = scal3 / scal1, res = (r, r), and
// scal1 = scal3 for the next iteration (XAMG recomputes dot(r, z) there from
// the same vectors, pcg.inl:105).
template <int NV>
struct EPcgDots {
    const double *r, *z;
    double *sc;
    bool first;
    template <int NR>
    __device__ void elem(uint64_t i, int k, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        const double rv = r[e];
        acc[0] = add(acc[0], mul(rv, z[e]));
        acc[1] = add(acc[1], mul(rv, rv));
    }
    __device__ void operator()(int k, const double *s) const {
        double *S = sc;
        if (first) {
            S[SC_SCAL1 * SC_STRIDE + k] = s[0];
            return;
        }
        S[SC_SCAL3 * SC_STRIDE + k] = s[0];
        S[SC_BETA * SC_STRIDE + k] = dvd(s[0], S[SC_SCAL1 * SC_STRIDE + k]);
        S[SC_SCAL1 * SC_STRIDE + k] = s[0];
        S[SC_RES * SC_STRIDE + k] = s[1];
    }
};

// x = alpha_conv*p + 1*x (x = alpha_conv*p while x is zero-flagged);
// r = (-alpha)*Ap + 1*r  (pcg.inl:123-127, axpby blas.inl:89-151)
struct OpPcgXR {
    double *x, *r;
    const double *p, *Ap, *sc;
    int nv;
    bool x_zero;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double ac = sc[SC_ALPHA_C * SC_STRIDE + k], na = sc[SC_NSCAL * SC_STRIDE + k];
        x[e] = x_zero ? mul(ac, p[e]) : add(mul(ac, p[e]), mul(1.0, x[e]));
        r[e] = add(mul(na, Ap[e]), mul(1.0, r[e]));
    }
};

// p = 1*z + beta*p  (pcg.inl:142)
struct OpPcgP {
    double *p;
    const double *z, *sc;
    int nv;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        p[e] = add(mul(1.0, z[e]), mul(sc[SC_BETA * SC_STRIDE + k], p[e]));
    }
};

// Reordered BiCGStab (rbicgstab.inl:44-243, merged_rbicgstab.inl:44-230).
// merged_rbicgstab_group1 (blas_merged_rbicgstab.inl:33-116): r = r - alpha v,
// then theta = (t, r), phi = (t, t), psi = (t, r0), eta = (r, r). The
// unmerged form's r = (-alpha) v + 1 r is the same value bit for bit.
// Finaliser: omega = theta / phi; res = 1 eta + (-1)(omega theta);
// alpha_conv, omega_conv; rho = -(omega psi); beta = rho / (delta omega),
// delta = (v, r0) in SC_SCAL1.
template <int NV>
struct ERbGroup1 {
    double *r;
    const double *v, *t, *r0;
    double *sc;
    template <int NR>
    __device__ void elem(uint64_t i, int k, double (&acc)[NR]) const {
        const uint64_t e = i * NV + k;
        const double rv = sub(r[e], mul(sc[SC_ALPHA * SC_STRIDE + k], v[e]));
        r[e] = rv;
        const double tv = t[e];
        acc[0] = add(acc[0], mul(tv, rv));
        acc[1] = add(acc[1], mul(tv, tv));
        acc[2] = add(acc[2], mul(tv, r0[e]));
        acc[3] = add(acc[3], mul(rv, rv));
    }
    __device__ void operator()(int k, const double *s4) const {
        double *S = sc;
        const double theta = s4[0], phi = s4[1], psi = s4[2], eta = s4[3];
        S[SC_THETA * SC_STRIDE + k] = theta;
        S[SC_PHI * SC_STRIDE + k] = phi;
        S[SC_PSI * SC_STRIDE + k] = psi;
        S[SC_ETA * SC_STRIDE + k] = eta;
        const double omega = dvd(theta, phi);
        S[SC_OMEGA * SC_STRIDE + k] = omega;
        S[SC_RES * SC_STRIDE + k] = add(mul(1.0, eta), mul(-1.0, mul(omega, theta)));
        const double ic = S[SC_ICONV * SC_STRIDE + k];
        S[SC_ALPHA_C * SC_STRIDE + k] = mul(ic, S[SC_ALPHA * SC_STRIDE + k]);
        S[SC_OMEGA_C * SC_STRIDE + k] = mul(ic, omega);
        const double rho = mul(-1.0, mul(omega, psi));
        S[SC_RHO * SC_STRIDE + k] = rho;
        S[SC_BETA * SC_STRIDE + k] = dvd(rho, mul(S[SC_SCAL1 * SC_STRIDE + k], omega));
    }
};

// t_ = 1 z + (-alpha) s  (axpby_z, blas_ext.inl:193-239, with its zero-flag
// branches)
struct OpRbT {
    double *t_;
    const double *z, *s, *sc;
    int nv;
    bool z_zero, s_zero;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double na = mul(-1.0, sc[SC_ALPHA * SC_STRIDE + k]);
        t_[e] = z_zero ? mul(na, s[e]) : s_zero ? mul(1.0, z[e]) : add(mul(1.0, z[e]), mul(na, s[e]));
    }
};

// x = alpha_conv v_ + omega_conv t_ + 1 x (axpbypcz; x zero-flagged: without
// the x term)
__device__ __forceinline__ double rb_x(double ac, double v, double oc, double t, double x,
                                       bool x_zero) {
    return x_zero ? add(mul(ac, v), mul(oc, t)) : add(add(mul(ac, v), mul(oc, t)), mul(1.0, x));
}

// r = (-omega) t + 1 r; with x: the unmerged form's x update before the
// convergence test (rbicgstab.inl:200-205)
struct OpRbR {
    double *r, *x;
    const double *t, *v_, *t_, *sc;
    int nv;
    bool x_zero;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        r[e] = add(mul(mul(-1.0, sc[SC_OMEGA * SC_STRIDE + k]), t[e]), mul(1.0, r[e]));
        if (x)
            x[e] = rb_x(sc[SC_ALPHA_C * SC_STRIDE + k], v_[e], sc[SC_OMEGA_C * SC_STRIDE + k],
                        t_[e], x[e], x_zero);
    }
};

// the merged form's x update on convergence (merged_rbicgstab.inl:199-203)
struct OpRbX {
    double *x;
    const double *v_, *t_, *sc;
    int nv;
    bool x_zero;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        x[e] = rb_x(sc[SC_ALPHA_C * SC_STRIDE + k], v_[e], sc[SC_OMEGA_C * SC_STRIDE + k], t_[e],
                    x[e], x_zero);
    }
};

// Merged: merged_rbicgstab_group2 (blas_merged_rbicgstab.inl:120-193) with
// alpha_conv, omega_conv taken with the updated iconv:
//   x = x + (ac v_ + oc t_); z = t_ - omega z; v_ = (z + beta v_) - (beta omega) s.
// Unmerged (rbicgstab.inl:226-236): z = 1 t_ + (-omega) z;
//   v_ = (1 z + ((-omega) beta) s) + beta v_.
struct OpRbG2 {
    double *x, *v_, *z;
    const double *t_, *s, *sc;
    int nv;
    bool merged, x_zero;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double om = sc[SC_OMEGA * SC_STRIDE + k], be = sc[SC_BETA * SC_STRIDE + k];
        const double tv = t_[e];
        if (merged) {
            const double ic = sc[SC_ICONV * SC_STRIDE + k];
            const double ac = mul(ic, sc[SC_ALPHA * SC_STRIDE + k]), oc = mul(ic, om);
            const double xo = x_zero ? 0.0 : x[e];
            x[e] = add(xo, add(mul(ac, v_[e]), mul(oc, tv)));
            const double zn = sub(tv, mul(om, z[e]));
            z[e] = zn;
            v_[e] = sub(add(zn, mul(be, v_[e])), mul(mul(be, om), s[e]));
        } else {
            const double nom = mul(-1.0, om);
            const double zn = add(mul(1.0, tv), mul(nom, z[e]));
            z[e] = zn;
            v_[e] = add(add(mul(1.0, zn), mul(mul(nom, be), s[e])), mul(be, v_[e]));
        }
    }
};

// p = 1*r + nscal*v + beta*p  (merged_pbicgstab.inl:216-218)
struct OpPUpdate {
    double *p;
    const double *r, *v, *sc;
    int nv;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double ns = sc[SC_NSCAL * SC_STRIDE + k], be = sc[SC_BETA * SC_STRIDE + k];
        p[e] = add(add(mul(1.0, r[e]), mul(ns, v[e])), mul(be, p[e]));
    }
};

// merged_bicgstab_group5 (blas_merged_bicgstab.inl:241-248)
struct OpGroup5 {
    double *x, *p;
    const double *s, *r, *v, *sc;
    int nv;
    __device__ void operator()(uint64_t e) const {
        const int k = (int)(e % nv);
        const double ac = sc[SC_ALPHA_C * SC_STRIDE + k], oc = sc[SC_OMEGA_C * SC_STRIDE + k];
        const double be = sc[SC_BETA * SC_STRIDE + k];
        const double val = mul(be, sc[SC_OMEGA * SC_STRIDE + k]);
        x[e] = add(x[e], add(mul(ac, p[e]), mul(oc, s[e])));
        p[e] = sub(add(r[e], mul(be, p[e])), mul(val, v[e]));
    }
};

// First Jacobi sweep from x = 0 with r = 0 (blas_merged_jacobi.inl:61-67):
// x = relax*d*b
template <typename F>
struct OpJacobiZero {
    F *x;
    const F *b, *d;
    F relax;
    int nv;
    __device__ void operator()(uint64_t e) const {
        x[e] = mul(mul(relax, d[e / nv]), b[e]);
    }
};

template <typename T>
struct OpFill {
    T *x;
    T v;
    __device__ void operator()(uint64_t e) const { x[e] = v; }
};

template <typename TD, typename TS>
struct OpConvert {
    TD *d;
    const TS *s;
    __device__ void operator()(uint64_t e) const { d[e] = (TD)s[e]; }
};

// y = 1*x + 1*y, or y = 1*x when y is zero-flagged (axpby(a1, x, a1, y))
template <typename T>
struct OpAddInto {
    T *y;
    const T *x;
    int y_zero;
    __device__ void operator()(uint64_t e) const {
        y[e] = y_zero ? mul(T(1), x[e]) : add(mul(T(1), x[e]), mul(T(1), y[e]));
    }
};

// y[i][k] *= d[i]  (blas::scal with an nv = 1 vector, blas.inl:189-193)
template <typename F>
struct OpScaleRows {
    F *y;
    const F *d;
    int nv;
    __device__ void operator()(uint64_t e) const { y[e] = mul(y[e], d[e / nv]); }
};

// y = a_k*x + 1*y with a_k = coef[k] (axpby(relax, r, a1, x), jacobi.inl:103);
// y_zero: y = a_k*x (the ax_y branch)
template <typename F>
struct OpAxpyK {
    F *y;
    const F *x;
    const double *coef;
    int nv, y_zero;
    __device__ void operator()(uint64_t e) const {
        const F a = (F)coef[e % nv];
        y[e] = y_zero ? mul(a, x[e]) : add(mul(a, x[e]), mul(F(1), y[e]));
    }
};

// ---------------------------------------------------------------------------
// Hybrid symmetric Gauss-Seidel sweep (csr_gs.inl:77-130) over GS blocks:
// thread (block g, component k) runs the forward then the backward sweep of
// rows [off_g, off_g + size_g) with the block-local entries; t already holds
// b - A_offblock x_old. Blocks are independent, so no thread reads another
// thread's writes.
// ---------------------------------------------------------------------------
template <typename F, typename I, int NV>
__global__ void __launch_bounds__(CT)
    k_hsgs_sweep(const uint32_t *__restrict__ row, const I *__restrict__ col,
                 const F *__restrict__ val, const uint64_t *__restrict__ boff, int nblocks,
                 const F *__restrict__ t, F *__restrict__ x, const F *__restrict__ d,
                 const double *__restrict__ relax_sc) {
    const uint64_t gt = (uint64_t)blockIdx.x * CT + threadIdx.x;
    const int g = (int)(gt / NV), k = (int)(gt % NV);
    if (g >= nblocks) return;
    const uint64_t r0 = boff[g], r1 = boff[g + 1];
    if (r0 >= r1) return;
    const F w = (F)relax_sc[k];
    auto upd = [&](uint64_t i) {
        const uint64_t e = i * NV + k;
        F sum = t[e];
        for (uint32_t j = row[i]; j < row[i + 1]; ++j) {
            const uint64_t c = (uint64_t)col[j] + r0;
            sum = sub(sum, mul(x[c * NV + k], val[j]));
        }
        const F coeff = mul(w, d[i]);
        x[e] = add(x[e], mul(coeff, sum));
    };
    for (uint64_t i = r0; i < r1; ++i) upd(i);
    for (uint64_t i = r1; i-- > r0;) upd(i);
}

// Dense y = A_inv b (dense_matvec.inl:109-117): thread (i, k) accumulates
// over j in order. The inverse is stored column by column (element (i, j)
// at j*n + i). A block of DT threads holds DT/NV consecutive rows; it copies
// chunks of DJ columns of its rows and the matching DJ rows of x into shared
// memory with coalesced loads, then every thread runs its sum over the chunk
// from shared memory, so the sequential sums wait on shared memory rather
// than on L2.
constexpr int DT = 64;
constexpr int DJ = 64;
template <typename F, int NV>
__global__ void __launch_bounds__(DT)
    k_dense(const F *__restrict__ a, uint64_t n, const F *__restrict__ x, F *__restrict__ y) {
    constexpr int RB = DT / NV;  // rows a block
    __shared__ F xs[DJ * NV];
    __shared__ F as[DJ * RB];
    const int r = threadIdx.x / NV, k = threadIdx.x % NV;
    const uint64_t i0 = (uint64_t)blockIdx.x * RB;
    const uint64_t i = i0 + r;
    F acc = F(0);
    for (uint64_t j0 = 0; j0 < n; j0 += DJ) {
        const int jc = (int)(n - j0 < (uint64_t)DJ ? n - j0 : (uint64_t)DJ);
        __syncthreads();  // the previous chunk is consumed
        for (int t = threadIdx.x; t < jc * NV; t += DT) xs[t] = __ldg(&x[j0 * NV + t]);
        for (int t = threadIdx.x; t < jc * RB; t += DT) {
            const int jj = t / RB, rr = t % RB;
            as[t] = i0 + rr < n ? __ldg(&a[(j0 + jj) * n + i0 + rr]) : F(0);
        }
        __syncthreads();
        if (i < n)
            for (int jj = 0; jj < jc; ++jj) acc = add(acc, mul(as[jj * RB + r], xs[jj * NV + k]));
    }
    if (i < n) y[i * NV + k] = acc;
}

// --- persistent preconditioned BiCGStab ----------------------------------------
// Grid barrier with a bounded wait: every block of a cooperative launch
// arrives on one 64-bit counter (zero at the launch's start; round r ends when
// it reaches (r + 1) * expected). Thread 0 of a block arrives with a
// release-ordered atomic add and polls the counter with acquire-ordered loads;
// __syncthreads() on both sides extends that ordering to the whole block (the
// writes of every thread before the barrier are visible to every thread of
// every block after it). A monotonic counter needs no reset by the last
// arriver, so the round ends with its own arrival. A block whose wait passes
// limit_ns raises the timeout flag (read by the host as XAMG_ERR_TIMEOUT) and
// returns false, and the kernel then ends; the other blocks' next waits run
// out the same way, so no block waits without bound.
struct GridSync {
    unsigned long long *arrivals;  // zero at the launch's start
    unsigned *flag;                // bit 0: a wait ran out
    uint64_t limit_ns;
};
__device__ __forceinline__ bool grid_sync(const GridSync &g, unsigned expected) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        unsigned long long old;
        asm volatile("atom.add.release.gpu.global.u64 %0, [%1], 1;"
                     : "=l"(old)
                     : "l"(g.arrivals)
                     : "memory");
        const unsigned long long target = (old / expected + 1ull) * expected;
        uint64_t t0 = 0;
        for (uint32_t it = 0;; ++it) {
            unsigned long long cur;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];"
                         : "=l"(cur)
                         : "l"(g.arrivals)
                         : "memory");
            if (cur >= target) break;
            if ((it & 63u) == 0) {  // the clock is read every 64 polls
                const uint64_t t = global_ns();
                if (it == 0) {
                    t0 = t;
                } else if (t - t0 > g.limit_ns || it >= 0xffffff00u) {
                    atomicOr(g.flag, 1u);
                    ok = 0;
                    break;
                }
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

// The last step of the canonical reduction run by every block for itself
// (the same sums, in the same order, as canon_final's last block), with the
// finaliser writing the block's own copy of the scalar block: no block
// depends on another's finaliser.
template <int NV, int NRED, class Fin>
__device__ __forceinline__ void canon_final_local(const double *part, uint32_t B, const Fin &fin) {
    __shared__ double sums[NV * NRED];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = warp; o < NV * NRED; o += CT / 32) {
        double a = 0.0;
        for (unsigned bb = lane; bb < B; bb += 32) a = add(a, ld_cg(&part[(size_t)bb * NV * NRED + o]));
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) a = add(a, shfl_xor(a, off));
        if (lane == 0) sums[o] = a;
    }
    __syncthreads();
    for (int kk = threadIdx.x; kk < NV; kk += CT) fin(kk, &sums[kk * NRED]);
    __syncthreads();
}

struct PersistArgs {
    double *x, *r0, *r, *p, *v, *s, *t, *pa, *sa, *tmp;
    const double *d;   // Jacobi inverse diagonal; null: no Jacobi preconditioner
    int ident;         // with d null: 1 the Identity preconditioner (pa, sa copies of p, s),
                       // 0 none (pa = p, sa = s)
    double relax;
    int sweeps;        // Jacobi sweeps (max_iters of the preconditioner list)
    double *sc;        // the solver's scalar block: read at the start, written at the end
    double *out;       // [3][32]: abs_res, rel_res, conv (0/1); [96]: iterations
    int max_iters, check;
    float abs_tol, rel_tol;
    RedArgs ra;        // partial sums: two halves used in turn
    GridSync gs;
    uint32_t B;        // canonical blocks (canon_blocks(n, NV)); the grid may be smaller
};

// A BiCGStab solve recorded as one graph (csrc/loop.cu): the convergence
// test's settings and the conditional handles it sets: loop (iterate again),
// rest (the rest of a non-converged iteration), last (the final x update).
struct LoopCtl {
    int nv, max_iters, check;
    float abs_tol, rel_tol;
    cudaGraphConditionalHandle loop, rest, last;
};
// The statistics the loop leaves in device memory (doubles): abs_res,
// rel_res and conv (0/1) per right-hand side, the iterations, and whether
// the last test passed.
constexpr int LOOP_ABS = 0, LOOP_REL = 32, LOOP_CONV = 64, LOOP_ITERS = 96, LOOP_DONE = 97,
              LOOP_COUNT = 98;

// merged_pbicgstab.inl:44-225 after its start (r0, rho0, p = r = r0 and the
// first test, done by Krylov::begin/started): every iteration, its
// convergence test (solver.h:173-241 with float32 tolerances) and the final
// x update in one cooperative launch of 256-thread blocks (grid barriers
// between the steps). Physical block p plays canonical blocks p, p + grid,
// ... of the B = canon_blocks(n, NV) (a grid smaller than B has fewer
// blocks at each barrier); every reduction is summed per canonical block in
// tile order. Each step applies the same element operations, row sums and
// canonical reductions as the separate kernels of Krylov::step_tail,
// step_body and stepped, so the iterates are the same bit for bit.
template <int NV, typename I>
__global__ void __launch_bounds__(CT, 1) k_pbicgstab_persist(CsrArgs<double> A, PersistArgs P) {
    constexpr int R = CT / NV;
    __shared__ double SCS[SC_COUNT * SC_STRIDE];
    __shared__ double st_abs[NV], st_rel[NV];
    __shared__ int st_conv[NV];
    __shared__ int go;
    const uint32_t B = P.B;
    const uint64_t n = A.n;
    const uint64_t ntiles = (n + R - 1) / R;
    const int rt = threadIdx.x / NV, kk = threadIdx.x % NV;
    const uint32_t *__restrict__ row = A.row;
    const I *__restrict__ col = (const I *)A.col;
    const double *__restrict__ val = A.val;
    for (int o = threadIdx.x; o < SC_COUNT * SC_STRIDE; o += CT) SCS[o] = P.sc[o];
    for (int o = threadIdx.x; o < NV; o += CT) {
        st_abs[o] = 0.0;
        st_rel[o] = 0.0;
        st_conv[o] = 0;
    }
    __syncthreads();
    uint32_t half = 0;  // which half of the partial-sum buffer this reduction writes
    const size_t HALF = (size_t)B * NV * 4;
    auto part = [&]() { return (double *)P.ra.part + (size_t)half * HALF; };
    // every (row, right-hand side) this thread owns: canonical thread
    // threadIdx.x of the canonical blocks this block plays, tiles in order
    auto each_of = [&](uint64_t cb, auto &&fn) {
        for (uint64_t tile = cb; tile < ntiles; tile += B) {
            const uint64_t i = tile * R + rt;
            if (i < n) fn(i, (uint64_t)i * NV + kk);
        }
    };
    auto each = [&](auto &&fn) {
        for (uint64_t cb = blockIdx.x; cb < B; cb += gridDim.x) each_of(cb, fn);
    };
    // x written by other blocks in this launch: read through L2 (ld.cg), not
    // from a possibly stale L1 line
    auto rowsum = [&](const double *xv, uint64_t i) {
        double y = 0.0;
        for (uint32_t j = __ldg(&row[i]); j < __ldg(&row[i + 1]); ++j)
            y = add(y, mul(ld_cg(&xv[col_at<I>(__ldg(&col[j]), i) * NV + kk]), __ldg(&val[j])));
        return y;
    };
    auto sync = [&]() { return grid_sync(P.gs, gridDim.x); };
    // elem(i, e, acc) over every (row, right-hand side) this block owns,
    // summed per canonical block in tile order; then the grid's partials
    // summed in canonical order by every block (fin writes the scalars)
    auto reduce_each = [&](auto &acc, auto &&elem, auto &&fin) {
        constexpr int NR = sizeof(acc[0]) / sizeof(double);
        for (uint64_t cb = blockIdx.x; cb < B; cb += gridDim.x) {
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[0][r] = 0.0;
            each_of(cb, [&](uint64_t i, uint64_t e) { elem(i, e, acc[0]); });
            canon_partial<double, NV, NR, 1>(acc, RedArgs{part(), nullptr, nullptr},
                                             (uint32_t)cb);
        }
        if (!sync()) return false;
        canon_final_local<NV, NR>(part(), B, fin);
        half ^= 1u;
        return true;
    };
    // out = M^-1 in: Jacobi sweeps from zero (jacobi.inl:113-119,
    // blas_merged_jacobi.inl), the last landing in out; the Identity copies;
    // without a preconditioner pa/sa are p/s themselves
    auto precond = [&](double *out, const double *in) {
        if (!P.d) {
            if (P.ident) {  // Identity::solve: x = b (ops::convert)
                const OpConvert<double, double> cp{out, in};
                each([&](uint64_t, uint64_t e) { cp(e); });
            }
            return true;
        }
        const int m = P.sweeps < 1 ? 1 : P.sweeps;
        auto tgt = [&](int j) { return ((m - j) % 2 == 0) ? out : P.tmp; };
        double *cur = tgt(1);
        const OpJacobiZero<double> jz{cur, in, P.d, P.relax, NV};
        each([&](uint64_t, uint64_t e) { jz(e); });
        for (int j = 2; j <= m; ++j) {
            if (!sync()) return false;
            double *o = tgt(j);
            const EJacobi<double, NV> ej{{}, o, cur, in, P.d, P.relax};
            double none[1];
            each([&](uint64_t i, uint64_t) { ej.store(i, kk, rowsum(cur, i), none); });
            cur = o;
        }
        return true;
    };
    int it = 0;
    bool tail = false, done = false, ok = true;
    const EGroup4<NV, true> g4{P.s, P.t, P.r0, P.r, P.x, P.pa, P.sa, SCS};
    const OpPUpdate pu{P.p, P.r, P.v, SCS, NV};
    auto do_tail = [&]() {
        double acc[1][1] = {{0.0}};
        if (!reduce_each(acc, [&](uint64_t i, uint64_t, double(&a)[1]) { g4.elem(i, kk, a); },
                         g4))
            return false;
        each([&](uint64_t, uint64_t e) { pu(e); });
        return true;
    };
    while (ok) {
        ++it;
        if (tail && !(ok = do_tail())) break;
        if (!(ok = precond(P.pa, P.p))) break;
        if (!(ok = sync())) break;
        {   // v = A p_; alpha = rho / (v, r0)
            const EDotAlpha<NV> ea{P.v, P.r0, SCS};
            double acc[1][1] = {{0.0}};
            if (!(ok = reduce_each(
                      acc,
                      [&](uint64_t i, uint64_t, double(&a)[1]) {
                          ea.store(i, kk, rowsum(P.pa, i), a);
                      },
                      ea)))
                break;
        }
        {   // s = r - alpha v
            const OpSUpdate su{P.s, P.r, P.v, SCS, NV};
            each([&](uint64_t, uint64_t e) { su(e); });
        }
        if (!(ok = precond(P.sa, P.s))) break;
        if (!(ok = sync())) break;
        {   // t = A s_; omega, res
            const EDot3<NV> e3{P.t, P.s, SCS};
            double acc[1][3] = {{0.0, 0.0, 0.0}};
            if (!(ok = reduce_each(
                      acc,
                      [&](uint64_t i, uint64_t, double(&a)[3]) {
                          e3.store(i, kk, rowsum(P.sa, i), a);
                      },
                      e3)))
                break;
        }
        // convergence test (host_converged): every block decides alike
        if (threadIdx.x == 0) {
            bool flag = P.check != 0;
            if (flag) {
                for (int k2 = 0; k2 < NV; ++k2) {
                    if (SCS[SC_ICONV * SC_STRIDE + k2] != 0.0) {
                        const double a = sqrt(SCS[SC_RES * SC_STRIDE + k2]);
                        const double rr = a / sqrt(SCS[SC_RHO0 * SC_STRIDE + k2]);
                        if ((a > (double)P.abs_tol) && (rr > (double)P.rel_tol)) {
                            flag = false;
                        } else if (!st_conv[k2]) {
                            st_abs[k2] = a;
                            st_rel[k2] = rr;
                            st_conv[k2] = 1;
                        }
                    }
                }
                if (!flag)
                    for (int k2 = 0; k2 < NV; ++k2)
                        SCS[SC_ICONV * SC_STRIDE + k2] =
                            mul(SCS[SC_ICONV * SC_STRIDE + k2], (double)(!st_conv[k2]));
            }
            go = flag ? 0 : (it >= P.max_iters ? 1 : 2);
        }
        __syncthreads();
        if (go == 0) {   // converged: x = alpha_c p_ + omega_c s_ + x
            const OpXUpdate xu{P.x, P.pa, P.sa, SCS, NV};
            each([&](uint64_t, uint64_t e) { xu(e); });
            done = true;
            break;
        }
        tail = true;
        if (go == 1) {   // max_iters reached: the pending rest of the iteration
            ok = do_tail();
            done = ok;
            break;
        }
    }
    if (blockIdx.x == 0 && done) {
        for (int o = threadIdx.x; o < SC_COUNT * SC_STRIDE; o += CT) P.sc[o] = SCS[o];
        for (int o = threadIdx.x; o < NV; o += CT) {
            P.out[o] = st_abs[o];
            P.out[32 + o] = st_rel[o];
            P.out[64 + o] = (double)st_conv[o];
        }
        if (threadIdx.x == 0) P.out[96] = (double)it;
    }
}

// Waits at a grid barrier that one more block than the grid must reach:
// every wait runs out after limit_ns and raises the timeout flag (the
// barrier's bounded wait, exercised without a fault).
static __global__ void k_grid_selftest(GridSync g) { (void)grid_sync(g, gridDim.x + 1); }

}  // namespace k
}  // namespace xg
