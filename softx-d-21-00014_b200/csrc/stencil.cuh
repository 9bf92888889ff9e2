// Grid-stencil storage of a square CSR block and its SpMV kernel.
//
// A matrix whose every entry (i, j) lies on an offset j - i = dz*S2 + dy*S +
// dx with |dz|, |dy|, |dx| <= 1 (a 27-point box or a 7-point star on a
// lexicographically numbered grid of line stride S and plane stride S2, the
// finest level of a structured-grid problem) needs no column indices: the
// offset of each of its K slots is known. The upload keeps the CSR block and
// adds a copy in this form (gpu_index_compress = 3):
//   val[s][i]: the value of row i's entry in slot s (slot order = ascending
//              offset), 0 where row i has no such entry;
//   mask[i]:   bit s set where row i has the entry of slot s.
// The SpMV reads no column indices and no row pointers.
//
// Schedule: a thread carries M rows i, i+S, ..., i+(M-1)S (M consecutive grid
// lines) and VK right-hand sides; its values and masks come from shared
// memory (staged below). For each plane dz and each of the M+2
// lines l = -1..M around them it loads x at i + dz*S2 + l*S + dx once and adds
// it to every carried row m it is a neighbour of (dy = l - m), so a
// 27-point row costs 9(M+2)/M instead of 27 gathers of x; consecutive threads
// carry consecutive rows, so every gather of a warp is one contiguous run of
// x. Row m receives its terms in (dz, dy, dx) order, i.e. in ascending column
// order, which is the CSR row's own order: the upload requires every row
// sorted by column, or every row with its diagonal first and the rest sorted
// (diag_first; hypre's and the generators' order), in which case the
// diagonal term is added first. Every output element equals the CSR
// kernel's, bit for bit. Entries a row does not have are skipped (not added
// as zeros), so signed zeros and non-finite x behave as in the CSR sum.
#pragma once

#include "kernels.cuh"

namespace xg {
namespace k {

// Slot patterns: 0 = 27-point box (slot (dz+1)*9 + (dy+1)*3 + (dx+1)),
// 1 = 7-point star (slots -S2, -S, -1, 0, 1, S, S2).
constexpr int ST_BOX27 = 0, ST_STAR7 = 1;

template <int PAT>
__host__ __device__ constexpr int st_slots() { return PAT == ST_BOX27 ? 27 : 7; }

// Slot of offset (dz, dy, dx) in pattern PAT, or -1 where the pattern has none.
template <int PAT>
__host__ __device__ constexpr int st_slot(int dz, int dy, int dx) {
    if (PAT == ST_BOX27) return (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
    if (dz != 0) return dy == 0 && dx == 0 ? (dz < 0 ? 0 : 6) : -1;
    if (dy != 0) return dx == 0 ? (dy < 0 ? 1 : 5) : -1;
    return dx + 3;
}

struct StencilArgs {
    const void *val;       // [K][n] values (stored type V)
    const uint32_t *mask;  // [n]
    uint32_t n, S, S2;
    int diag_first;        // rows store their diagonal first
};

constexpr int ST_THREADS = 128;  // threads per block

// Tiles and staging. A tile is TX = ST_THREADS/G consecutive positions of a
// group of M grid lines (rows b0 + m*S + p, p < TX); its K*M value runs and
// M mask runs are copied into shared memory by the bulk-copy engine
// (cp.async.bulk, completion on an mbarrier; unaligned run ends with plain
// loads, as k_spmv stages its tiles), one or two buffers a block, the next
// tile's copies issued before the current tile is computed. x is gathered
// from global memory. Blocks are persistent (one wave) and take tiles
// t = blockIdx.x, blockIdx.x + gridDim.x, ...
__host__ __device__ constexpr uint32_t st_r16(uint32_t b) { return (b + 15u) & ~15u; }
template <typename V, int G>
__host__ __device__ constexpr uint32_t st_val_slot() {
    return st_r16((ST_THREADS / G) * (uint32_t)sizeof(V) + 32u);
}
template <int G>
__host__ __device__ constexpr uint32_t st_mask_slot() {
    return st_r16((ST_THREADS / G) * 4u + 32u);
}
template <typename V, int G, int M, int PAT>
__host__ __device__ constexpr uint32_t st_buffer_bytes() {
    return (uint32_t)(st_slots<PAT>() * M) * st_val_slot<V, G>() + (uint32_t)M * st_mask_slot<G>();
}

// MINB: resident blocks the register budget is set for (8: 64 registers a
// thread, 1,024 threads an SM, some spilled; 4: 128 registers, 512 threads,
// more gathers in flight a thread); the autotuner picks between them.
template <typename F, typename FX, int NV, int VK, int M, int PAT, int MINB, class Epi,
          typename V = F>
__global__ void __launch_bounds__(ST_THREADS, MINB)
    k_spmv_stencil(StencilArgs A, const FX *__restrict__ x, Epi epi, uint32_t nbuf,
                   unsigned *flag) {
    constexpr int G = NV / VK;
    constexpr uint32_t TX = ST_THREADS / G;
    constexpr int K = st_slots<PAT>();
    constexpr int NRV = K * M, NR = NRV + M;  // staged runs: values (s, m), masks (m)
    constexpr int NU = (NR + 31) / 32;        // runs a lane of warp 0 stages
    constexpr uint32_t VS = st_val_slot<V, G>(), MS = st_mask_slot<G>();
    constexpr uint32_t BUF = st_buffer_bytes<V, G, M, PAT>();
    constexpr int CENTER = st_slot<PAT>(0, 0, 0);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint8_t shift[2][NR];  // where run r's first row lands in its slot
    const uint32_t n = A.n, S = A.S;
    const V *__restrict__ val = (const V *)A.val;
    const uint32_t *__restrict__ mask = A.mask;
    const uint32_t nchunks = (S + TX - 1) / TX;
    const uint32_t ngroups = (uint32_t)(((uint64_t)n + (uint64_t)M * S - 1) / ((uint64_t)M * S));
    const uint32_t ntiles = ngroups * nchunks;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t p = threadIdx.x / G;
    const int k0 = (threadIdx.x % G) * VK;
    if (threadIdx.x == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t n_issued = 0, n_used = 0;
    bool timed_out = false;
    // warp 0: stage tile t (rows b0 + m*S + [0, w) of each line m, cut at n)
    // into the next buffer
    auto issue = [&](uint32_t t) {
        if (t >= ntiles) return;
        const uint32_t bsel = n_issued % nbuf;
        unsigned char *buf = smem_raw + (size_t)bsel * BUF;
        uint64_t *mb = &mbar[bsel];
        ++n_issued;
        const uint32_t x0 = (t % nchunks) * TX;
        const uint32_t b0 = (t / nchunks) * (uint32_t)M * S + x0;
        const uint32_t w = S - x0 < TX ? S - x0 : TX;
        const void *src[NU];
        void *dst[NU];
        uint32_t nb[NU];
        uint32_t total = 0;
#pragma unroll
        for (int u = 0; u < NU; ++u) {
            const int r = lane + 32 * u;
            nb[u] = 0;
            if (r < NR) {
                const int m = r < NRV ? r % M : r - NRV;
                const uint64_t rb = (uint64_t)b0 + (uint64_t)m * S;
                const uint32_t r0 = rb < n ? (uint32_t)rb : n;
                const uint32_t r1 = rb + w < n ? (uint32_t)(rb + w) : n;
                if (r < NRV) {
                    const uint32_t e0 = (uint32_t)(r / M) * n + r0;
                    shift[bsel][r] = (uint8_t)stage_shift<V>(val, e0);
                    if (r1 > r0) {
                        const V *sp;
                        V *dp;
                        nb[u] = stage_range<V>((V *)(buf + (size_t)r * VS), val,
                                               (uint64_t)K * n, e0, e0 + (r1 - r0), sp, dp);
                        src[u] = sp;
                        dst[u] = dp;
                    }
                } else {
                    shift[bsel][r] = (uint8_t)stage_shift<uint32_t>(mask, r0);
                    if (r1 > r0) {
                        const uint32_t *sp;
                        uint32_t *dp;
                        nb[u] = stage_range<uint32_t>(
                            (uint32_t *)(buf + (size_t)NRV * VS + (size_t)m * MS), mask, n, r0,
                            r1, sp, dp);
                        src[u] = sp;
                        dst[u] = dp;
                    }
                }
            }
            total += nb[u];
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) total += __shfl_xor_sync(0xffffffffu, total, off);
        __syncwarp();
        if (lane == 0) mbar_arrive_expect(mb, total);  // releases the plain-load writes
        __syncwarp();
        fence_proxy_async_smem();
#pragma unroll
        for (int u = 0; u < NU; ++u)
            if (nb[u]) bulk_g2s(dst[u], src[u], nb[u], mb);
    };
    if (warp == 0) issue(blockIdx.x);
    const int64_t last = (int64_t)n - 1;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t tn = t + gridDim.x;
        if (nbuf == 2 && warp == 0) issue(tn);
        const uint32_t bsel = n_used % nbuf;
        // a copy that never landed: every thread of the block stops here
        if (__syncthreads_or(!mbar_wait(&mbar[bsel], (n_used / nbuf) & 1u))) {
            timed_out = true;
            break;
        }
        ++n_used;
        const unsigned char *buf = smem_raw + (size_t)bsel * BUF;
        const uint32_t x0 = (t % nchunks) * TX;
        const uint32_t i0 = (t / nchunks) * (uint32_t)M * S + x0 + p;  // row of line 0
        const uint32_t w = S - x0 < TX ? S - x0 : TX;
        if (p < w && i0 < n) {
            // staged value of slot s for line m's row
            auto vat = [&](int s, int m) -> V {
                const int r = s * M + m;
                return ((const V *)(buf + (size_t)r * VS))[shift[bsel][r] + p];
            };
            uint32_t msk[M];
            F y[M][VK];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const uint64_t i = (uint64_t)i0 + (uint64_t)m * S;
                const bool in = i < n;
                const uint32_t *mr = (const uint32_t *)(buf + (size_t)NRV * VS + (size_t)m * MS);
                msk[m] = in ? mr[shift[bsel][NRV + m] + p] : 0u;
#pragma unroll
                for (int v = 0; v < VK; ++v) y[m][v] = in ? epi.init(i, k0 + v) : F(0);
            }
            const bool df = A.diag_first != 0;
            if (df) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const bool has = (msk[m] >> CENTER) & 1u;
                    const uint32_t ic = has ? i0 + (uint32_t)m * S : 0u;
                    FX xv[VK];
                    ld_x<FX, VK>(x + (ic * (uint32_t)NV + (uint32_t)k0), xv);
                    const F av = val_as<F, V>(vat(CENTER, m));
#pragma unroll
                    for (int v = 0; v < VK; ++v) {
                        const F sum = add(y[m][v], mul((F)xv[v], av));
                        y[m][v] = has ? sum : y[m][v];
                    }
                }
            }
#pragma unroll
            for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll
                for (int l = -1; l <= M; ++l) {
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) {
                        // the carried rows this x row is a neighbour of (compile time)
                        bool any = false;
#pragma unroll
                        for (int m = 0; m < M; ++m) {
                            const int dy = l - m;
                            if (dy >= -1 && dy <= 1 && st_slot<PAT>(dz, dy, dx) >= 0) any = true;
                        }
                        if (!any) continue;
                        int64_t c = (int64_t)i0 + (int64_t)dz * A.S2 + (int64_t)l * S + dx;
                        // rows that have none of these entries may point outside x:
                        // read a valid row instead (its values are not used)
                        c = c < 0 ? 0 : (c > last ? last : c);
                        FX xv[VK];
                        ld_x<FX, VK>(x + ((uint32_t)c * (uint32_t)NV + (uint32_t)k0), xv);
#pragma unroll
                        for (int m = 0; m < M; ++m) {
                            const int dy = l - m;
                            if (dy < -1 || dy > 1) continue;
                            const int s = st_slot<PAT>(dz, dy, dx);
                            if (s < 0) continue;
                            const bool has = ((msk[m] >> s) & 1u) && !(s == CENTER && df);
                            const F av = val_as<F, V>(vat(s, m));
#pragma unroll
                            for (int v = 0; v < VK; ++v) {
                                const F sum = add(y[m][v], mul((F)xv[v], av));
                                y[m][v] = has ? sum : y[m][v];
                            }
                        }
                    }
                }
            }
            F none[1] = {F(0)};
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const uint64_t i = (uint64_t)i0 + (uint64_t)m * S;
                if (i < n) {
#pragma unroll
                    for (int v = 0; v < VK; ++v) epi.store(i, k0 + v, y[m][v], none);
                }
            }
        }
        __syncthreads();  // every reader is done with this tile's buffer
        if (nbuf == 1 && warp == 0) issue(tn);
    }
    if (timed_out && threadIdx.x == 0) {
        // raise the flag; no block exits with a copy into its shared memory
        // still in flight (bounded waits)
        atomicOr(flag, 1u);
        for (uint32_t u = n_used; u < n_issued; ++u) mbar_wait(&mbar[u % nbuf], (u / nbuf) & 1u);
    }
}

}  // namespace k
}  // namespace xg
