// Grid-stencil storage of a square CSR block and its SpMV kernel.
//
// A matrix whose every entry (i, j) lies on an offset j - i = dz*S2 + dy*S +
// dx with |dz|, |dy|, |dx| <= 1 (a 27-point box or a 7-point star on a
// lexicographically numbered grid of line stride S and plane stride S2, the
// finest level of a structured-grid problem) needs no column indices: the
// offset of each of its K slots is known. The upload keeps the CSR block and
// adds a copy in this form (gpu_index_compress = 3):
//   val[s][.]: the value of each row's entry in slot s (slot order =
//              ascending offset), 0 where the row has no such entry;
//   mask[.]:   bit s set where the row has the entry of slot s
// (rows at padded positions, below).
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
    const void *val;       // [K][LP][SP] values (stored type V)
    const uint32_t *mask;  // [LP][SP]
    uint32_t n, S, S2;
    uint32_t SP;           // padded line length (a multiple of 8)
    uint64_t slot;         // elements per slot array: LP * SP
    int diag_first;        // rows store their diagonal first
};

constexpr int ST_THREADS = 128;  // threads per block
constexpr int ST_LINES = 4;      // grid lines a thread carries (M)
constexpr uint32_t ST_LINE_PAD = 8;

// Stored layout: row i = line L * S + x is kept at element L * SP + x of its
// slot's array (SP = S rounded up to a multiple of 8), lines padded to a
// multiple of ST_LINES (and the arrays by one tile), so that every run a
// tile stages starts 16-byte aligned and has a fixed length.
//
// Tiles and staging. A tile is TX = ST_THREADS/G consecutive positions x0 ..
// x0+TX-1 of a group of M grid lines; its K*M value runs and M mask runs
// (TX elements each, those past the line unused) are copied into shared
// memory by the bulk-copy engine (cp.async.bulk, completion on an
// mbarrier), one or two buffers a block, the next tile's copies issued
// before the current tile is computed. x is gathered from global memory.
// Blocks are persistent (one wave) and take tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ...
template <int G>
__host__ __device__ constexpr uint32_t st_tx() { return ST_THREADS / G; }
template <typename V, int G, int M, int PAT>
__host__ __device__ constexpr uint32_t st_buffer_bytes() {
    return (uint32_t)(st_slots<PAT>() * M) * st_tx<G>() * (uint32_t)sizeof(V) +
           (uint32_t)M * st_tx<G>() * 4u;
}

// y[m][v] += x * a for the entries each carried row has (has: the select
// that skips an absent entry; FAST: every carried row has every entry of the
// pattern, so no select is needed).
template <typename F, int VK>
__device__ __forceinline__ void st_acc(F (&y)[VK], const F (&xv)[VK], F av, bool has) {
#pragma unroll
    for (int v = 0; v < VK; ++v) {
        const F sum = add(y[v], mul(xv[v], av));
        y[v] = has ? sum : y[v];
    }
}

// MINB: resident blocks the register budget is set for (8: 64 registers a
// thread, 1,024 threads an SM; 4: 128 registers, 512 threads, more gathers in
// flight a thread); the autotuner picks between them.
template <typename F, typename FX, int NV, int VK, int M, int PAT, int MINB, class Epi,
          typename V = F>
__global__ void __launch_bounds__(ST_THREADS, MINB)
    k_spmv_stencil(StencilArgs A, const FX *__restrict__ x, Epi epi, uint32_t nbuf,
                   unsigned *flag) {
    constexpr int G = NV / VK;
    constexpr uint32_t TX = st_tx<G>();
    constexpr int K = st_slots<PAT>();
    constexpr int NRV = K * M, NR = NRV + M;  // staged runs: values (s, m), masks (m)
    constexpr int NU = (NR + 31) / 32;        // runs a lane of warp 0 stages
    constexpr uint32_t BUF = st_buffer_bytes<V, G, M, PAT>();
    constexpr uint32_t VRUN = TX * (uint32_t)sizeof(V);
    constexpr int CENTER = st_slot<PAT>(0, 0, 0);
    constexpr uint32_t FULL = PAT == ST_BOX27 ? 0x7ffffffu : 0x7fu;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar[2];
    const uint32_t n = A.n, S = A.S, SP = A.SP;
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
    // warp 0: stage tile t into the next buffer
    auto issue = [&](uint32_t t) {
        if (t >= ntiles) return;
        const uint32_t bsel = n_issued % nbuf;
        unsigned char *buf = smem_raw + (size_t)bsel * BUF;
        uint64_t *mb = &mbar[bsel];
        ++n_issued;
        const uint64_t line0 = (uint64_t)(t / nchunks) * M, x0 = (t % nchunks) * TX;
        if (lane == 0) mbar_arrive_expect(mb, BUF);
        __syncwarp();
        fence_proxy_async_smem();
#pragma unroll
        for (int u = 0; u < NU; ++u) {
            const int r = lane + 32 * u;
            if (r < NRV) {
                const uint64_t e = (uint64_t)(r / M) * A.slot + (line0 + r % M) * SP + x0;
                bulk_g2s(buf + (size_t)r * VRUN, val + e, VRUN, mb);
            } else if (r < NR) {
                const uint64_t e = (line0 + (r - NRV)) * SP + x0;
                bulk_g2s(buf + (size_t)NRV * VRUN + (size_t)(r - NRV) * TX * 4u, mask + e, TX * 4u,
                         mb);
            }
        }
    };
    if (warp == 0) issue(blockIdx.x);
    const int64_t last = (int64_t)n - 1;
    const bool df = A.diag_first != 0;
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
        const V *vb = (const V *)buf + p;  // value of slot s, line m: vb[(s * M + m) * TX]
        const uint32_t *mbuf = (const uint32_t *)(buf + (size_t)NRV * VRUN) + p;
        const uint32_t x0 = (t % nchunks) * TX;
        const uint32_t i0 = (t / nchunks) * (uint32_t)M * S + x0 + p;  // row of line 0
        const bool active = x0 + p < S && i0 < n;
        uint32_t msk[M];
        bool full = active;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            msk[m] = active && (uint64_t)i0 + (uint64_t)m * S < n ? mbuf[m * TX] : 0u;
            full = full && msk[m] == FULL;
        }
        // a warp whose rows all have the whole pattern takes the path
        // without selects and clamps
        const bool fast = __all_sync(0xffffffffu, full);
        if (active) {
            F y[M][VK];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const uint64_t i = (uint64_t)i0 + (uint64_t)m * S;
#pragma unroll
                for (int v = 0; v < VK; ++v) y[m][v] = i < n ? epi.init(i, k0 + v) : F(0);
            }
            if (df) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const bool has = (msk[m] >> CENTER) & 1u;
                    const uint32_t ic = has ? i0 + (uint32_t)m * S : 0u;
                    FX xr[VK];
                    ld_x<FX, VK>(x + (ic * (uint32_t)NV + (uint32_t)k0), xr);
                    F xv[VK];
#pragma unroll
                    for (int v = 0; v < VK; ++v) xv[v] = (F)xr[v];
                    st_acc<F, VK>(y[m], xv, val_as<F, V>(vb[(CENTER * M + m) * TX]), has);
                }
            }
            // the plane loop stays rolled: both paths unrolled three times over
            // overflow the instruction cache (measured: instruction-fetch
            // stalls five times the issue rate)
            auto body = [&](auto fastc) {
                constexpr bool FAST = decltype(fastc)::value;
#pragma unroll 1
                for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll
                    for (int l = -1; l <= M; ++l) {
#pragma unroll
                        for (int dx = -1; dx <= 1; ++dx) {
                            // the carried rows this x row is a neighbour of
                            bool any = false;
#pragma unroll
                            for (int m = 0; m < M; ++m) {
                                const int dy = l - m;
                                if (dy >= -1 && dy <= 1 && st_slot<PAT>(dz, dy, dx) >= 0)
                                    any = true;
                            }
                            if (!any) continue;
                            int64_t c = (int64_t)i0 + (int64_t)dz * A.S2 + (int64_t)l * S + dx;
                            // rows that have none of these entries may point
                            // outside x: read a valid row instead (not used)
                            if (!FAST) c = c < 0 ? 0 : (c > last ? last : c);
                            FX xr[VK];
                            ld_x<FX, VK>(x + ((uint32_t)c * (uint32_t)NV + (uint32_t)k0), xr);
                            F xv[VK];
#pragma unroll
                            for (int v = 0; v < VK; ++v) xv[v] = (F)xr[v];
#pragma unroll
                            for (int m = 0; m < M; ++m) {
                                const int dy = l - m;
                                if (dy < -1 || dy > 1) continue;
                                const int s = st_slot<PAT>(dz, dy, dx);
                                if (s < 0) continue;
                                const F av = val_as<F, V>(vb[(s * M + m) * TX]);
                                if (FAST && s != CENTER)
                                    st_acc<F, VK>(y[m], xv, av, true);
                                else if (FAST)
                                    st_acc<F, VK>(y[m], xv, av, !df);
                                else
                                    st_acc<F, VK>(y[m], xv, av,
                                                  ((msk[m] >> s) & 1u) && !(s == CENTER && df));
                            }
                        }
                    }
                }
            };
            if (fast)
                body(std::true_type());
            else
                body(std::false_type());
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
