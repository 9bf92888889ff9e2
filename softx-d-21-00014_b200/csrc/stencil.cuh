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
// lines) and VK right-hand sides. For each plane dz and each of the M+2
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

template <typename F, typename FX, int NV, int VK, int M, int PAT, class Epi, typename V = F>
__global__ void __launch_bounds__(ST_THREADS, 8)
    k_spmv_stencil(StencilArgs A, const FX *__restrict__ x, Epi epi) {
    constexpr int G = NV / VK;
    const uint32_t n = A.n, S = A.S;
    const uint64_t t = (uint64_t)blockIdx.x * ST_THREADS + threadIdx.x;
    const uint64_t slot_row = t / G;  // (group of M lines, position in the line)
    const int k0 = (int)(t % G) * VK;
    const uint64_t b = (slot_row / S) * (uint64_t)M * S + slot_row % S;
    if (b >= n) return;
    const V *__restrict__ val = (const V *)A.val;
    uint32_t msk[M];
    F y[M][VK];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const uint64_t i = b + (uint64_t)m * S;
        msk[m] = i < n ? __ldg(&A.mask[i]) : 0u;
#pragma unroll
        for (int v = 0; v < VK; ++v) y[m][v] = i < n ? epi.init(i, k0 + v) : F(0);
    }
    const int64_t bi = (int64_t)b;
    const int64_t last = (int64_t)n - 1;
    constexpr int CENTER = st_slot<PAT>(0, 0, 0);
    const bool df = A.diag_first != 0;
    if (df) {
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const uint64_t i = b + (uint64_t)m * S;
            const uint64_t ic = i < n ? i : (uint64_t)last;
            FX xv[VK];
            ld_x<FX, VK>(x + ((uint32_t)ic * (uint32_t)NV + (uint32_t)k0), xv);
            const F av = val_as<F, V>(__ldg(&val[(uint64_t)CENTER * n + ic]));
            const bool has = (msk[m] >> CENTER) & 1u;
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
                int64_t c = bi + (int64_t)dz * A.S2 + (int64_t)l * S + dx;
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
                    const uint64_t i = b + (uint64_t)m * S;
                    const uint64_t ic = i < n ? i : (uint64_t)last;
                    const F av = val_as<F, V>(__ldg(&val[(uint64_t)s * n + ic]));
                    const bool has = ((msk[m] >> s) & 1u) && !(s == CENTER && df);
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
        const uint64_t i = b + (uint64_t)m * S;
        if (i < n) {
#pragma unroll
            for (int v = 0; v < VK; ++v) epi.store(i, k0 + v, y[m][v], none);
        }
    }
}

}  // namespace k
}  // namespace xg
