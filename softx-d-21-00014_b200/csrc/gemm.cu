// BF16 GEMM on the fifth-generation tensor cores (tcgen05), FP32 accumulate:
//   C[M][N] = A[M][K] * B[N][K]^T   (both operands K-major, row-major storage)
// with a fused epilogue (bias, ReLU, ReLU-derivative mask, BF16 or FP32
// output). It carries the dense layers of the learned coarse initial guess,
// the only tensor-core work of the solve phase.
//
// One CTA computes a 128 x 128 tile: warp 0 streams 128 x 64 tiles of A and B
// into a ring of 128-byte-swizzled shared-memory stages with TMA
// (cp.async.bulk.tensor, completion on an mbarrier per stage), warp 1 issues
// tcgen05.mma (M = 128, N = 128, K = 16 per instruction) into a 128-column
// TMEM accumulator and releases each stage with tcgen05.commit, and warps 2-5
// read the accumulator back with tcgen05.ld (each warp its 32-lane quarter),
// apply the epilogue and store. Every wait is bounded (global timer); a wait
// that runs out raises the library's timeout flag and the CTA still frees its
// TMEM before it exits.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "device.h"
#include "ops.h"

namespace xg {
namespace ops {
namespace mm {

#ifndef XG_GEMM_STAGES
#define XG_GEMM_STAGES 3
#endif
// Three stages (97 KB of shared memory) let two CTAs share an SM, so that one
// CTA's epilogue overlaps the other's main loop.
constexpr int BM = 128, BN = 128, BK = 64, STAGES = XG_GEMM_STAGES;
constexpr int CTAS_PER_SM = STAGES <= 3 ? 2 : 1;
constexpr uint32_t TILE_A = BM * BK * 2, TILE_B = BN * BK * 2;  // 16 KB each
constexpr uint32_t STAGE_BYTES = TILE_A + TILE_B;
constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
constexpr int THREADS = 192;
constexpr uint32_t TMEM_COLS = 128;

enum Mode : int {
    F32 = 0,         // C = acc (+ bias)
    BF16 = 1,        // C = bf16(acc (+ bias))
    BF16_RELU = 2,   // C = bf16(max(acc + bias, 0))
    BF16_MASK = 3,   // C = bf16(acc) where aux > 0, else 0 (ReLU derivative)
};

__device__ __forceinline__ uint32_t saddr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory matrix descriptor for a K-major operand tile stored with
// the 128-byte swizzle: rows of 128 B (64 BF16), 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);  // start address, 16-byte units
    d |= (uint64_t)1 << 16;                   // leading byte offset (unused when swizzled)
    d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset: one 8-row group
    d |= (uint64_t)1 << 46;                   // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                   // layout: 128-byte swizzle
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 128, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
        "{%2, %3}], [%4];" ::"r"(saddr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(THREADS, CTAS_PER_SM)
    k_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                int K, void *C, uint64_t ldc, int mode, const float *__restrict__ bias,
                const __nv_bfloat16 *__restrict__ aux, uint64_t ld_aux, unsigned *flag) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], acc_full;
    __shared__ uint32_t tmem_holder;
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int KB = K / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            k::mbar_init(&full[s], 1);
            k::mbar_init(&empty[s], 1);
        }
        k::mbar_init(&acc_full, 1);
        k::mbar_init_fence();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         saddr(&tmem_holder)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_holder;
    bool ok = true;

    if (warp == 0 && lane == 0) {
        // producer: TMA loads of the K blocks into the stage ring
        for (int kb = 0; kb < KB && ok; ++kb) {
            const int s = kb % STAGES;
            const uint32_t u = (uint32_t)(kb / STAGES);
            if (kb >= STAGES && !k::mbar_wait(&empty[s], (u - 1) & 1u)) ok = false;
            if (!ok) break;
            k::mbar_arrive_expect(&full[s], STAGE_BYTES);
            unsigned char *a = smem + (size_t)s * STAGE_BYTES;
            tma_load_2d(a, &ta, kb * BK, m0, &full[s]);
            tma_load_2d(a + TILE_A, &tb, kb * BK, n0, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: four K = 16 steps per stage, then release the stage
        for (int kb = 0; kb < KB && ok; ++kb) {
            const int s = kb % STAGES;
            const uint32_t u = (uint32_t)(kb / STAGES);
            if (!k::mbar_wait(&full[s], u & 1u)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t a = saddr(smem + (size_t)s * STAGE_BYTES);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
                mma_bf16(tmem, sw128_desc(a + kk * 32), sw128_desc(a + TILE_A + kk * 32),
                         (kb | kk) != 0);
            mma_commit(&empty[s]);
        }
        mma_commit(&acc_full);  // arrives once every MMA issued above has completed
    } else if (warp >= 2) {
        // epilogue: this warp's 32 TMEM lanes are rows q*32 .. q*32+31 of the tile
        const int q = warp & 3;
        if (!k::mbar_wait(&acc_full, 0)) ok = false;
        tc_fence_after();
        if (ok) {
            const uint64_t row = (uint64_t)m0 + q * 32 + lane;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
                const int n = n0 + c0;
                if (bias && mode != BF16_MASK) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] += __ldg(&bias[n + i]);
                }
                if (mode == F32) {
                    float4 *dst = (float4 *)((float *)C + row * ldc + n);
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                } else {
                    if (mode == BF16_RELU) {
#pragma unroll
                        for (int i = 0; i < 32; ++i) v[i] = fmaxf(v[i], 0.f);
                    } else if (mode == BF16_MASK) {
                        const __nv_bfloat16 *m = aux + row * ld_aux + n;
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (!(__bfloat162float(m[i]) > 0.f)) v[i] = 0.f;
                    }
                    uint4 *dst = (uint4 *)((__nv_bfloat16 *)C + row * ldc + n);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        __nv_bfloat162 h[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            h[j] = __floats2bfloat162_rn(v[8 * i + 2 * j], v[8 * i + 2 * j + 1]);
                        dst[i] = *reinterpret_cast<uint4 *>(h);
                    }
                }
            }
        }
    }
    if (!ok) atomicOr(flag, 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        XG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        XG_REQUIRE(p && q == cudaDriverEntryPointSuccess, XAMG_ERR_CUDA,
                   "cuTensorMapEncodeTiled not available");
        fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// Tensor map of a row-major [rows][K] BF16 matrix read in 64 x box_rows boxes
// with the 128-byte swizzle.
CUtensorMap make_map(const void *ptr, uint64_t rows, uint64_t K, uint32_t box_rows) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {K, rows};
    const cuuint64_t strides[1] = {K * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr),
                                   dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    XG_REQUIRE(r == CUDA_SUCCESS, XAMG_ERR_CUDA, "tensor map encoding failed");
    return m;
}

}  // namespace

void gemm_bf16(uint64_t M, uint64_t N, uint64_t K, const void *A, const void *B, void *C,
               uint64_t ldc, int mode, const float *bias, const void *aux, uint64_t ld_aux,
               cudaStream_t s) {
    XG_REQUIRE(M % BM == 0 && N % BN == 0 && K % BK == 0 && K > 0, XAMG_ERR_INVALID_ARG,
               "gemm: M and N must be multiples of 128, K a positive multiple of 64");
    XG_REQUIRE(mode >= F32 && mode <= BF16_MASK, XAMG_ERR_INVALID_ARG, "gemm: unknown mode");
    XG_REQUIRE(ldc >= N && ldc % 8 == 0, XAMG_ERR_INVALID_ARG, "gemm: ldc below N or not a multiple of 8");
    XG_REQUIRE(((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) % 16 == 0, XAMG_ERR_INVALID_ARG,
               "gemm: A, B and C must be 16-byte aligned");
    XG_REQUIRE(mode != BF16_MASK || (aux && ld_aux >= N), XAMG_ERR_INVALID_ARG,
               "gemm: the mask mode needs aux");
    XG_REQUIRE(M / BM <= 65535, XAMG_ERR_INVALID_ARG, "gemm: M too large");
    const CUtensorMap ta = make_map(A, M, K, BM), tb = make_map(B, N, K, BN);
    static bool attr = false;
    if (!attr) {
        XG_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SMEM_BYTES));
        attr = true;
    }
    dim3 grid((unsigned)(N / BN), (unsigned)(M / BM));
    k_gemm_bf16<<<grid, THREADS, SMEM_BYTES, s>>>(ta, tb, (int)K, C, ldc, mode, bias,
                                                  (const __nv_bfloat16 *)aux, ld_aux,
                                                  ctx().red().flag);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

}  // namespace mm
}  // namespace ops
}  // namespace xg
