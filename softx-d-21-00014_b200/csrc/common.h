// Shared definitions of the B200 solve-phase library: error codes, checks,
// the runtime NV set and small host utilities.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/xamg_b200.h"

namespace xg {

// An error raised anywhere below the C ABI; the ABI layer turns it into the
// negative status code and keeps the message for XAMG_b200_last_error().
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define XG_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw ::xg::Error(XAMG_ERR_CUDA, std::string(#call) + ": " +                   \
                                                 cudaGetErrorString(e_) + " at " __FILE__ \
                                                 ":" + std::to_string(__LINE__));          \
    } while (0)

#define XG_REQUIRE(cond, code, msg)                 \
    do {                                            \
        if (!(cond)) throw ::xg::Error(code, msg);  \
    } while (0)

// Right-hand-side block widths the kernels are instantiated for.
inline bool nv_supported(int nv) {
    return nv == 1 || nv == 2 || nv == 4 || nv == 8 || nv == 16 || nv == 32;
}

// XAMG's integer type codes (xamg_types.h:49-75) and the per-block hash
// F | I1<<3 | I2<<5 | I3<<7 | I4<<9 (bit_operations.h:67-88).
enum : uint16_t { I8_TYPE = 0, I16_TYPE = 1, I32_TYPE = 2, I64_TYPE = 3 };
enum : uint16_t { F32_TYPE = 5, F64_TYPE = 6 };
enum : uint16_t { I1_OFFSET = 3, I2_OFFSET = 5, I3_OFFSET = 7, I4_OFFSET = 9, F_MASK = 7 };

// define_int_type (bit_operations.h:119-129): smallest unsigned type whose
// maximum is >= range.
inline uint16_t define_int_type(uint64_t range) {
    if (range <= UINT8_MAX) return I8_TYPE;
    if (range <= UINT16_MAX) return I16_TYPE;
    if (range <= UINT32_MAX) return I32_TYPE;
    return I64_TYPE;
}

inline int int_type_bytes(uint16_t t) { return 1 << t; }

// encode_hash (csr_matrix.h:455-461) with the reduced-precision override of
// matrix_block::assemble (matrix.h:80-84).
inline uint16_t encode_hash(uint64_t nonzeros, uint64_t ncols, uint64_t block_nrows,
                            uint64_t block_ncols, bool f32, bool reduced_prec) {
    uint16_t hash = (uint16_t)((define_int_type(nonzeros) << I1_OFFSET) |
                               (define_int_type(ncols) << I2_OFFSET) |
                               (define_int_type(block_nrows) << I3_OFFSET) |
                               (define_int_type(block_ncols) << I4_OFFSET));
    hash |= f32 ? F32_TYPE : F64_TYPE;
    if (reduced_prec) {
        hash |= F_MASK;
        hash &= (uint16_t)(~F_MASK | F32_TYPE);
    }
    return hash;
}

// XAMG's core-range split (misc.h:47-55 with T = float64_t, part.h:115-134):
// the per-block size is n/nblocks rounded up to the next multiple of 8 (a
// full 8 is added when already aligned), the last blocks take what is left.
inline uint64_t split_range_f64(uint64_t size, int nblocks) {
    const uint32_t factor = 8;
    uint64_t core_size = size / nblocks;
    core_size += factor - (core_size % factor);
    return core_size;
}

}  // namespace xg
