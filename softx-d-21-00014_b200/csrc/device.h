// Device-side containers of the library: owned device buffers, the per-process
// context (stream, reduction scratch, pinned staging), device vectors with
// XAMG's zero/initialised flags, and narrowed device CSR blocks.
#pragma once

#include <memory>
#include <vector>

#include "common.h"
#include "hcsr.h"
#include "kernels.cuh"

namespace xg {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t b) { alloc(b); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t b) {
        release();
        if (b) {
            cudaError_t e = cudaMalloc(&p, b);
            if (e != cudaSuccess) {
                p = nullptr;
                throw Error(XAMG_ERR_ALLOC, std::string("cudaMalloc(") + std::to_string(b) +
                                                " bytes): " + cudaGetErrorString(e));
            }
        }
        bytes = b;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T>
    T *as() const {
        return (T *)p;
    }
};

// A stream with its own reduction scratch and pinned host slots: the state a
// solve's kernels and scalar read-backs use. Lane 0 is the library's stream;
// the batch solve runs each system on a lane of its own, so that their
// kernels run concurrently without sharing scratch.
struct Lane {
    cudaStream_t stream = nullptr;
    DevBuf red_part, red_ticket, red_out;
    double *pinned = nullptr;
};

// Process-wide state created by XAMG_init (or lazily by the first call that
// needs the GPU). The stream and scratch fields are those of the current
// lane (use_lane swaps them).
struct Ctx {
    cudaStream_t stream = nullptr;
    DevBuf red_part;    // canonical-reduction partials: BMAX x 32 x 3 doubles
    DevBuf red_ticket;  // [0] reduction counter (zero between launches),
                        // [1] tile-size scratch, [2] wait-timeout flag
    DevBuf red_out;     // 96 doubles for reductions returned to the host
    double *pinned = nullptr;  // 256 doubles of pinned host memory
    int device = 0;
    int sms = 148;            // streaming multiprocessors of the device
    int device_request = -1;  // set by XAMG_b200_set_device before init
    bool ready = false;
    int lane = 0;             // current lane
    std::vector<Lane> lanes;  // parked state of the lanes not current

    void init();
    void shutdown();
    // Makes lane i current (creating it on first use); lane 0 is the default.
    void use_lane(int i);
    k::RedArgs red() const {
        return k::RedArgs{red_part.p, red_ticket.as<unsigned>(), red_ticket.as<unsigned>() + 2};
    }
    // Throws XAMG_ERR_TIMEOUT (and clears the flag) if a kernel's bounded wait
    // ran out since the last check; synchronises the stream.
    void check_flags();
};

Ctx &ctx();
Ctx &ctx_uninit();  // the context object without initialising it

// Count of kernel launches issued by this library (all launch helpers bump it).
extern uint64_t g_kernel_launches;

// A device vector: size rows of nv interleaved values (float or double), plus
// XAMG's state flags (vector.h:90-99). `zero` means "the contents are known to
// be zero and need not be read"; `init` means "has been written".
struct DVec {
    uint64_t n = 0;
    int nv = 0;
    bool f32 = false;
    bool zero = true;
    bool init = false;
    std::shared_ptr<DevBuf> buf;

    // New vectors start with zero contents (as XAMG's zero-flagged vectors
    // do in host memory): kernels that accumulate into a vector's memory
    // whatever its flag says (the F-cycle's prolongation) then read the
    // same values the reference reads.
    void alloc(uint64_t n_, int nv_, bool f32_);
    template <typename T>
    T *p() const {
        return buf ? (T *)buf->p : nullptr;
    }
    uint64_t elems() const { return n * (uint64_t)nv; }
};

// A CSR block on the device with XAMG's narrowed column type.
struct DCsr {
    uint64_t nrows = 0, ncols = 0, nnz = 0;
    int col_bytes = 4;
    bool f32 = false;
    bool bf16 = false;  // float matrix whose values are stored in BF16
    // float matrix whose values are stored in FP16 divided by vscale, a power
    // of two that puts the largest magnitude in [2^14, 2^15) (vscale at least
    // 2^-126)
    bool fp16 = false;
    float vscale = 1.0f;
    uint16_t hash = 0;
    DevBuf row, col, val;
    // largest number of entries in one tile of 256/nv rows, per nv = 1..32
    // (index log2 nv); 0 = not known yet
    uint32_t tile_max[6] = {0, 0, 0, 0, 0, 0};
    // SpMV autotuning (library-owned matrices, gpu_spmv_tune): the launch
    // shape measured fastest for the SpMVs without dot products, per
    // [value type is float][x type is float][log2 nv]: 0 = not tuned yet,
    // else 1 + 9 * (right-hand sides a thread: 0 default, 1 alternative, 2
    // eight) + 3 * (staging: 0 one buffer, 1 two, 2 none) + (tile run: 0 one,
    // 1 four, 2 sixteen), or 28: the warp-per-row kernel (k_spmv_wide), or
    // 29 + 3 * (right-hand sides a thread) + (staging): the plane walk
    bool tune_on = false;
    mutable uint8_t tuned[2][2][6] = {};
    // Plane walk (square matrices with long-range neighbours): walk_rows is
    // the distance, in rows, from a middle row to the centre of its farthest
    // neighbour cluster (the next grid plane of a structured grid; 0: none).
    // A block of the walk takes tiles one such distance apart in turn, so the
    // x rows of the two planes it gathered last are still in its SM's L1.
    // walk_force (gpu_spmv_tune = 5): always walk where walk_rows allows.
    uint32_t walk_rows = 0;
    bool walk_force = false;
    // Grid-stencil copy (gpu_index_compress = 3, csrc/stencil.cuh): the slot
    // pattern (-1: none, else k::ST_BOX27 or k::ST_STAR7), the line and plane
    // strides, the row order, the per-slot values in the CSR values' type and
    // the per-row entry masks (lines padded, csrc/stencil.cuh). The SpMVs
    // without dot products use it.
    int st_pat = -1;
    uint32_t st_S = 0, st_S2 = 0, st_SP = 0;  // strides; padded line length
    uint64_t st_slot = 0;                     // elements per slot array
    bool st_diag_first = false;  // rows store their diagonal first
    DevBuf st_val, st_mask;
    // with tuning on: the kernel measured fastest for the SpMVs without dot
    // products, per [value type is float][log2 nv]: 0 = not tuned yet, 1 the
    // stencil kernel with 64 registers a thread, 2 with 128, 3 the CSR kernel
    mutable uint8_t st_choice[2][6] = {};
    uint8_t st_force = 0;     // gpu_spmv_tune = 2: always the 128-register form
    bool wide_force = false;  // gpu_spmv_tune = 3: the warp-per-row kernel where allowed
    bool xs_force = false;    // gpu_spmv_tune = 4: the x-staged kernel where built
    // x-staged copy (gpu_spmv_tune = 4 with gpu_index_compress >= 2 on
    // multigrid levels, csrc/xstage.cuh), built for one nv: per canonical
    // tile of 256/nv rows its sorted unique columns, and every entry's slot
    // among them
    int xs_nv = 0;  // 0: none
    uint32_t xs_umax = 0, xs_emax = 0;
    DevBuf xs_uptr, xs_ucol, xs_slot;

    template <typename F>
    k::CsrArgs<F> args() const {
        return k::CsrArgs<F>{row.as<uint32_t>(), col.p, val.as<F>(), nrows, vscale};
    }
    bool empty() const { return nnz == 0; }
};

// Upload `h` narrowed per XAMG's rule (define_int_type on ncols for the
// column width; the I1 row-pointer width only enters the hash since row
// pointers stay 32-bit on the device). reduced_prec stores float values.
// narrow: 0 keeps 32-bit columns; 1 applies XAMG's rule; 2 additionally
// stores signed 16-bit offsets col - row (col_bytes = -2) for square
// matrices whose columns need more than 16 bits but whose entries all lie
// within 32767 of the diagonal; 3 also adds the grid-stencil copy where the
// matrix has that structure (stencil_layout).
// tune: let the SpMVs without dot products on this matrix pick their launch
// shape by measurement (gpu_spmv_tune = 1); 2: no measurement, the stencil
// copy's SpMVs use the 128-register form; 3: no measurement, SpMVs without
// dot products on matrices of at most 2^20 rows times nv use the
// warp-per-row kernel.
// bf16 (with f32): store the values rounded to float and then to BF16
// (round to nearest even), the arithmetic staying in float.
// fp16 (with f32, instead of bf16): store each value rounded to float,
// divided by the matrix's power-of-two scale (exact) and rounded to FP16
// (nearest even); the SpMVs read h * scale (exact). No grid-stencil or
// x-staged copy is built for such a matrix.
// xs_nv (narrow >= 2, tune = 4): also build the x-staged copy for SpMVs with
// xs_nv right-hand sides, where the rows are long enough and a tile's x rows
// fit in shared memory.
void upload_csr(const HCsr &h, DCsr &d, bool f32, int narrow, cudaStream_t s, int tune = 0,
                bool bf16 = false, int xs_nv = 0, bool fp16 = false);
void download_csr(const DCsr &d, uint32_t *row, void *col, void *val);

// Whether a square CSR block has the grid-stencil structure of
// csrc/stencil.cuh: every row sorted by column (or every row with its
// diagonal first and the rest sorted: diag_first), every offset col - row
// equal to dz*S2 + dy*S + dx (|dz|, |dy|, |dx| <= 1) with a slot in the
// pattern, S >= 3 and S2 >= 2S + 3 (so that ascending offsets are ascending
// (dz, dy, dx)). Sets the pattern, strides and order.
bool stencil_layout(const HCsr &h, int &pat, uint32_t &S, uint32_t &S2, bool &diag_first);

template <typename T>
void upload(DevBuf &b, const std::vector<T> &v, cudaStream_t s) {
    b.alloc(v.size() * sizeof(T));
    if (!v.empty()) XG_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T),
                                            cudaMemcpyHostToDevice, s));
}

}  // namespace xg
