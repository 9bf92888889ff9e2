// C entry points over the parts of the reference that compile on their own
// (bit_operations.h, xamg_types.h, misc/misc.h): XAMG's integer-type
// narrowing, bit-hash packing and core-range split. Built from the reference
// headers by `make ref` into oracle/_ref/ (never committed); the tests use it
// to pin the oracle's restatement of the same functions. Test infrastructure.
#include "xamg_headers.h"
#include "xamg_types.h"
#include "bit_operations.h"
#include "misc/misc.h"

// the reference headers declare `extern ID id` (the process identity of init.h)
ID id;

extern "C" {

uint16_t ref_define_int_type(uint64_t range) { return XAMG::define_int_type(range); }

// csr_matrix::encode_hash (csr_matrix.h:455-461) composed from the reference's
// own define_int_type, bit_encoding and create_bit_hash
uint16_t ref_encode_hash(uint64_t nnz, uint64_t ncols, uint64_t bnrows, uint64_t bncols,
                         int f32) {
    uint16_t F = f32 ? XAMG::bit_encoding<float32_t>() : XAMG::bit_encoding<float64_t>();
    return XAMG::matrix::create_bit_hash(F, XAMG::define_int_type(nnz),
                                         XAMG::define_int_type(ncols),
                                         XAMG::define_int_type(bnrows),
                                         XAMG::define_int_type(bncols));
}

void ref_parse_bit_hash(uint16_t hash, uint16_t *out5) {
    XAMG::matrix::parse_bit_hash(hash, out5[0], out5[1], out5[2], out5[3], out5[4]);
}

uint64_t ref_split_range_f64(uint64_t size, int nblocks) {
    return XAMG::misc::split_range<float64_t>(size, nblocks);
}

uint32_t ref_search_range(uint64_t col, const uint64_t *range, uint64_t len) {
    std::vector<uint64_t> r(range, range + len);
    return XAMG::misc::search_range(col, r);
}

}
