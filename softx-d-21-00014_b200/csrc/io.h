// Files: XAMG's binary system format and the library's hierarchy files.
#pragma once

#include <cstdint>
#include <memory>
#include <string>

#include "amg.h"
#include "common.h"
#include "hcsr.h"

namespace xg {

struct SystemSize {
    uint32_t nrows, nnz;
};

// XAMG's binary system file (src/io/detail/reader.inl:47-177): u32 nrows,
// u32 nnz, u32 row[nrows+1], u32 col[nnz], f64 val[nnz], then optionally
// f64 b[nrows*nv] and f64 x[nrows*nv], both [row][rhs] interleaved.
SystemSize read_system_size(const char *path);
// Fills row/col/val and, when given, b and x (b = 1 and x = 0 where the file
// has none); returns bit 0 = b read, bit 1 = x read.
int read_system(const char *path, int nv, uint32_t *row, uint32_t *col, double *val, double *b,
                double *x);
void write_system(const char *path, uint32_t nrows, uint32_t nnz, const uint32_t *row,
                  const uint32_t *col, const double *val, int nv, const double *b,
                  const double *x);

// Hierarchy files: the host multigrid hierarchy built for a matrix under a
// parameter key, tied to that matrix by a fingerprint of its arrays.
uint64_t matrix_fingerprint(const HCsr &m);
void save_hierarchy(const char *path, const std::string &key, const HCsr &A0, const Hierarchy &H);
std::shared_ptr<const Hierarchy> load_hierarchy(const char *path, const HCsr &A0,
                                                std::string &key);

}  // namespace xg
