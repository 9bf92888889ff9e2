// Host CSR block with 32-bit indices and double values: the form the C API
// fills (api/c/xamg_c_api.cpp:414-423) and the host setup produces.
#pragma once

#include <cstdint>
#include <vector>

namespace xg {

struct HCsr {
    uint64_t nrows = 0, ncols = 0;
    std::vector<uint32_t> row, col;
    std::vector<double> val;
    uint64_t nnz() const { return col.size(); }
};

}  // namespace xg
