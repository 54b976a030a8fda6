// csr_host.h -- the row-major copy of a CompressedDataMatrix (host side).
#pragma once

#include <cstdint>
#include <vector>

namespace ccdb {

struct HostCsr {
    std::vector<int64_t> row_ptr;  // K + 1
    std::vector<int32_t> col;      // entries of each row in increasing column order
    std::vector<double> val;
};

// Every entry of the matrix, row by row: per row its columns in increasing
// order, dense-like columns (DENSE, INTERCEPT) included at every row.  The
// result does not depend on `threads` (column ranges are counted and placed by
// one thread each, in column order).  A thread takes at least
// `min_per_thread` entries, and the per-thread row tables stay under 256 MiB.
HostCsr build_csr(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                  const int64_t* val_start, const double* vals, const uint8_t* fmt, int threads,
                  int64_t min_per_thread = int64_t(1) << 20);

}  // namespace ccdb
