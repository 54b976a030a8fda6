// csr_device.h -- the row-major copy of a CompressedDataMatrix built on the
// device from the uploaded column-major arrays (csr_device.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ccdb {

// Rows longer than this are not sorted on the device (the caller builds the
// copy on the host instead): a row is sorted by one thread.
constexpr int32_t kCsrDeviceMaxRow = 1024;

struct CsrDeviceArgs {
    int64_t K;
    int32_t J;
    const int64_t* col_ptr;  // J + 1 row-id offsets (sparse, indicator columns)
    const int32_t* rows;
    const int64_t* val_ptr;  // J + 1 value offsets (sparse, dense columns)
    const double* vals;
    const uint8_t* fmt;
};

// Pass 1: per-row entry counts (`counts`, K int32, zeroed here), their
// exclusive sum into `row_ptr` (K + 1) and `cursor` (K), and the longest row
// into `*max_row` (device).  The caller reads max_row and, when it is at most
// kCsrDeviceMaxRow, runs pass 2.
cudaError_t csr_device_count(const CsrDeviceArgs& a, int32_t* counts, int64_t* row_ptr, int64_t* cursor,
                             int32_t* max_row, cudaStream_t s);
// Pass 2: every entry placed in its row (`col`, `val`), then each row sorted
// by column: per row the columns in increasing order, dense-like columns
// (DENSE, INTERCEPT) at every row -- the layout of build_csr (csr_host.h).
cudaError_t csr_device_fill(const CsrDeviceArgs& a, const int64_t* row_ptr, int64_t* cursor, int32_t* col,
                            double* val, cudaStream_t s);

}  // namespace ccdb
