// resident.h -- the single-CTA sweep of independent-row fits (resident.cu):
// the row state lives in shared memory for the whole findMode when it fits
// there, else in a global array the CTA alone reads and writes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "indep.h"

namespace ccdb {

// One active column in visiting order: its index, format flags (bit 0: row
// ids, bit 1: values, bit 2: indicator or intercept), entry count and the
// offsets of its row ids and values.
struct ResCol {
    int32_t j;
    int32_t flags;
    int64_t n;
    int64_t cb;
    int64_t vb;
};

struct ResidentParams {
    IndepParams P;         // matrix, row and column state, convergence (no schedule)
    const ResCol* recs;    // the active columns in visiting order
    int32_t n_active;
    int32_t weighted;      // 0: every row weight is 1.0 and is not read
    // optional per-batch SM-clock stamps of the first trace_n batches (profiling
    // aid): start, gradients done, decided, applied, next; batch size, first
    // nonzero step (kResidentTraceWords per batch)
    long long* trace;
    int32_t trace_n;
    int32_t pad;
    // {xBeta, denominator} of every row in global memory (K entries), for fits
    // whose row state does not fit shared memory; nullptr: shared memory
    double2* rs;
};

constexpr int kResidentTraceWords = 8;

int resident_threads();
// the most rows whose state fits the kernel's shared memory on the current device
cudaError_t resident_max_rows(int model, int64_t* rows);
// a column of at most this many entries is one warp's in a speculative batch
// when the row state is in global memory (shared memory: 256)
constexpr int64_t kResidentWarpMaxGlobal = 2048;
cudaError_t launch_resident_sweep(const ResidentParams& R, cudaStream_t stream);

}  // namespace ccdb
