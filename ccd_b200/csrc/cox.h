// cox.h -- parameters and launchers of the Breslow Cox engine (cox.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "types.h"

namespace ccdb {

struct CoxParams {
    // CompressedDataMatrix
    const int64_t* col_ptr;
    const int32_t* rows;
    const int64_t* val_ptr;
    const double* vals;
    const uint8_t* fmt;
    int64_t K;
    int64_t N;  // risk-set groups after regrouping
    // rows
    double2* xbe;          // {xBeta, offsExpXBeta}
    const double* w;       // row weights (1.0 when unweighted)
    const double* y;
    const int32_t* grp;    // group of each row (N: dropped by a zero weight)
    const int32_t* rstrat; // stratum index of each row
    int32_t weighted;
    int32_t mixed;  // Cox, CCDB_PRECISION_MIXED: FP32 exp and per-entry gradient terms
    // groups (N + 1 slots; slot N absorbs dropped rows and reads as zero)
    double* denom;
    double* D;
    double* S1;
    double* S2;
    const double* nEv;
    const uint8_t* gfirst;  // group starts its stratum
    const uint8_t* glast;   // group ends its stratum
    const int64_t* grow;    // first row of each group (N + 1 entries)
    const double* xjy;
    DevStatus* st;
    long long wait_limit_ns;
};

int cox_scan_tiles(int64_t N);
size_t cox_tail_bytes();
cudaError_t launch_cox_gh(const CoxParams& P, const int32_t* cols, int ncols, double2* out,
                          cudaStream_t s);
cudaError_t launch_cox_update(const CoxParams& P, int j, double delta, cudaStream_t s);
cudaError_t launch_cox_remaining(const CoxParams& P, cudaStream_t s);
// D from denom, then S1/S2 from D (two single-pass look-back scans); `epoch`
// must differ from every earlier call on the same status arrays.
cudaError_t launch_cox_scans(const CoxParams& P, unsigned* tickets, int* status, void* tails,
                             int epoch, cudaStream_t s);
cudaError_t launch_cox_objective(const CoxParams& P, double2* red, int nblocks, cudaStream_t s);

// Grouped models (conditional logistic / Poisson): grp = stratum, N = strata,
// denom per stratum, grow = first row of each stratum.
cudaError_t launch_grouped_gh(const CoxParams& P, const int32_t* cols, int ncols, double2* out,
                              cudaStream_t s);
cudaError_t launch_grouped_update(const CoxParams& P, int j, double delta, cudaStream_t s);
cudaError_t launch_grouped_remaining(const CoxParams& P, cudaStream_t s);
cudaError_t launch_grouped_objective(const CoxParams& P, double2* red, int nblocks, cudaStream_t s);

}  // namespace ccdb
