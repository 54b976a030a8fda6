// postfit.h -- calls on a fitted state outside the coordinate-descent loop:
// the Fisher information over a set of columns (fisher.cu) and the predictive
// log-likelihood / estimates (predict.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "types.h"

namespace ccdb {

// Columns whose Fisher information rows one pass of fisher.cu produces: 32
// passes over the gathered columns four times fewer than 8 (238 registers a
// thread, no spills; 1.07 ms against 2.05 ms for a 1,001-column matrix).
constexpr int kFisherSlots = 32;

struct FisherParams {
    // CompressedDataMatrix
    const int64_t* col_ptr;
    const int32_t* rows;
    const int64_t* val_ptr;
    const double* vals;
    const uint8_t* fmt;
    int64_t K;
    int32_t model;     // M_LOGISTIC, M_POISSON, M_CLR, M_CPR, M_COX
    int32_t grouped;   // 1: Survival increment + strata cross terms (CLR, CPR, Cox)
    // independent rows: row[2k] = {xBeta, offsExpXBeta}, row[2k+1] = {denominator, weight}
    const double2* row;
    // grouped rows: xbe[k] = {xBeta, offsExpXBeta}, group of the row, per-group denominator
    const double2* xbe;
    const int32_t* grp;
    const double* gden;
    int64_t N;         // groups; group N holds rows dropped by a zero weight
    // scratch: U[k * kFisherSlots + t] = value of the t-th slot's column at row k (0 if absent);
    // C[g * kFisherSlots + t] = sum of offsExpXBeta * x over the t-th column's rows of group g
    double* U;
    double* C;
    // the requested columns and the n x n row-major result
    const int32_t* idx;
    int32_t n;
    int32_t pad;
    double* out;
};

// Slots t < n_slots take columns idx[p0 + t]; U (and C) must be zero on entry.
cudaError_t launch_fisher_scatter(const FisherParams& P, int p0, int n_slots, int64_t max_entries,
                                  cudaStream_t s);
// Entries (p0 + t, q) and (q, p0 + t) of `out` for every q >= p0 + t.
cudaError_t launch_fisher_gather(const FisherParams& P, int p0, int n_slots, cudaStream_t s);

struct PredictParams {
    int64_t K;
    int32_t model;
    int32_t grouped;
    const double2* row;   // independent rows (see FisherParams)
    const double2* xbe;   // grouped rows
    const int32_t* grp;
    const double* gden;   // CLR/CPR: per-stratum denominator; Cox: accumulated denominator
    int64_t N;
    const double* y;
    const double* w;      // held-out weights
};

// Per-block partial sums of the predictive log-likelihood into part[0 .. n_blocks).
cudaError_t launch_predictive_loglik(const PredictParams& P, double* part, int n_blocks, cudaStream_t s);
// out[k] = predictEstimate(xBeta_k) for every row.
cudaError_t launch_predictive_estimates(const PredictParams& P, double* out, cudaStream_t s);

}  // namespace ccdb
