// batch.h -- parameters of the instance-batched sweep (batch.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "types.h"

namespace ccdb {

struct BatchResult {
    int32_t flag;
    int32_t iterations;
    double loglik;
    double objective;
    double pred_loglik;  // held-out rows' predictive log-likelihood
    int64_t steps;       // coordinate steps taken (all sweeps)
    int64_t updates;     // nonzero steps
    int64_t update_entries;  // entries touched by the nonzero steps
    int64_t sweep_entries;   // entries gathered by the gradient passes
};

struct BatchParams {
    const int64_t* col_ptr;
    const int32_t* rows;
    const int64_t* val_ptr;
    const double* vals;
    const uint8_t* fmt;
    int64_t K;
    int32_t J;
    int32_t model;
    int32_t n_inst;
    int32_t conv;
    int32_t max_iter;
    int32_t pad0;
    double tol;
    double initial_bound;
    const double* y;
    const int32_t* row_fold;   // K or NULL
    const int32_t* holdout;    // n_inst or NULL
    const double* variance;    // n_inst
    const int32_t* ptype;      // J
    const double* offset_vals; // K values of an offset column 0, or NULL
    const double* ll_fixed;    // n_inst (Poisson) or NULL
    double2* row;              // n_inst x 2K
    double* beta;              // n_inst x J
    double* hdelta;            // n_inst x J
    double* xjy;               // n_inst x J
    BatchResult* results;      // n_inst
    const int32_t* order;      // launch order of the instances (CTA b runs order[b]), or NULL
    // mixed precision (batch_mixed.cu): CTA b runs instances order[b*group .. b*group+group-1]
    // in lockstep; their state is interleaved instance-minor so that one row's
    // state for the whole group is one 32-byte sector at group 4.
    int32_t group;             // instances per CTA: 1, 2 or 4
    int32_t pad1;
    double* xg;                // n_groups x K x group: xBeta
    double* beta_g;            // n_groups x J x group
    double* hd_g;              // n_groups x J x group
    double* xjy_g;             // n_groups x J x group
    // optional phase trace of CTA 0, sweep `trace_sweep`: per column six SM clock
    // stamps (start, issued, terms, reduced, updated, end); NULL: off
    long long* trace;
    int32_t trace_sweep;
    int32_t pad6;
    // mixed: per entry of the row-indexed columns, row id | fold code << 24
    // (fold code: the row's fold id, or 127 for rows in no fold)
    const int32_t* keys;
    // mixed: CTAs per group (a thread-block cluster; CTA r owns rows
    // [K r / C, K (r + 1) / C)) and, when above 1, per row-indexed column the
    // C + 1 entry offsets where its rows cross those boundaries (J x (C + 1))
    int32_t cluster;
    int32_t stage_cap;         // mixed: staged entries per slice (1024 or 3072)
    int32_t pad5;
    int32_t pad4;
    const int32_t* split;
    int32_t* queue;            // mixed: next group to fit (zeroed before the launch)
    // mixed, clusters: raised (set to 1) by a CTA whose wait for the other CTAs'
    // column sums ran out; zeroed before the launch
    int32_t* abort;
    long long xch_wait_ns;     // mixed, clusters: bound on one exchange wait before abort
};

constexpr int kKeyRowBits = 24;
constexpr int32_t kKeyRowMask = (1 << kKeyRowBits) - 1;
constexpr int kKeyNoFold = 127;

cudaError_t launch_batch_sweep(const BatchParams& P, cudaStream_t stream);
cudaError_t launch_batch_mixed(const BatchParams& P, cudaStream_t stream);
constexpr int32_t kBatchTimeoutFlag = -100;  // result flag: a bounded device wait ran out

// keys[e] = rows[e] | code(fold[rows[e]]) << 24 for e < nnz
cudaError_t launch_batch_keys(const int32_t* rows, int64_t nnz, const int32_t* fold, int32_t* keys,
                              cudaStream_t stream);

}  // namespace ccdb
