// group_sweep.h -- the persistent findMode of the group engine (group_sweep.cu):
// Breslow Cox and the grouped models (conditional logistic / Poisson), one
// cooperative launch per findMode, no host round trip per coordinate.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "cox.h"
#include "types.h"

namespace ccdb {

constexpr int kGroupBatchMax = 1024;  // columns per speculative gradient batch
constexpr int kTraceStamps = 8;       // timestamps per traced nonzero step

// Aggregate of one CTA's share of a segmented scan (one or two channels).
struct SegAgg {
    int32_t f;
    int32_t pad;
    double v0, v1;
};

struct GroupSweepParams {
    CoxParams P;
    int32_t cox;            // 1: Breslow Cox (accumulated denominators and suffix sums)
    int32_t n_active;       // columns visited per sweep
    const int32_t* cols;    // the active columns in visiting order
    double* beta;
    double* hdelta;
    const int32_t* ptype;
    const double* pvar;
    int32_t conv;
    int32_t max_iter;
    double tol;
    double ll_fixed;
    int32_t batch_max;      // at most kGroupBatchMax
    int32_t J;
    double2* gh;            // 2 x kGroupBatchMax: (g, h) of the current batch, halves alternating
    double* dd;             // per entry of the updated column: w e_new - w e_old
    int32_t* ddg;           // per entry of the updated column: its group
    double2* red;           // 2 x grid: objective partials
    SegAgg* agg;            // 2 x grid: scan aggregates (prefix, suffix)
    unsigned* grid_bar;
    DevStatus* st;
    long long wait_limit_ns;
    int64_t* counters;      // [0]: nonzero steps, [1]: gradient batches (whole launch)
    // optional timestamps of the first trace_steps nonzero steps (profiling aid): per
    // step (kTraceStamps), the start of its batch, decided, rows updated, denominators,
    // rebuild phases 1 and 2 done, rebuilt, done
    unsigned long long* trace;
    int32_t trace_steps;
    int32_t pad;
};

cudaError_t group_sweep_occupancy(int* blocks_per_sm);
// The cluster form: one thread-block cluster of up to kMaxGroupCluster CTAs,
// hardware cluster barriers instead of grid barriers (fits whose groups and
// columns a few SMs cover).
constexpr int kMaxGroupCluster = 16;
constexpr int64_t kGroupClusterWork = 16384;  // groups + longest column per CTA below which a cluster serves
cudaError_t group_sweep_max_cluster(int* cluster);
cudaError_t launch_group_sweep(const GroupSweepParams& Q, int n_cta, bool cluster, cudaStream_t stream);
int group_sweep_threads();

}  // namespace ccdb
