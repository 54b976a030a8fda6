// indep.h -- parameters and launchers of the independent-row engine (indep.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "types.h"

namespace ccdb {

struct IndepParams {
    // CompressedDataMatrix on the device
    const int64_t* col_ptr;
    const int32_t* rows;
    const int64_t* val_ptr;
    const double* vals;
    const uint8_t* fmt;
    int64_t K;
    int32_t J;
    int32_t model;  // M_LOGISTIC or M_POISSON
    // row state: row[2k] = {xBeta, offsExpXBeta}, row[2k+1] = {denominator, weight}
    double2* row;
    const double* y;
    // per-column state
    double* beta;
    double* hdelta;
    const double* xjy;
    const int32_t* ptype;
    const double* pvar;
    // schedule
    const Seg* segs;
    const int64_t* cta_seg;
    const Task* tasks;
    int32_t n_levels;
    int32_t max_iter;
    unsigned* level_done;
    const int32_t* level_need;
    unsigned* col_arrive;
    double2* partials;
    unsigned* grid_bar;
    double2* red;  // 2 buffers x n_cta x 2 double2: {LL num, LL den}, {grad obj, log prior}
    // convergence
    int32_t conv;
    int32_t pad0;
    double tol;
    double ll_fixed;
    DevStatus* st;
    long long wait_limit_ns;  // bound on any single device-side wait
    // optional per-segment timestamps of the first sweep (profiling aid):
    // trace[3*si + {0,1,2}] = globaltimer at wait start, wait end, arrival
    unsigned long long* trace;
    // finer points: trace2[2*si] = end of phase 1, trace2[2*si+1] = last warp's end of phase 2
    unsigned long long* trace2;
    // cluster sweep: per level, 1 when it holds a split column (a second cluster barrier)
    const uint8_t* level_split;
};

int indep_threads();
int indep_max_split();
cudaError_t indep_sweep_occupancy(int model, int* blocks_per_sm);
cudaError_t launch_indep_sweep(const IndepParams& P, int n_cta, cudaStream_t stream);
// The cluster sweep: one thread-block cluster of `cluster` CTAs runs the whole
// findMode, levels separated by hardware cluster barriers.
constexpr int kMaxClusterSweep = 16;
// largest cluster size (16, 8, 4, 2, 1) of which one can be resident; 0 if none
cudaError_t cluster_sweep_max_size(int model, int* cluster);
cudaError_t launch_cluster_sweep(const IndepParams& P, int cluster, cudaStream_t stream);
cudaError_t launch_indep_gh(const IndepParams& P, int j, int64_t entries, double2* parts,
                            int max_parts, double2* out, cudaStream_t stream);
cudaError_t launch_indep_gh_batch(const IndepParams& P, const int32_t* cols, int ncols, double2* out,
                                  cudaStream_t stream);
cudaError_t launch_indep_update(const IndepParams& P, int j, uint8_t fmt, int64_t entries,
                                double delta, cudaStream_t stream);
cudaError_t launch_remaining_stats(double2* row, const double* xb, const double* w, int64_t K,
                                   double null_denom, cudaStream_t stream);
// one pass of the objective reduction into P.red[0 .. n_blocks) (buffer 0)
cudaError_t launch_indep_objective(const IndepParams& P, int n_blocks, cudaStream_t stream);
cudaError_t launch_xjy(const int64_t* col_ptr, const int32_t* rows, const int64_t* val_ptr,
                       const double* vals, const uint8_t* fmt, const double* y, const double* w,
                       int64_t K, int32_t J, double* xjy, cudaStream_t stream);
cudaError_t launch_xbeta_dense(const double* vals, double b, int64_t K, double* xb,
                               cudaStream_t stream);
// unit_values: count every non-zero entry as 1 (the MM product, see xbeta_csr_kernel)
cudaError_t launch_xbeta_csr(const int64_t* row_ptr, const int32_t* col_idx, const double* val,
                             const double* beta, int64_t K, double* xb, cudaStream_t stream,
                             int unit_values = 0);

}  // namespace ccdb
