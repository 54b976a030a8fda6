// engine.h -- host-side objects behind the C ABI: a device context with an
// HBM budget, an immutable device CompressedDataMatrix, and per-fit state
// mirroring ModelSpecifics + CyclicCoordinateDescent.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ccdb.h"
#include "cox.h"
#include "indep.h"
#include "resident.h"
#include "schedule.h"
#include "step.h"

namespace ccdb {

// A failure with its C ABI status code (CCDB_ERR_*), raised by host code and
// turned into the status at the ABI boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, const char* what);

struct Context {
    int device = 0;
    int n_sm = 0;
    int max_ctas = 0;  // persistent sweep grids: at most this many CTAs (0: n_sm)
    int sweep_cluster = -1;  // largest resident cluster of the cluster sweep (-1: not queried)
    int64_t resident_rows = -1;  // most rows of a shared-memory resident sweep (-1: not queried)
    int group_cluster = -1;      // largest resident cluster of the group sweep (-1: not queried)
    size_t budget = 0;
    size_t in_use = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;  // this context's own stream-ordered pool
    std::mutex mu;
    std::map<void*, size_t> sizes;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;  // around a one-call fit
    // timing events of this context's fits (their calls are serialised on its
    // stream): [0], [1] around the sweep launches, [2], [3] around a whole
    // findMode.  Made once: creating and destroying events per fit waited on
    // other streams' work while they ran
    cudaEvent_t fev[4] = {nullptr, nullptr, nullptr, nullptr};
    // host waits: spin (default) or sleep until the device signals (blocking_wait),
    // for processes that run many contexts' calls at once (serving slots)
    bool blocking_wait = false;
    cudaEvent_t ev_wait = nullptr;

    void* alloc(size_t bytes);
    void release(void* p);
    // wait for everything queued on the context's stream
    cudaError_t wait();
    // event flags of this context's timing events
    unsigned event_flags() const { return blocking_wait ? cudaEventBlockingSync : cudaEventDefault; }
};

struct Matrix {
    Context* ctx = nullptr;
    int64_t K = 0;
    int32_t J = 0;
    std::vector<int64_t> col_start, val_start;
    std::vector<uint8_t> fmt;
    std::vector<int32_t> rows_h;
    std::vector<double> vals_h;
    int64_t* d_col_ptr = nullptr;
    int32_t* d_rows = nullptr;
    int64_t* d_val_ptr = nullptr;
    double* d_vals = nullptr;
    uint8_t* d_fmt = nullptr;
    // row-major copy, built on first need (computeXBeta with nonzero beta)
    int64_t* d_row_ptr = nullptr;
    int32_t* d_csr_col = nullptr;
    double* d_csr_val = nullptr;

    int64_t entries(int j) const;
    void ensure_csr(cudaStream_t s);
    ~Matrix();
};

struct DevSchedule {
    std::vector<uint8_t> fixed;
    int kind = 0;     // kSchedGrid or kSchedCluster
    int cluster = 0;  // CTAs of the cluster sweep
    uint8_t* level_split = nullptr;
    Schedule host;
    Seg* segs = nullptr;
    int64_t* cta_seg = nullptr;
    Task* tasks = nullptr;
    int32_t* level_need = nullptr;
    unsigned* level_done = nullptr;
    unsigned* col_arrive = nullptr;
    double2* partials = nullptr;
};

// Device tables of the Breslow Cox engine (cox.cu).
struct CoxDev {
    int64_t N = 0;  // risk-set groups
    int epoch = 0;  // scan epoch (status words are never reset)
    double2* xbe = nullptr;
    int32_t* grp = nullptr;
    int32_t* rstrat = nullptr;
    double *denom = nullptr, *D = nullptr, *S1 = nullptr, *S2 = nullptr, *nEv = nullptr;
    uint8_t *gfirst = nullptr, *glast = nullptr;
    int64_t* grow = nullptr;
    unsigned* tickets = nullptr;
    int* status = nullptr;
    void* tails = nullptr;
    int32_t* batch_cols = nullptr;
    double2* batch_out = nullptr;
    // the persistent sweep (group_sweep.cu): active columns, the updated
    // column's per-entry changes, scan aggregates, counters
    int32_t* sweep_cols = nullptr;
    double2* sweep_gh = nullptr;
    double* dd = nullptr;
    int32_t* ddg = nullptr;
    int64_t dd_cap = 0;
    void* agg = nullptr;
    int64_t* counters = nullptr;
    int64_t last_updates = 0, last_batches = 0;  // of the last persistent findMode
};

int64_t cox_group_rows(const std::vector<int32_t>& pid0, const std::vector<double>& time,
                       const std::vector<double>& y, const double* weights, std::vector<int32_t>& grp);

struct Fit {
    static constexpr int kGhParts = 1024;
    static constexpr int kBatchMax = 1024;  // columns per speculative gradient batch
    Context* ctx = nullptr;
    const Matrix* m = nullptr;
    int model = 0, precision = 0;
    int64_t K = 0;
    int32_t J = 0;
    bool offset_col0 = false;
    cudaStream_t stream = nullptr;
    // bounds on device-side waits (ccdb_fit_set_wait_limit): the grid sweep's level,
    // column and grid waits, and the mixed batch engine's cluster exchange
    static constexpr long long kDefaultWaitNs = 20LL * 1000 * 1000 * 1000;
    static constexpr long long kDefaultXchWaitNs = 2LL * 1000 * 1000 * 1000;
    long long wait_limit_ns = kDefaultWaitNs;
    long long xch_wait_ns = kDefaultXchWaitNs;

    // device state
    double2* row = nullptr;
    double* y = nullptr;
    double* beta = nullptr;
    double* hdelta = nullptr;
    double* xjy = nullptr;
    int32_t* ptype = nullptr;
    double* pvar = nullptr;
    DevStatus* st = nullptr;
    unsigned* grid_bar = nullptr;
    double2* red = nullptr;
    double* xb_tmp = nullptr;
    double* w = nullptr;
    double2* gh_parts = nullptr;
    double2* gh_out = nullptr;
    int64_t launches = 0;                        // engine kernels launched so far
    double last_call_seconds = 0.0;              // device time of the last fisher_information passes
    int last_iterations = 0;                     // getIterationCount: the last findMode's cycles
    int64_t nz_steps = 0;                        // nonzero coordinate steps of the current find_mode
    bool nz_known = true;                        // every path of the call counted them
    std::unique_ptr<DevSchedule> sched;
    CoxDev cox;

    // host mirror and lazy flags (CyclicCoordinateDescent.h:152-166)
    std::vector<double> y_h, w_h, beta_h, pvar_h, time_h;
    std::vector<int64_t> stratum_h;
    std::vector<int32_t> pid0_h;
    std::vector<int64_t> cox_grow_h;
    std::vector<int32_t> ptype_h;
    std::vector<uint8_t> fixed;
    bool weighted = false;
    bool valid_weights = false, xb_known = false, suff_known = false, touched_y = true;
    bool xb_pending = false, beta_dirty_host = false;
    double ll_fixed = 0.0;

    ~Fit();
    IndepParams params() const;
    void release_schedule();
    // kSchedGrid: the grid-wide persistent sweep (one CTA per SM, levels ordered
    // by global counters); kSchedCluster: one cluster, levels ordered by cluster
    // barriers
    static constexpr int kSchedGrid = 0, kSchedCluster = 1;
    void ensure_schedule(int kind);
    int sweep_kind(const ccdb_mode_args& a) const;
    void apply_weights();
    void compute_xbeta();
    void compute_xbeta_transpose();  // the MM cycle's product (ModelSpecifics::computeXBeta(beta))
    void remaining_statistics();
    void check_lazy();
    void upload_beta();
    void download_beta();
    void objective_terms(double* out4);
    double log_likelihood();
    double objective(int conv);
    void gradient_hessian(int j, double* g, double* h);
    void update_xbeta(int j, double delta);
    void find_mode_once(const ccdb_mode_args& a, double bound, int* flag, int* iters, double* obj,
                        float* ms);
    void find_mode(const ccdb_mode_args& a, double* beta_inout, ccdb_fit_result* res);
    // speculative batched sweeps (models without a fused sweep kernel)
    void find_mode_batched(const ccdb_mode_args& a, double bound, int* flag, int* iters, double* obj);
    // (g, h) of several columns against the current state; nonzero step of one column
    void gh_batch(const int32_t* cols, int n, double2* out);
    void apply_step(int j, double delta);
    bool use_speculative(const ccdb_mode_args& a) const;
    // the single-CTA sweep with the row state in shared memory (resident.cu)
    bool use_resident(const ccdb_mode_args& a);
    void find_mode_resident(const ccdb_mode_args& a, int* flag, int* iters, double* obj, float* ms);
    ResCol* d_res_recs = nullptr;  // its active columns' records in visiting order
    int32_t d_res_cap = 0;
    double2* d_res_rs = nullptr;   // the row state of the global form (K entries)
    int32_t* d_batch_cols = nullptr;  // independent-row models
    double2* d_batch_out = nullptr;
    bool is_cox() const { return model == M_COX; }
    bool is_grouped() const { return model == M_CLR || model == M_CPR; }
    // models served by the group engine (cox.cu) rather than the fused sweep
    bool group_engine() const { return is_cox() || is_grouped(); }
    // Cox engine (cox_host.cu)
    CoxParams cox_params() const;
    void cox_allocate();
    void cox_release();
    void cox_apply_weights();
    void cox_scans();
    void cox_remaining();
    void cox_objective_terms(double* out4);
    void cox_gh_batch(const int32_t* cols, int n, double2* out);
    void cox_update(int j, double delta);
    // one findMode of the group engine in one persistent launch (group_sweep.cu)
    void find_mode_group_sweep(const ccdb_mode_args& a, int* flag, int* iters, double* obj, float* ms);
    // mode-finding variants (modes_host.cu): the MM cycle, the KKT swindle, and
    // the MM all-coordinate (g, h) into out[J] (fixed may be nullptr)
    void find_mode_mm(const ccdb_mode_args& a, int* flag, int* iters, double* obj);
    void kkt_swindle(const ccdb_mode_args& a, double bound, int* flag, int* iters, double* obj, float* ms);
    void mm_gradient_hessian(const uint8_t* fixed_flags, double2* out);
    // post-fit calls (postfit_host.cu)
    void fisher_information(const int32_t* idx, int n, double* out);
    double predictive_log_likelihood(const double* weights);
    double predictive_sum(const double* weights);
    void predictive_estimates(double* out);
};

}  // namespace ccdb
