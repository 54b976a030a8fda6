// cox_host.cu -- host side of the Breslow Cox engine: risk-set grouping,
// per-group tables, and the per-coordinate calls on the device.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <vector>

#include "cox.h"
#include "engine.h"
#include "group_sweep.h"

namespace ccdb {

// setPidForAccumulation (ModelSpecifics.hpp:1809-1868) on rows sorted by
// (stratum, -time, y): group id per row (N for rows dropped by a zero weight)
// and the number of groups N.  Integer work, identical to the reference.
int64_t cox_group_rows(const std::vector<int32_t>& pid0, const std::vector<double>& time,
                       const std::vector<double>& y, const double* weights,
                       std::vector<int32_t>& grp) {
    const int64_t K = (int64_t)y.size();
    const int ignore = -1;
    grp.assign(K, 0);
    for (int64_t k = 0; k < K; ++k) grp[k] = pid0[k];
    int64_t index = 0;
    while (weights != nullptr && index < K && weights[index] == 0.0) {
        grp[index] = ignore;
        index++;
    }
    if (index >= K) {  // every row dropped
        for (int64_t k = 0; k < K; ++k) grp[k] = 0;
        return 0;
    }
    int lastPid = grp[index];
    double lastTime = time[index];
    double lastEvent = y[index];
    int pid = grp[index] = 0;
    for (int64_t k = index + 1; k < K; ++k) {
        if (weights == nullptr || weights[k] != 0.0) {
            const int nextPid = grp[k];
            if (nextPid != lastPid) {
                pid++;
                lastPid = nextPid;
            } else if (!(lastEvent == 1.0 && lastTime == time[k] && lastEvent == y[k])) {
                pid++;
            }
            lastTime = time[k];
            lastEvent = y[k];
            grp[k] = pid;
        } else {
            grp[k] = ignore;
        }
    }
    const int64_t N = (int64_t)pid + 1;
    for (int64_t k = 0; k < K; ++k)
        if (grp[k] == ignore) grp[k] = (int32_t)N;
    return N;
}

CoxParams Fit::cox_params() const {
    CoxParams P{};
    P.col_ptr = m->d_col_ptr;
    P.rows = m->d_rows;
    P.val_ptr = m->d_val_ptr;
    P.vals = m->d_vals;
    P.fmt = m->d_fmt;
    P.K = K;
    P.N = cox.N;
    P.xbe = cox.xbe;
    P.w = w;
    P.y = y;
    P.grp = cox.grp;
    P.rstrat = cox.rstrat;
    P.weighted = weighted ? 1 : 0;
    P.mixed = (is_cox() && precision == CCDB_PRECISION_MIXED) ? 1 : 0;
    P.denom = cox.denom;
    P.D = cox.D;
    P.S1 = cox.S1;
    P.S2 = cox.S2;
    P.nEv = cox.nEv;
    P.gfirst = cox.gfirst;
    P.glast = cox.glast;
    P.grow = cox.grow;
    P.xjy = xjy;
    P.st = st;
    P.wait_limit_ns = wait_limit_ns;
    return P;
}

void Fit::cox_allocate() {
    // stratum index of each row, as ModelData::loadY numbers them (ModelData.cpp:96-125)
    std::vector<int32_t> rs(K);
    int32_t p = 0;
    for (int64_t k = 0; k < K; ++k) {
        if (k > 0 && stratum_h[k] != stratum_h[k - 1]) p++;
        rs[k] = p;
    }
    pid0_h = rs;
    const int64_t n_strata = K > 0 ? (int64_t)p + 1 : 0;
    // Cox: the most groups any weighting can produce; grouped models: the strata; + slot N
    const size_t G = is_cox() ? (size_t)K + 1 : (size_t)n_strata + 1;
    cox.xbe = static_cast<double2*>(ctx->alloc(sizeof(double2) * K));
    cox.grp = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * K));
    cox.rstrat = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * K));
    cox.denom = static_cast<double*>(ctx->alloc(sizeof(double) * G));
    cox.D = static_cast<double*>(ctx->alloc(sizeof(double) * G));
    cox.S1 = static_cast<double*>(ctx->alloc(sizeof(double) * G));
    cox.S2 = static_cast<double*>(ctx->alloc(sizeof(double) * G));
    cox.nEv = static_cast<double*>(ctx->alloc(sizeof(double) * G));
    cox.gfirst = static_cast<uint8_t*>(ctx->alloc(G));
    cox.glast = static_cast<uint8_t*>(ctx->alloc(G));
    cox.grow = static_cast<int64_t*>(ctx->alloc(sizeof(int64_t) * (G + 1)));
    const int tiles = cox_scan_tiles((int64_t)G);
    cox.tickets = static_cast<unsigned*>(ctx->alloc(2 * sizeof(unsigned)));
    cox.status = static_cast<int*>(ctx->alloc(sizeof(int) * 2 * std::max(1, tiles)));
    cox.tails = ctx->alloc(cox_tail_bytes() * 2 * std::max(1, tiles));
    cox.batch_cols = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * kBatchMax));
    cox.batch_out = static_cast<double2*>(ctx->alloc(sizeof(double2) * kBatchMax));
    check_cuda(cudaMemsetAsync(cox.status, 0, sizeof(int) * 2 * std::max(1, tiles), stream), "status");
    check_cuda(cudaMemsetAsync(cox.S1, 0, sizeof(double) * G, stream), "S1");
    check_cuda(cudaMemsetAsync(cox.S2, 0, sizeof(double) * G, stream), "S2");
    check_cuda(cudaMemsetAsync(cox.xbe, 0, sizeof(double2) * K, stream), "xbe");
    check_cuda(cudaMemcpyAsync(cox.rstrat, rs.data(), sizeof(int32_t) * K, cudaMemcpyHostToDevice, stream),
               "rstrat");
    if (is_grouped()) {  // the group of a row is its stratum (GroupedData::getGroup)
        cox.N = n_strata;
        std::vector<int64_t> grow(n_strata + 1, K);
        for (int64_t k = K - 1; k >= 0; --k) grow[rs[k]] = k;
        grow[n_strata] = K;
        check_cuda(cudaMemcpyAsync(cox.grp, rs.data(), sizeof(int32_t) * K, cudaMemcpyHostToDevice, stream),
                   "grp");
        check_cuda(cudaMemcpyAsync(cox.grow, grow.data(), sizeof(int64_t) * (n_strata + 1),
                                   cudaMemcpyHostToDevice, stream), "grow");
        cox_grow_h = grow;
    }
    check_cuda(ctx->wait(), "cox alloc");
}

void Fit::cox_release() {
    for (void* p : {(void*)cox.xbe, (void*)cox.grp, (void*)cox.rstrat, (void*)cox.denom, (void*)cox.D,
                    (void*)cox.S1, (void*)cox.S2, (void*)cox.nEv, (void*)cox.gfirst, (void*)cox.glast,
                    (void*)cox.grow, (void*)cox.tickets, (void*)cox.status, cox.tails,
                    (void*)cox.batch_cols, (void*)cox.batch_out, (void*)cox.sweep_cols, (void*)cox.dd,
                    (void*)cox.ddg, cox.agg, (void*)cox.counters, (void*)cox.sweep_gh})
        ctx->release(p);
}

// setWeights for the Cox model (ModelSpecifics.hpp:427-484): regroup with the
// weights, N-weights = events (observationCount = y) times weight per group,
// then computeXjY (x * y * w; survival models use observationCount(y) = y).
void Fit::cox_apply_weights() {
    std::vector<double> wh(K, 1.0);
    if (weighted) wh = w_h;
    if (is_grouped()) {
        // setWeights (ModelSpecifics.hpp:427-484): nEv per stratum = y * w
        // (observationCount = y); computeXjY: x * y * w; fixed terms for CPR.
        const int64_t N = cox.N;
        std::vector<double> nev(N + 1, 0.0);
        for (int64_t k = 0; k < K; ++k) nev[pid0_h[k]] += y_h[k] * wh[k];
        check_cuda(cudaMemcpyAsync(w, wh.data(), sizeof(double) * K, cudaMemcpyHostToDevice, stream), "w");
        check_cuda(cudaMemcpyAsync(cox.nEv, nev.data(), sizeof(double) * (N + 1), cudaMemcpyHostToDevice,
                                   stream), "nev");
        check_cuda(launch_xjy(m->d_col_ptr, m->d_rows, m->d_val_ptr, m->d_vals, m->d_fmt, y,
                              weighted ? w : nullptr, K, J, xjy, stream), "xjy");
        ++launches;
        ll_fixed = 0.0;
        if (model == M_CPR) {  // ConditionalPoissonRegression::logLikeFixedTermsContrib (ModelSpecifics.h:722-727)
            for (int64_t i = 0; i < K; ++i) {
                double t = 0.0;
                for (int c = 2; c <= (int)y_h[i]; c++) t -= std::log((double)c);
                ll_fixed += weighted ? t * wh[i] : t;
            }
        }
        check_cuda(ctx->wait(), "grouped weights");
        valid_weights = true;
        suff_known = false;
        return;
    }
    std::vector<int32_t> grp;
    const int64_t N = cox_group_rows(pid0_h, time_h, y_h, weighted ? w_h.data() : nullptr, grp);
    cox.N = N;
    std::vector<double> nev(N + 1, 0.0);
    for (int64_t k = 0; k < K; ++k) nev[grp[k]] += y_h[k] * wh[k];
    std::vector<uint8_t> gf(N + 1, 0), gl(N + 1, 0);
    std::vector<int64_t> grow(N + 2, K);
    std::vector<int32_t> gstrat(N + 1, -1);
    for (int64_t k = K - 1; k >= 0; --k)
        if (grp[k] < N) {
            grow[grp[k]] = k;
            gstrat[grp[k]] = pid0_h[k];
        }
    for (int64_t g = N - 1; g >= 0; --g)
        if (grow[g] == K) grow[g] = grow[g + 1];
    for (int64_t g = 0; g < N; ++g) {
        gf[g] = (g == 0 || gstrat[g] != gstrat[g - 1]) ? 1 : 0;
        gl[g] = (g == N - 1 || gstrat[g] != gstrat[g + 1]) ? 1 : 0;
    }
    grow[N] = K;
    check_cuda(cudaMemcpyAsync(w, wh.data(), sizeof(double) * K, cudaMemcpyHostToDevice, stream), "w");
    check_cuda(cudaMemcpyAsync(cox.grp, grp.data(), sizeof(int32_t) * K, cudaMemcpyHostToDevice, stream), "grp");
    check_cuda(cudaMemcpyAsync(cox.nEv, nev.data(), sizeof(double) * (N + 1), cudaMemcpyHostToDevice, stream), "nev");
    check_cuda(cudaMemcpyAsync(cox.gfirst, gf.data(), N + 1, cudaMemcpyHostToDevice, stream), "gfirst");
    check_cuda(cudaMemcpyAsync(cox.glast, gl.data(), N + 1, cudaMemcpyHostToDevice, stream), "glast");
    check_cuda(cudaMemcpyAsync(cox.grow, grow.data(), sizeof(int64_t) * (N + 1), cudaMemcpyHostToDevice, stream),
               "grow");
    check_cuda(cudaMemsetAsync(cox.S1 + N, 0, sizeof(double), stream), "S1N");
    check_cuda(cudaMemsetAsync(cox.S2 + N, 0, sizeof(double), stream), "S2N");
    // slot N gathers the rows a zero weight drops; like the reference's denomPid[N]
    // it holds 0, which the MM bound reads (0 * e / 0 for such a row, as there)
    check_cuda(cudaMemsetAsync(cox.denom + N, 0, sizeof(double), stream), "denomN");
    check_cuda(cudaMemsetAsync(cox.D + N, 0, sizeof(double), stream), "DN");
    check_cuda(launch_xjy(m->d_col_ptr, m->d_rows, m->d_val_ptr, m->d_vals, m->d_fmt, y,
                          weighted ? w : nullptr, K, J, xjy, stream),
               "xjy");
    ++launches;
    ll_fixed = 0.0;
    check_cuda(ctx->wait(), "cox weights");
    valid_weights = true;
    suff_known = false;
}

void Fit::cox_scans() {
    if (!is_cox()) return;
    ++cox.epoch;
    CoxParams P = cox_params();
    check_cuda(launch_cox_scans(P, cox.tickets, cox.status, cox.tails, cox.epoch, stream), "cox scans");
    launches += 2;
}

// computeRemainingStatistics (ModelSpecifics.hpp:1588-1617) + the accumulated scans.
void Fit::cox_remaining() {
    if (xb_pending) {  // xBeta computed into xb_tmp: place it into {xBeta, e}
        check_cuda(cudaMemcpy2DAsync(cox.xbe, sizeof(double2), xb_tmp, sizeof(double), sizeof(double), K,
                                     cudaMemcpyDeviceToDevice, stream),
                   "xb place");
        xb_pending = false;
    }
    CoxParams P = cox_params();
    if (is_cox()) check_cuda(launch_cox_remaining(P, stream), "cox remaining");
    else check_cuda(launch_grouped_remaining(P, stream), "grouped remaining");
    launches += 2;
    cox_scans();
    suff_known = true;
}

void Fit::cox_objective_terms(double* out4) {
    const int nb = ctx->n_sm;
    CoxParams P = cox_params();
    if (is_cox()) check_cuda(launch_cox_objective(P, red, nb, stream), "cox objective");
    else check_cuda(launch_grouped_objective(P, red, nb, stream), "grouped objective");
    ++launches;
    std::vector<double2> parts(2 * nb);
    check_cuda(cudaMemcpyAsync(parts.data(), red, sizeof(double2) * 2 * nb, cudaMemcpyDeviceToHost, stream),
               "objective copy");
    check_cuda(ctx->wait(), "objective sync");
    double t[4] = {0, 0, 0, 0};
    for (int c = 0; c < nb; ++c) {
        t[0] += parts[2 * c].x;
        t[1] += parts[2 * c].y;
        t[2] += parts[2 * c + 1].x;
    }
    // log prior on the host (JointPrior.h:121-128)
    for (int j = 0; j < J; ++j) t[3] += log_prior_host(beta_h[j], ptype_h[j], pvar_h[j]);
    for (int i = 0; i < 4; ++i) out4[i] = t[i];
}

void Fit::cox_gh_batch(const int32_t* cols, int n, double2* out) {
    check_cuda(cudaMemcpyAsync(cox.batch_cols, cols, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream),
               "batch cols");
    CoxParams P = cox_params();
    if (is_cox()) check_cuda(launch_cox_gh(P, cox.batch_cols, n, cox.batch_out, stream), "cox gh");
    else check_cuda(launch_grouped_gh(P, cox.batch_cols, n, cox.batch_out, stream), "grouped gh");
    ++launches;
    check_cuda(cudaMemcpyAsync(out, cox.batch_out, sizeof(double2) * n, cudaMemcpyDeviceToHost, stream),
               "gh copy");
    check_cuda(ctx->wait(), "gh sync");
}

void Fit::cox_update(int j, double delta) {
    CoxParams P = cox_params();
    if (is_cox()) check_cuda(launch_cox_update(P, j, delta, stream), "cox update");
    else check_cuda(launch_grouped_update(P, j, delta, stream), "grouped update");
    ++launches;
    cox_scans();
}

// findMode (CyclicCoordinateDescent.cpp:909-1216) of the Cox and grouped
// models as one cooperative launch: speculative gradient batches, the nonzero
// steps, the denominator updates, the Cox scans and the convergence test all on
// the device (group_sweep.cu).  The bounds are set by the caller.
void Fit::find_mode_group_sweep(const ccdb_mode_args& a, int* flag, int* iters, double* obj, float* ms) {
    std::vector<int32_t> cols;
    int64_t max_entries = 1;
    for (int j = 0; j < J; ++j)
        if (!fixed[j]) {
            cols.push_back(j);
            max_entries = std::max<int64_t>(max_entries, m->entries(j));
        }
    if (cols.empty()) {  // an empty cycle: the first check sees conv = 0
        *obj = objective(a.convergence_type);
        *flag = (*obj != *obj) ? R_ILLCONDITIONED
                : (a.tolerance > 0 ? R_SUCCESS : (a.max_iterations == 1 ? R_MAX_ITERATIONS : R_SUCCESS));
        *iters = 1;
        *ms = 0.f;
        return;
    }
    int bps = 0;
    check_cuda(group_sweep_occupancy(&bps), "occupancy");
    if (bps < 1) throw Error(CCDB_ERR_CUDA, "the group sweep kernel does not fit on an SM");
    int n_cta = ctx->n_sm;
    if (ctx->max_ctas > 0) n_cta = std::min(n_cta, ctx->max_ctas);
    // the cluster form (hardware barriers) when the fit is small enough for a few
    // SMs or the context's share is a cluster's worth; CCDB_SWEEP_GRID_LEVELS asks
    // for the grid form, CCDB_SWEEP_LEVELS for the cluster form
    if (ctx->group_cluster < 0) {
        int c = 0;
        check_cuda(group_sweep_max_cluster(&c), "cluster occupancy");
        ctx->group_cluster = c;
    }
    bool use_cluster = false;
    if (ctx->group_cluster >= 2 && a.strategy != CCDB_SWEEP_GRID_LEVELS) {
        const int64_t work = cox.N + max_entries;
        use_cluster = a.strategy == CCDB_SWEEP_LEVELS || n_cta <= ctx->group_cluster + ctx->group_cluster / 4 ||
                      work <= (int64_t)ctx->group_cluster * kGroupClusterWork;
        if (use_cluster) {
            int c = ctx->group_cluster;
            while (c > 1 && c > n_cta) c /= 2;
            n_cta = c;
        }
    }
    if (!cox.sweep_cols) {
        cox.sweep_cols = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * std::max(1, J)));
        cox.agg = ctx->alloc(sizeof(SegAgg) * 2 * ctx->n_sm);
        cox.counters = static_cast<int64_t*>(ctx->alloc(sizeof(int64_t) * 2));
    }
    if (cox.dd_cap < max_entries) {
        ctx->release(cox.dd);
        ctx->release(cox.ddg);
        cox.dd = static_cast<double*>(ctx->alloc(sizeof(double) * max_entries));
        cox.ddg = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * max_entries));
        cox.dd_cap = max_entries;
    }
    check_cuda(cudaMemcpyAsync(cox.sweep_cols, cols.data(), sizeof(int32_t) * cols.size(), cudaMemcpyHostToDevice,
                               stream), "columns");
    if (!cox.sweep_gh) cox.sweep_gh = static_cast<double2*>(ctx->alloc(sizeof(double2) * 2 * kGroupBatchMax));
    if (!beta_dirty_host) upload_beta();
    DevStatus zero{};
    zero.flag = R_FAIL;
    check_cuda(cudaMemcpyAsync(st, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream), "status");
    check_cuda(cudaMemsetAsync(grid_bar, 0, sizeof(unsigned), stream), "barrier");
    check_cuda(cudaMemsetAsync(cox.counters, 0, sizeof(int64_t) * 2, stream), "counters");
    GroupSweepParams Q{};
    Q.P = cox_params();
    Q.cox = is_cox() ? 1 : 0;
    Q.n_active = (int32_t)cols.size();
    Q.cols = cox.sweep_cols;
    Q.beta = beta;
    Q.hdelta = hdelta;
    Q.ptype = ptype;
    Q.pvar = pvar;
    Q.conv = a.convergence_type;
    Q.max_iter = a.max_iterations;
    Q.tol = a.tolerance;
    Q.ll_fixed = ll_fixed;
    Q.batch_max = std::min(kBatchMax, kGroupBatchMax);
    Q.J = J;
    Q.gh = cox.sweep_gh;
    Q.dd = cox.dd;
    Q.ddg = cox.ddg;
    Q.red = red;
    Q.agg = static_cast<SegAgg*>(cox.agg);
    Q.grid_bar = grid_bar;
    Q.st = st;
    Q.wait_limit_ns = wait_limit_ns;
    Q.counters = cox.counters;
    // CCDB_TRACE_FILE=<path>: timestamps of the first 4,096 nonzero steps (profiling aid; off by default)
    const char* trace_path = std::getenv("CCDB_TRACE_FILE");
    unsigned long long* d_trace = nullptr;
    const int trace_steps = 4096;
    if (trace_path) {
        d_trace = static_cast<unsigned long long*>(ctx->alloc(sizeof(unsigned long long) * kTraceStamps * trace_steps));
        check_cuda(cudaMemsetAsync(d_trace, 0, sizeof(unsigned long long) * kTraceStamps * trace_steps, stream), "trace");
        Q.trace = d_trace;
        Q.trace_steps = trace_steps;
    }
    check_cuda(cudaEventRecord(ctx->fev[0], stream), "event");
    check_cuda(launch_group_sweep(Q, n_cta, use_cluster, stream), "group sweep launch");
    ++launches;
    check_cuda(cudaEventRecord(ctx->fev[1], stream), "event");
    check_cuda(ctx->wait(), "group sweep");  // the sweep is done before a copy is queued behind it
    DevStatus out{};
    int64_t cnt[2] = {0, 0};
    check_cuda(cudaMemcpyAsync(&out, st, sizeof(out), cudaMemcpyDeviceToHost, stream), "status");
    check_cuda(cudaMemcpyAsync(cnt, cox.counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream), "counters");
    check_cuda(ctx->wait(), "group sweep");
    check_cuda(cudaEventElapsedTime(ms, ctx->fev[0], ctx->fev[1]), "elapsed");
    if (d_trace) {
        std::vector<unsigned long long> tr(kTraceStamps * (size_t)trace_steps);
        check_cuda(cudaMemcpy(tr.data(), d_trace, sizeof(unsigned long long) * tr.size(), cudaMemcpyDeviceToHost),
                   "trace copy");
        ctx->release(d_trace);
        if (FILE* fh = std::fopen(trace_path, "wb")) {
            std::fwrite(tr.data(), sizeof(unsigned long long), tr.size(), fh);
            std::fclose(fh);
        }
    }
    if (out.error != E_NONE)
        throw Error(CCDB_ERR_TIMEOUT, "device wait timed out (code " + std::to_string(out.error) + " at " +
                                          std::to_string(out.error_where) + ")");
    cox.last_updates = cnt[0];
    cox.last_batches = cnt[1];
    nz_steps += cnt[0];
    *flag = out.flag;
    *iters = out.iterations;
    *obj = out.objective;
    beta_dirty_host = true;
}

}  // namespace ccdb
