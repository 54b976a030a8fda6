// api.cu -- the C ABI of libccdb.so (include/ccdb.h) and the host runtime
// behind it: device memory under a per-context HBM budget, matrix upload,
// per-fit lazy state (the flags of CyclicCoordinateDescent::checkAllLazyFlags,
// CyclicCoordinateDescent.cpp:388-406), schedule caching, and the mode-finding
// driver (CyclicCoordinateDescent::update, .cpp:586-615).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ccdb.h"
#include "batch.h"
#include "csr_device.h"
#include "csr_host.h"
#include "engine.h"
#include "resident.h"

namespace ccdb {

thread_local std::string g_last_error;

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(CCDB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void* Context::alloc(size_t bytes) {
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) / 256 * 256;
    {
        std::lock_guard<std::mutex> g(mu);
        if (budget && in_use + bytes > budget)
            throw Error(CCDB_ERR_BUDGET, "device allocation of " + std::to_string(bytes) +
                                             " bytes exceeds the HBM budget");
        in_use += bytes;
    }
    // stream-ordered from the context's own pool: allocation and release are
    // ordered with the context's own work and never wait on another context's
    // stream (the device's shared pool may reuse a block another stream freed by
    // making this stream wait for that one), so fits of other contexts keep
    // running through them
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, stream);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> g(mu);
        in_use -= bytes;
        check_cuda(e, "cudaMallocFromPoolAsync");
    }
    std::lock_guard<std::mutex> g(mu);
    sizes[p] = bytes;
    return p;
}

void Context::release(void* p) {
    if (!p) return;
    cudaFreeAsync(p, stream);
    std::lock_guard<std::mutex> g(mu);
    auto it = sizes.find(p);
    if (it != sizes.end()) {
        in_use -= it->second;
        sizes.erase(it);
    }
}

cudaError_t Context::wait() {
    if (!blocking_wait) return cudaStreamSynchronize(stream);
    cudaError_t e = cudaEventRecord(ev_wait, stream);
    return e == cudaSuccess ? cudaEventSynchronize(ev_wait) : e;
}

template <typename T>
T* upload(Context* c, const T* h, size_t n, cudaStream_t s) {
    T* d = static_cast<T*>(c->alloc(sizeof(T) * (n ? n : 1)));
    if (n && h) check_cuda(cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s), "upload");
    return d;
}

int64_t Matrix::entries(int j) const {
    if (fmt[j] == F_DENSE || fmt[j] == F_INTERCEPT) return K;
    return col_start[j + 1] - col_start[j];
}

Matrix::~Matrix() {
    for (void* p : {(void*)d_col_ptr, (void*)d_rows, (void*)d_val_ptr, (void*)d_vals, (void*)d_fmt,
                    (void*)d_row_ptr, (void*)d_csr_col, (void*)d_csr_val})
        ctx->release(p);
}

// Row-major copy for computeXBeta: per row, entries in increasing column order
// (dense-like columns included), built once, on the device from the uploaded
// columns (csr_device.cu); a matrix with a row longer than kCsrDeviceMaxRow
// entries is built on the host threads instead (csr_host.cpp, the same layout).
void Matrix::ensure_csr(cudaStream_t s) {
    if (d_row_ptr) return;
    int64_t total = 0;
    for (int j = 0; j < J; ++j) total += entries(j);
    CsrDeviceArgs a{K, J, d_col_ptr, d_rows, d_val_ptr, d_vals, d_fmt};
    auto* counts = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(K, 1)));
    auto* cursor = static_cast<int64_t*>(ctx->alloc(sizeof(int64_t) * (size_t)std::max<int64_t>(K, 1)));
    auto* d_max = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t)));
    d_row_ptr = static_cast<int64_t*>(ctx->alloc(sizeof(int64_t) * (size_t)(K + 1)));
    int32_t longest = 0;
    check_cuda(csr_device_count(a, counts, d_row_ptr, cursor, d_max, s), "row counts");
    check_cuda(cudaMemcpyAsync(&longest, d_max, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "longest row");
    check_cuda(ctx->wait(), "row counts");
    if (longest <= kCsrDeviceMaxRow) {
        d_csr_col = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(total, 1)));
        d_csr_val = static_cast<double*>(ctx->alloc(sizeof(double) * (size_t)std::max<int64_t>(total, 1)));
        check_cuda(csr_device_fill(a, d_row_ptr, cursor, d_csr_col, d_csr_val, s), "row-major fill");
    } else {
        ctx->release(d_row_ptr);
        const HostCsr h = build_csr(K, J, col_start.data(), rows_h.data(), val_start.data(), vals_h.data(),
                                    fmt.data(), (int)std::max(1u, std::thread::hardware_concurrency()));
        d_row_ptr = upload(ctx, h.row_ptr.data(), h.row_ptr.size(), s);
        d_csr_col = upload(ctx, h.col.data(), h.col.size(), s);
        d_csr_val = upload(ctx, h.val.data(), h.val.size(), s);
    }
    ctx->release(counts);
    ctx->release(cursor);
    ctx->release(d_max);
    check_cuda(ctx->wait(), "row-major copy");
}

// ------------------------------------------------------------------ Fit

Fit::~Fit() {
    for (void* p : {(void*)row, (void*)y, (void*)beta, (void*)hdelta, (void*)xjy, (void*)ptype,
                    (void*)pvar, (void*)st, (void*)grid_bar, (void*)red, (void*)xb_tmp, (void*)w,
                    (void*)gh_parts, (void*)gh_out, (void*)d_batch_cols, (void*)d_batch_out,
                    (void*)d_res_recs, (void*)d_res_rs})
        ctx->release(p);
    release_schedule();
    if (group_engine()) cox_release();
}

void Fit::release_schedule() {
    if (!sched) return;
    for (void* p : {(void*)sched->segs, (void*)sched->cta_seg, (void*)sched->tasks,
                    (void*)sched->level_need, (void*)sched->level_done, (void*)sched->col_arrive,
                    (void*)sched->partials, (void*)sched->level_split})
        ctx->release(p);
    sched.reset();
}

IndepParams Fit::params() const {
    IndepParams P{};
    P.col_ptr = m->d_col_ptr;
    P.rows = m->d_rows;
    P.val_ptr = m->d_val_ptr;
    P.vals = m->d_vals;
    P.fmt = m->d_fmt;
    P.K = K;
    P.J = J;
    P.model = model;
    P.row = row;
    P.y = y;
    P.beta = beta;
    P.hdelta = hdelta;
    P.xjy = xjy;
    P.ptype = ptype;
    P.pvar = pvar;
    P.red = red;
    P.grid_bar = grid_bar;
    P.st = st;
    P.ll_fixed = ll_fixed;
    P.wait_limit_ns = wait_limit_ns;
    if (sched) {
        P.segs = sched->segs;
        P.cta_seg = sched->cta_seg;
        P.tasks = sched->tasks;
        P.n_levels = sched->host.n_levels;
        P.level_done = sched->level_done;
        P.level_need = sched->level_need;
        P.col_arrive = sched->col_arrive;
        P.partials = sched->partials;
        P.level_split = sched->level_split;
    }
    return P;
}

// ModelSpecifics::setWeights + computeFixedTermsInLogLikelihood + computeXjY
// (ModelSpecifics.hpp:427-484, 570-587, 486-524).  Independent rows: the
// N-weights equal the row weights (observationCount = 1).
void Fit::apply_weights() {
    if (group_engine()) {
        cox_apply_weights();
        return;
    }
    std::vector<double> wh(K, 1.0);
    if (weighted) wh = w_h;
    check_cuda(cudaMemcpyAsync(w, wh.data(), sizeof(double) * K, cudaMemcpyHostToDevice, stream),
               "weights");
    check_cuda(launch_xjy(m->d_col_ptr, m->d_rows, m->d_val_ptr, m->d_vals, m->d_fmt, y,
                          weighted ? w : nullptr, K, J, xjy, stream),
               "xjy");
    ++launches;
    ll_fixed = 0.0;
    if (model == M_POISSON) {
        // PoissonRegression::logLikeFixedTermsContrib (ModelSpecifics.h:1596-1601) sums
        // -log(c) for c = 2..y in order; the running table reproduces each sum exactly.
        std::vector<double> table(1, 0.0);
        for (int64_t i = 0; i < K; ++i) {
            const int yi = (int)y_h[i];
            while ((int)table.size() <= yi) {
                const int c = (int)table.size();
                table.push_back(c >= 2 ? table.back() + -std::log((double)c) : 0.0);
            }
            const double t = yi >= 2 ? table[yi] : 0.0;
            ll_fixed += weighted ? t * wh[i] : t;
        }
    }
    check_cuda(ctx->wait(), "weights sync");
    valid_weights = true;
    suff_known = false;
}

// CyclicCoordinateDescent::computeXBeta (.cpp:1452-1470).
void Fit::compute_xbeta() {
    int nonzero = 0, only = -1;
    for (int j = 0; j < J; ++j)
        if (beta_h[j] != 0.0) {
            ++nonzero;
            only = j;
        }
    if (nonzero == 0) {
        check_cuda(cudaMemsetAsync(xb_tmp, 0, sizeof(double) * K, stream), "xb zero");
    } else if (nonzero == 1 && (m->fmt[only] == F_DENSE || m->fmt[only] == F_INTERCEPT)) {
        // one dense-like column (the offset of a cold start): xBeta = 0 + b*x
        const double* v = (m->fmt[only] == F_DENSE) ? m->d_vals + m->val_start[only] : nullptr;
        check_cuda(launch_xbeta_dense(v, beta_h[only], K, xb_tmp, stream), "xbeta");
        ++launches;
    } else {
        const_cast<Matrix*>(m)->ensure_csr(stream);
        check_cuda(launch_xbeta_csr(m->d_row_ptr, m->d_csr_col, m->d_csr_val, beta, K, xb_tmp, stream),
                   "xbeta");
        ++launches;
    }
    xb_pending = true;
    xb_known = true;
    suff_known = false;
}

// computeRemainingStatistics (ModelSpecifics.hpp:1588-1633).
void Fit::remaining_statistics() {
    if (group_engine()) {
        cox_remaining();
        return;
    }
    const double null_denom = (model == M_LOGISTIC) ? 1.0 : 0.0;
    check_cuda(launch_remaining_stats(row, xb_pending ? xb_tmp : nullptr, w, K, null_denom, stream),
               "remaining statistics");
    ++launches;
    xb_pending = false;
    suff_known = true;
}

void Fit::check_lazy() {
    if (!xb_known) compute_xbeta();
    if (!valid_weights) apply_weights();
    if (!suff_known) remaining_statistics();
}

void Fit::upload_beta() {
    check_cuda(cudaMemcpyAsync(beta, beta_h.data(), sizeof(double) * J, cudaMemcpyHostToDevice, stream),
               "beta upload");
}

void Fit::download_beta() {
    check_cuda(cudaMemcpyAsync(beta_h.data(), beta, sizeof(double) * J, cudaMemcpyDeviceToHost, stream),
               "beta download");
    check_cuda(ctx->wait(), "beta sync");
}

int Fit::sweep_kind(const ccdb_mode_args& a) const {
    return a.strategy == CCDB_SWEEP_GRID_LEVELS ? kSchedGrid : kSchedCluster;
}

void Fit::ensure_schedule(int kind) {
    int C = 0;  // the cluster sweep's size: the largest resident, within the context's CTA share
    if (kind == kSchedCluster) {
        if (ctx->sweep_cluster < 0) {
            int c = 0;
            check_cuda(cluster_sweep_max_size(model, &c), "cluster occupancy");
            ctx->sweep_cluster = c;
        }
        C = ctx->sweep_cluster;
        if (C < 1) throw Error(CCDB_ERR_CUDA, "the cluster sweep kernel cannot be resident");
        while (ctx->max_ctas > 0 && C > ctx->max_ctas && C > 1) C /= 2;
    }
    if (sched && sched->fixed == fixed && sched->kind == kind && (kind != kSchedCluster || sched->cluster == C))
        return;
    release_schedule();
    if (kind == kSchedCluster) {
        ScheduleParams sp;
        sp.n_cta = C;
        sp.warps_per_cta = indep_threads() / 32;
        sp.warp_max = 128;   // warp tasks stage 4 entries per lane
        sp.cta_max = 4096;   // CTA tasks and chunks stage 8 entries per thread
        sp.chunk = 1024;     // split columns: chunks of ~1024 entries spread a long column over more CTAs
        std::vector<int64_t> entries(J);
        for (int j = 0; j < J; ++j) entries[j] = m->entries(j);
        auto s = std::make_unique<DevSchedule>();
        s->fixed = fixed;
        s->kind = kind;
        s->cluster = C;
        s->host = build_schedule(K, J, m->col_start.data(), m->rows_h.data(), m->fmt.data(),
                                 fixed.data(), nullptr, K, entries.data(), sp);
        if (s->host.max_split_per_seg > indep_max_split() || s->host.max_split_per_level > indep_max_split())
            throw Error(CCDB_ERR_UNSUPPORTED, "too many split columns on one level");
        s->segs = upload(ctx, s->host.segs.data(), s->host.segs.size(), stream);
        s->cta_seg = upload(ctx, s->host.cta_seg.data(), s->host.cta_seg.size(), stream);
        s->tasks = upload(ctx, s->host.tasks.data(), s->host.tasks.size(), stream);
        s->level_split = upload(ctx, s->host.level_split.data(), s->host.level_split.size(), stream);
        check_cuda(ctx->wait(), "schedule upload");
        sched = std::move(s);
        return;
    }
    int bps = 0;
    check_cuda(indep_sweep_occupancy(model, &bps), "occupancy");
    if (bps < 1) throw Error(CCDB_ERR_CUDA, "sweep kernel does not fit on an SM");
    ScheduleParams sp;
    sp.n_cta = ctx->n_sm * std::min(bps, 1);
    if (ctx->max_ctas > 0) sp.n_cta = std::min(sp.n_cta, ctx->max_ctas);
    // columns up to cta_max entries run on one CTA; longer ones split over CTAs
    sp.warps_per_cta = indep_threads() / 32;
    std::vector<int64_t> entries(J);
    for (int j = 0; j < J; ++j) entries[j] = m->entries(j);
    auto s = std::make_unique<DevSchedule>();
    s->fixed = fixed;
    s->kind = kind;
    s->host = build_schedule(K, J, m->col_start.data(), m->rows_h.data(), m->fmt.data(),
                             fixed.data(), nullptr, K, entries.data(), sp);
    if (s->host.max_split_per_seg > indep_max_split())
        throw Error(CCDB_ERR_UNSUPPORTED, "too many split columns on one level");
    s->segs = upload(ctx, s->host.segs.data(), s->host.segs.size(), stream);
    s->cta_seg = upload(ctx, s->host.cta_seg.data(), s->host.cta_seg.size(), stream);
    s->tasks = upload(ctx, s->host.tasks.data(), s->host.tasks.size(), stream);
    s->level_need = upload(ctx, s->host.level_need.data(), s->host.level_need.size(), stream);
    s->level_done = static_cast<unsigned*>(ctx->alloc(sizeof(unsigned) * std::max(1, s->host.n_levels)));
    s->col_arrive = static_cast<unsigned*>(ctx->alloc(sizeof(unsigned) * std::max(1, J)));
    s->partials = static_cast<double2*>(ctx->alloc(sizeof(double2) * std::max(1, s->host.n_partials)));
    check_cuda(ctx->wait(), "schedule upload");
    sched = std::move(s);
}

// Objective terms {LL num, LL den, gradient objective, log prior} of the
// current state, reduced in a fixed order.
void Fit::objective_terms(double* out4) {
    check_lazy();
    if (group_engine()) {
        cox_objective_terms(out4);
        return;
    }
    const int nb = ctx->n_sm;
    IndepParams P = params();
    check_cuda(launch_indep_objective(P, nb, stream), "objective");
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
        t[3] += parts[2 * c + 1].y;
    }
    for (int i = 0; i < 4; ++i) out4[i] = t[i];
}

double Fit::log_likelihood() {
    double t[4];
    objective_terms(t);
    return (t[0] - t[1]) + ll_fixed;
}

double Fit::objective(int conv) {
    double t[4];
    objective_terms(t);
    const double ll = (t[0] - t[1]) + ll_fixed;
    if (conv == C_GRADIENT) return t[2];
    if (conv == C_MITTAL) return ll;
    return ll + t[3];
}

void Fit::gradient_hessian(int j, double* g, double* h) {
    check_lazy();
    if (group_engine()) {
        const int32_t col = j;
        double2 r;
        cox_gh_batch(&col, 1, &r);
        *g = r.x;
        *h = r.y;
        return;
    }
    IndepParams P = params();
    check_cuda(launch_indep_gh(P, j, m->entries(j), gh_parts, kGhParts, gh_out, stream), "gh");
    launches += 2;
    double2 r;
    check_cuda(cudaMemcpyAsync(&r, gh_out, sizeof(double2), cudaMemcpyDeviceToHost, stream), "gh copy");
    check_cuda(ctx->wait(), "gh sync");
    *g = r.x;
    *h = r.y;
}

void Fit::update_xbeta(int j, double delta) {
    check_lazy();
    beta_h[j] += delta;
    check_cuda(cudaMemcpyAsync(beta + j, &beta_h[j], sizeof(double), cudaMemcpyHostToDevice, stream),
               "beta j");
    if (group_engine()) {
        cox_update(j, delta);
        check_cuda(ctx->wait(), "update sync");
        return;
    }
    IndepParams P = params();
    check_cuda(launch_indep_update(P, j, m->fmt[j], m->entries(j), delta, stream), "update");
    launches += m->entries(j) > 0 ? 1 : 0;
    check_cuda(ctx->wait(), "update sync");
}

// findMode (CyclicCoordinateDescent.cpp:909-1216), CCD algorithm.
void Fit::find_mode_once(const ccdb_mode_args& a, double bound, int* flag, int* iters,
                         double* obj, float* ms) {
    if (!valid_weights || touched_y) {
        apply_weights();
        touched_y = false;
    }
    if (!xb_known) compute_xbeta();
    if (!suff_known) remaining_statistics();
    std::vector<double> hd(J, bound);  // resetBounds
    check_cuda(cudaMemcpyAsync(hdelta, hd.data(), sizeof(double) * J, cudaMemcpyHostToDevice, stream),
               "bounds");
    if (a.algorithm == CCDB_ALGORITHM_MM) {
        auto t0 = std::chrono::steady_clock::now();
        nz_known = false;  // the MM cycle moves every coordinate at once
        find_mode_mm(a, flag, iters, obj);
        *ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return;
    }
    if (a.per_coordinate) {
        // the reference's call pattern: one host round trip per coordinate
        double last = objective(a.convergence_type);
        int iteration = 0;
        bool done = false;
        auto t0 = std::chrono::steady_clock::now();
        while (!done) {
            for (int j = 0; j < J; ++j) {
                if (fixed[j]) continue;
                double g, h;
                gradient_hessian(j, &g, &h);
                double delta = newton_prior_delta(g, h, beta_h[j], ptype_h[j], pvar_h[j]);
                delta = apply_bounds(delta, hd[j]);
                if (delta != 0.0) {
                    update_xbeta(j, delta);
                    ++nz_steps;
                }
            }
            ++iteration;
            const double cur = objective(a.convergence_type);
            double conv;
            bool ill = false;
            if (cur != cur) {
                conv = 0.0;
                ill = true;
            } else {
                conv = std::fabs(cur - last) / (std::fabs(cur) + 1.0);
            }
            last = cur;
            if (a.tolerance > 0 && conv < a.tolerance) {
                *flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
                done = true;
            } else if (iteration == a.max_iterations) {
                *flag = R_MAX_ITERATIONS;
                done = true;
            }
        }
        *iters = iteration;
        *obj = last;
        *ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        check_cuda(cudaMemcpyAsync(hdelta, hd.data(), sizeof(double) * J, cudaMemcpyHostToDevice, stream),
                   "bounds");
        return;
    }
    if (group_engine() && a.strategy != CCDB_SWEEP_SPECULATIVE) {
        find_mode_group_sweep(a, flag, iters, obj, ms);
        return;
    }
    if (use_resident(a)) {
        find_mode_resident(a, flag, iters, obj, ms);
        return;
    }
    if (group_engine() || use_speculative(a)) {
        auto t0 = std::chrono::steady_clock::now();
        find_mode_batched(a, bound, flag, iters, obj);
        *ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return;
    }
    const int kind = sweep_kind(a);
    ensure_schedule(kind);
    if (sched->host.n_levels == 0) {
        // every coordinate is fixed: each cycle changes nothing, so the first
        // convergence check sees conv = 0 (findMode with an empty cycle)
        *obj = objective(a.convergence_type);
        *flag = (*obj != *obj) ? R_ILLCONDITIONED
                : (a.tolerance > 0 ? R_SUCCESS : (a.max_iterations == 1 ? R_MAX_ITERATIONS : R_SUCCESS));
        *iters = 1;
        *ms = 0.f;
        return;
    }
    DevStatus zero{};
    zero.flag = R_FAIL;
    check_cuda(cudaMemcpyAsync(st, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream), "status");
    if (kind == kSchedGrid) {
        check_cuda(cudaMemsetAsync(sched->level_done, 0, sizeof(unsigned) * std::max(1, sched->host.n_levels), stream), "reset");
        check_cuda(cudaMemsetAsync(sched->col_arrive, 0, sizeof(unsigned) * std::max(1, J), stream), "reset");
        check_cuda(cudaMemsetAsync(grid_bar, 0, sizeof(unsigned), stream), "reset");
    }
    IndepParams P = params();
    P.conv = a.convergence_type;
    P.tol = a.tolerance;
    P.max_iter = a.max_iterations;
    // CCDB_TRACE_FILE=<path>: dump per-segment timestamps of the first sweep
    // together with the schedule (profiling aid; off by default)
    const char* trace_path = std::getenv("CCDB_TRACE_FILE");
    unsigned long long* d_trace = nullptr;
    const size_t n_seg = sched->host.segs.size();
    if (trace_path && kind == kSchedCluster) {
        // the cluster sweep: 4 timestamps per level and CTA of the first sweep
        const size_t n = 4 * (size_t)sched->host.n_levels * sched->cluster;
        d_trace = static_cast<unsigned long long*>(ctx->alloc(sizeof(unsigned long long) * n));
        check_cuda(cudaMemsetAsync(d_trace, 0, sizeof(unsigned long long) * n, stream), "trace");
        P.trace = d_trace;
    } else if (trace_path) {
        d_trace = static_cast<unsigned long long*>(ctx->alloc(sizeof(unsigned long long) * 5 * n_seg));
        check_cuda(cudaMemsetAsync(d_trace, 0, sizeof(unsigned long long) * 5 * n_seg, stream), "trace");
        P.trace = d_trace;
        P.trace2 = d_trace + 3 * n_seg;
    }
    check_cuda(cudaEventRecord(ctx->fev[0], stream), "event");
    if (kind == kSchedCluster) check_cuda(launch_cluster_sweep(P, sched->cluster, stream), "sweep launch");
    else check_cuda(launch_indep_sweep(P, sched->host.n_cta, stream), "sweep launch");
    ++launches;
    check_cuda(cudaEventRecord(ctx->fev[1], stream), "event");
    // the host waits for the sweep before it queues the copy back: a device-to-host
    // copy queued behind a long kernel held up the copies of other contexts'
    // streams, so fits served side by side finished together with the longest one
    check_cuda(ctx->wait(), "sweep");
    DevStatus out{};
    check_cuda(cudaMemcpyAsync(&out, st, sizeof(out), cudaMemcpyDeviceToHost, stream), "status");
    check_cuda(ctx->wait(), "sweep");
    check_cuda(cudaEventElapsedTime(ms, ctx->fev[0], ctx->fev[1]), "elapsed");
    if (d_trace && kind == kSchedCluster) {
        const size_t n = 4 * (size_t)sched->host.n_levels * sched->cluster;
        std::vector<unsigned long long> tr(n);
        check_cuda(cudaMemcpy(tr.data(), d_trace, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost),
                   "trace copy");
        ctx->release(d_trace);
        d_trace = nullptr;
        if (FILE* fh = std::fopen(trace_path, "wb")) {
            // header: levels, CTAs; then the level of every column, the split flags, the stamps
            const int64_t hdr[2] = {sched->host.n_levels, sched->cluster};
            std::fwrite(hdr, sizeof(int64_t), 2, fh);
            std::fwrite(sched->host.level_of.data(), sizeof(int32_t), sched->host.level_of.size(), fh);
            std::fwrite(sched->host.level_split.data(), 1, sched->host.level_split.size(), fh);
            std::fwrite(tr.data(), sizeof(unsigned long long), n, fh);
            std::fclose(fh);
        }
    }
    if (d_trace) {
        std::vector<unsigned long long> tr(5 * n_seg);
        check_cuda(cudaMemcpy(tr.data(), d_trace, sizeof(unsigned long long) * 5 * n_seg,
                              cudaMemcpyDeviceToHost), "trace copy");
        ctx->release(d_trace);
        if (FILE* fh = std::fopen(trace_path, "wb")) {
            const int64_t ns = (int64_t)n_seg, nt = (int64_t)sched->host.tasks.size();
            std::fwrite(&ns, sizeof(ns), 1, fh);
            std::fwrite(&nt, sizeof(nt), 1, fh);
            std::fwrite(sched->host.segs.data(), sizeof(Seg), n_seg, fh);
            std::fwrite(sched->host.cta_seg.data(), sizeof(int64_t), sched->host.cta_seg.size(), fh);
            std::fwrite(sched->host.tasks.data(), sizeof(Task), nt, fh);
            std::fwrite(tr.data(), sizeof(unsigned long long), tr.size(), fh);
            std::fclose(fh);
        }
    }
    if (out.error != E_NONE)
        throw Error(CCDB_ERR_TIMEOUT, "device wait timed out (code " + std::to_string(out.error) +
                                          " at " + std::to_string(out.error_where) + ")");
    *flag = out.flag;
    *iters = out.iterations;
    *obj = out.objective;
    if (kind == kSchedCluster) nz_steps += (int64_t)out.nonzero_steps;
    else nz_known = false;  // the grid-wide sweep does not count them
    beta_dirty_host = true;
}

// findMode with speculative batches: the gradients of a run of consecutive
// coordinates are computed together against the same state; walking them in
// order, every zero step leaves the state untouched, so the next coordinate's
// gradient is exactly what a sequential sweep would compute.  At the first
// nonzero step the update is applied and the batch restarts after it.  The
// visiting order and every step are those of the sequential cycle
// (CyclicCoordinateDescent.cpp:1008-1021); only the wasted speculative
// gradients cost extra.  Batches shrink after a restart and grow while steps
// stay zero.
void Fit::find_mode_batched(const ccdb_mode_args& a, double bound, int* flag, int* iters, double* obj) {
    std::vector<double> hd(J, bound);
    std::vector<int32_t> cols;
    for (int j = 0; j < J; ++j)
        if (!fixed[j]) cols.push_back(j);
    const int n_active = (int)cols.size();
    std::vector<double2> gh(kBatchMax);
    double last = objective(a.convergence_type);
    int iteration = 0;
    bool done = false;
    while (!done) {
        int pos = 0, batch = 32;
        while (pos < n_active) {
            const int nb = std::min(batch, n_active - pos);
            gh_batch(cols.data() + pos, nb, gh.data());
            int advanced = nb;
            for (int i = 0; i < nb; ++i) {
                const int j = cols[pos + i];
                double delta = newton_prior_delta(gh[i].x, gh[i].y, beta_h[j], ptype_h[j], pvar_h[j]);
                delta = apply_bounds(delta, hd[j]);
                if (delta != 0.0) {
                    beta_h[j] += delta;
                    apply_step(j, delta);
                    ++nz_steps;
                    advanced = i + 1;
                    break;
                }
            }
            pos += advanced;
            batch = (advanced == nb) ? std::min(2 * batch, (int)kBatchMax) : 32;
        }
        upload_beta();
        ++iteration;
        const double cur = objective(a.convergence_type);
        double conv;
        bool ill = false;
        if (cur != cur) {
            conv = 0.0;
            ill = true;
        } else {
            conv = std::fabs(cur - last) / (std::fabs(cur) + 1.0);
        }
        last = cur;
        if (a.tolerance > 0 && conv < a.tolerance) {
            *flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
            done = true;
        } else if (iteration == a.max_iterations) {
            *flag = R_MAX_ITERATIONS;
            done = true;
        }
    }
    check_cuda(cudaMemcpyAsync(hdelta, hd.data(), sizeof(double) * J, cudaMemcpyHostToDevice, stream),
               "bounds");
    check_cuda(ctx->wait(), "batched sync");
    *iters = iteration;
    *obj = last;
}

void Fit::gh_batch(const int32_t* cols, int n, double2* out) {
    if (group_engine()) {
        cox_gh_batch(cols, n, out);
        return;
    }
    if (!d_batch_cols) {
        d_batch_cols = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * kBatchMax));
        d_batch_out = static_cast<double2*>(ctx->alloc(sizeof(double2) * kBatchMax));
    }
    check_cuda(cudaMemcpyAsync(d_batch_cols, cols, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream),
               "batch cols");
    IndepParams P = params();
    check_cuda(launch_indep_gh_batch(P, d_batch_cols, n, d_batch_out, stream), "gh batch");
    ++launches;
    check_cuda(cudaMemcpyAsync(out, d_batch_out, sizeof(double2) * n, cudaMemcpyDeviceToHost, stream),
               "gh copy");
    check_cuda(ctx->wait(), "gh sync");
}

void Fit::apply_step(int j, double delta) {
    if (group_engine()) {
        cox_update(j, delta);
        return;
    }
    IndepParams P = params();
    check_cuda(launch_indep_update(P, j, m->fmt[j], m->entries(j), delta, stream), "update");
    launches += m->entries(j) > 0 ? 1 : 0;
}

// The host-driven speculative batches (one round trip per batch of gradients
// and per nonzero step) run only when asked for; every default path of the
// independent-row models is the on-device cluster sweep.
bool Fit::use_speculative(const ccdb_mode_args& a) const { return a.strategy == CCDB_SWEEP_SPECULATIVE; }

// The resident sweep serves independent-row fits whose row state fits one
// CTA's shared memory (chosen by CCDB_SWEEP_AUTO), and in its global form
// (the row state in device memory) larger fits when asked for
// (CCDB_SWEEP_RESIDENT).  AUTO leaves larger fits to the cluster sweep: on 43
// L1 logistic fits of 14,000-96,000 rows the global form took 38 s in all
// against the cluster sweep's 17.8 s (it won only on some fits of columns
// below ~250 entries).
bool Fit::use_resident(const ccdb_mode_args& a) {
    if (group_engine()) return false;
    if (a.strategy != CCDB_SWEEP_AUTO && a.strategy != CCDB_SWEEP_RESIDENT) return false;
    if (ctx->resident_rows < 0) {
        int64_t r = 0;
        check_cuda(resident_max_rows(model, &r), "resident capacity");
        ctx->resident_rows = r;
    }
    return K <= ctx->resident_rows || a.strategy == CCDB_SWEEP_RESIDENT;
}

void Fit::find_mode_resident(const ccdb_mode_args& a, int* flag, int* iters, double* obj, float* ms) {
    std::vector<int32_t> cols;
    for (int j = 0; j < J; ++j)
        if (!fixed[j]) cols.push_back(j);
    if (cols.empty()) {  // an empty cycle: the first check sees conv = 0
        *obj = objective(a.convergence_type);
        *flag = (*obj != *obj) ? R_ILLCONDITIONED
                : (a.tolerance > 0 ? R_SUCCESS : (a.max_iterations == 1 ? R_MAX_ITERATIONS : R_SUCCESS));
        *iters = 1;
        *ms = 0.f;
        return;
    }
    // the column records in visiting order
    std::vector<ResCol> recs(cols.size());
    for (size_t q = 0; q < cols.size(); ++q) {
        const int j = cols[q];
        const uint8_t f = m->fmt[j];
        const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
        ResCol& r = recs[q];
        r.j = j;
        r.flags = (has_rows ? 1 : 0) | ((f == F_SPARSE || f == F_DENSE) ? 2 : 0) |
                  ((f == F_INDICATOR || f == F_INTERCEPT) ? 4 : 0);
        r.n = has_rows ? m->col_start[j + 1] - m->col_start[j] : K;
        r.cb = m->col_start[j];
        r.vb = m->val_start[j];
    }
    if (d_res_cap < (int32_t)recs.size()) {
        ctx->release(d_res_recs);
        d_res_recs = static_cast<ResCol*>(ctx->alloc(sizeof(ResCol) * recs.size()));
        d_res_cap = (int32_t)recs.size();
    }
    check_cuda(cudaMemcpyAsync(d_res_recs, recs.data(), sizeof(ResCol) * recs.size(), cudaMemcpyHostToDevice,
                               stream), "column records");
    DevStatus zero{};
    zero.flag = R_FAIL;
    check_cuda(cudaMemcpyAsync(st, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream), "status");
    ResidentParams R{};
    R.P = params();
    R.P.conv = a.convergence_type;
    R.P.tol = a.tolerance;
    R.P.max_iter = a.max_iterations;
    R.recs = d_res_recs;
    R.n_active = (int32_t)recs.size();
    R.weighted = weighted ? 1 : 0;
    if (K > ctx->resident_rows) {  // the global form: the row state in a device array
        if (!d_res_rs) d_res_rs = static_cast<double2*>(ctx->alloc(sizeof(double2) * (size_t)K));
        R.rs = d_res_rs;
    }
    // CCDB_TRACE_FILE=<path>: SM-clock stamps of the first batches (profiling aid; off by default)
    const char* trace_path = std::getenv("CCDB_TRACE_FILE");
    const int trace_n = 4096;
    if (trace_path) {
        R.trace = static_cast<long long*>(ctx->alloc(sizeof(long long) * kResidentTraceWords * trace_n));
        check_cuda(cudaMemsetAsync(R.trace, 0, sizeof(long long) * kResidentTraceWords * trace_n, stream), "trace");
        R.trace_n = trace_n;
    }
    check_cuda(cudaEventRecord(ctx->fev[0], stream), "event");
    check_cuda(launch_resident_sweep(R, stream), "resident sweep launch");
    ++launches;
    check_cuda(cudaEventRecord(ctx->fev[1], stream), "event");
    check_cuda(ctx->wait(), "resident sweep");  // the sweep is done before a copy is queued behind it
    DevStatus out{};
    check_cuda(cudaMemcpyAsync(&out, st, sizeof(out), cudaMemcpyDeviceToHost, stream), "status");
    check_cuda(ctx->wait(), "resident sweep");
    check_cuda(cudaEventElapsedTime(ms, ctx->fev[0], ctx->fev[1]), "elapsed");
    if (R.trace) {
        std::vector<long long> tr((size_t)kResidentTraceWords * trace_n);
        check_cuda(cudaMemcpyAsync(tr.data(), R.trace, sizeof(long long) * tr.size(), cudaMemcpyDeviceToHost, stream),
                   "trace copy");
        check_cuda(ctx->wait(), "trace copy");
        ctx->release(R.trace);
        if (FILE* fh = std::fopen(trace_path, "wb")) {
            std::fwrite(tr.data(), sizeof(long long), tr.size(), fh);
            std::fclose(fh);
        }
    }
    *flag = out.flag;
    *iters = out.iterations;
    *obj = out.objective;
    nz_steps += (int64_t)out.nonzero_steps;
    beta_dirty_host = true;
}

void Fit::find_mode(const ccdb_mode_args& a, double* beta_inout, ccdb_fit_result* res) {
    if (!a.prior_type || !a.prior_var) throw Error(CCDB_ERR_INVALID, "prior arrays are required");
    ptype_h.assign(a.prior_type, a.prior_type + J);
    pvar_h.assign(a.prior_var, a.prior_var + J);
    for (int j = 0; j < J; ++j)
        if (ptype_h[j] < 0 || ptype_h[j] > 2) throw Error(CCDB_ERR_UNSUPPORTED, "prior type");
    check_cuda(cudaMemcpyAsync(ptype, ptype_h.data(), sizeof(int32_t) * J, cudaMemcpyHostToDevice, stream), "prior");
    check_cuda(cudaMemcpyAsync(pvar, pvar_h.data(), sizeof(double) * J, cudaMemcpyHostToDevice, stream), "prior");
    if (a.convergence_type < C_GRADIENT || a.convergence_type > C_MITTAL)
        throw Error(CCDB_ERR_UNSUPPORTED, "convergence type");
    if (a.algorithm != CCDB_ALGORITHM_CCD && a.algorithm != CCDB_ALGORITHM_MM)
        throw Error(CCDB_ERR_UNSUPPORTED, "algorithm");
    if (a.algorithm == CCDB_ALGORITHM_MM && !group_engine())
        throw Error(CCDB_ERR_UNSUPPORTED,
                    model == M_POISSON ? "Not model-specific" : "the MM algorithm needs stratified data");
    if (a.fixed)  // setFixedBeta for every column; the offset stays fixed
        for (int j = 0; j < J; ++j) fixed[j] = (a.fixed[j] != 0 || (offset_col0 && j == 0)) ? 1 : 0;
    bool any_laplace = false;
    for (int j = 0; j < J; ++j) any_laplace |= (ptype_h[j] == 1);
    const bool swindle = a.use_kkt_swindle && any_laplace;
    if (beta_inout) {
        for (int j = 0; j < J; ++j) beta_h[j] = beta_inout[j];
        upload_beta();
        xb_known = false;
        suff_known = false;
    }
    int active = 0;
    for (int j = 0; j < J; ++j) active += fixed[j] ? 0 : 1;
    const int64_t launches0 = launches;
    nz_steps = 0;
    nz_known = true;
    check_cuda(cudaEventRecord(ctx->fev[2], stream), "event");
    double bound = a.initial_bound;
    int count = 0, flag = R_FAIL, sweeps_total = 0;
    double obj = 0.0, secs = 0.0;
    int64_t updates = 0;
    for (;;) {
        float ms = 0.f;
        // A swindle whose active set stays empty runs no findMode and leaves the
        // count as it was: the reference then reports its lastIterationCount from
        // the previous fit (CyclicCoordinateDescent.cpp:696-709, :1209).
        int iters = -1;
        if (swindle) kkt_swindle(a, bound, &flag, &iters, &obj, &ms);
        else find_mode_once(a, bound, &flag, &iters, &obj, &ms);
        secs += ms * 1e-3;
        if (iters >= 0) {
            last_iterations = iters;
            updates += (int64_t)iters * active;
            sweeps_total += iters;
        }
        ++count;
        if (beta_dirty_host) {
            download_beta();
            beta_dirty_host = false;
        }
        if (flag == R_ILLCONDITIONED && count < a.max_bound_count) {
            bound /= 10.0;  // resetBeta (.cpp:256-264)
            for (int j = offset_col0 ? 1 : 0; j < J; ++j) beta_h[j] = 0.0;
            upload_beta();
            compute_xbeta();
            suff_known = false;
        } else {
            break;
        }
    }
    if (beta_inout)
        for (int j = 0; j < J; ++j) beta_inout[j] = beta_h[j];
    const double ll = log_likelihood();
    check_cuda(cudaEventRecord(ctx->fev[3], stream), "event");
    check_cuda(cudaEventSynchronize(ctx->fev[3]), "event sync");
    float call_ms = 0.f;
    check_cuda(cudaEventElapsedTime(&call_ms, ctx->fev[2], ctx->fev[3]), "elapsed");
    if (res) {
        res->return_flag = flag;
        res->iterations = last_iterations;
        res->objective = obj;
        res->log_likelihood = ll;
        res->coordinate_updates = updates;
        res->device_seconds = call_ms * 1e-3;
        res->kernel_seconds = secs;
        res->kernel_launches = launches - launches0;
        res->attempts = count;
        res->sweeps_total = sweeps_total;
        res->nonzero_steps = nz_known ? nz_steps : -1;
    }
}

}  // namespace ccdb

// ====================================================================== C ABI
using namespace ccdb;

struct ccdb_context : Context {};
struct ccdb_matrix : Matrix {};
struct ccdb_fit : Fit {};

namespace {

template <typename F>
int guard(F&& f) {
    try {
        f();
        return CCDB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return CCDB_ERR_INVALID;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return CCDB_ERR_INVALID;
    }
}

void require(bool ok, const char* msg) {
    if (!ok) throw Error(CCDB_ERR_INVALID, msg);
}

}  // namespace

extern "C" {

const char* ccdb_last_error(void) { return g_last_error.c_str(); }

int ccdb_context_create(int device, size_t hbm_budget_bytes, ccdb_context** out) {
    return guard([&] {
        require(out != nullptr, "out is NULL");
        int n = 0;
        check_cuda(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
        require(device >= 0 && device < n, "no such CUDA device");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        auto* c = new ccdb_context();
        c->device = device;
        c->budget = hbm_budget_bytes;
        check_cuda(cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, device), "attr");
        int coop = 0;
        check_cuda(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device), "attr");
        if (!coop) {
            delete c;
            throw Error(CCDB_ERR_UNSUPPORTED, "device lacks cooperative launch");
        }
        check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        check_cuda(cudaMemPoolCreate(&c->pool, &props), "memory pool");
        uint64_t keep = UINT64_MAX;  // freed blocks stay reserved for the next fit
        check_cuda(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
        check_cuda(cudaEventCreate(&c->ev_a), "event");
        check_cuda(cudaEventCreate(&c->ev_b), "event");
        for (cudaEvent_t& e : c->fev) check_cuda(cudaEventCreate(&e), "event");
        *out = c;
    });
}

int ccdb_context_destroy(ccdb_context* ctx) {
    return guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        cudaEventDestroy(ctx->ev_a);
        cudaEventDestroy(ctx->ev_b);
        for (cudaEvent_t e : ctx->fev) cudaEventDestroy(e);
        if (ctx->ev_wait) cudaEventDestroy(ctx->ev_wait);
        cudaStreamDestroy(ctx->stream);
        if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
        delete ctx;
    });
}

int ccdb_context_set_blocking_wait(ccdb_context* ctx, int32_t on) {
    return guard([&] {
        require(ctx != nullptr, "NULL context");
        check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        check_cuda(cudaStreamSynchronize(ctx->stream), "sync");
        ctx->blocking_wait = on != 0;
        if (ctx->blocking_wait && !ctx->ev_wait)
            check_cuda(cudaEventCreateWithFlags(&ctx->ev_wait, cudaEventBlockingSync | cudaEventDisableTiming),
                       "event");
        // the context's timing events follow the setting
        for (cudaEvent_t* e : {&ctx->ev_a, &ctx->ev_b, &ctx->fev[0], &ctx->fev[1], &ctx->fev[2], &ctx->fev[3]}) {
            if (*e) check_cuda(cudaEventDestroy(*e), "event");
            check_cuda(cudaEventCreateWithFlags(e, ctx->event_flags()), "event");
        }
    });
}

int ccdb_context_sm_count(const ccdb_context* ctx, int32_t* n_sm) {
    return guard([&] {
        require(ctx && n_sm, "NULL argument");
        *n_sm = ctx->n_sm;
    });
}

int ccdb_context_set_max_ctas(ccdb_context* ctx, int32_t max_ctas) {
    return guard([&] {
        require(ctx != nullptr, "NULL context");
        require(max_ctas >= 0, "max_ctas must be >= 0");
        ctx->max_ctas = max_ctas;
    });
}

int ccdb_context_memory(const ccdb_context* ctx, size_t* bytes) {
    return guard([&] {
        require(ctx && bytes, "NULL argument");
        *bytes = ctx->in_use;
    });
}

// The CompressedDataMatrix contract every matrix is checked against before any
// device work (host only).
// The first of columns [0, n_cols) whose row ids are not ascending within
// [0, K), or n_cols: column ranges of about equal entry counts checked on
// host threads (the check is a memory-bound walk of the row ids, vectorised
// within a column), the lowest failing column kept -- the one a walk in
// column order would report.
static int32_t first_row_error(int64_t K, int32_t n_cols, const int64_t* col_start, const int32_t* rows) {
    auto bad = [&](int32_t j) {
        const int64_t b = col_start[j], e = col_start[j + 1];
        if (e <= b) return false;
        unsigned ok = (unsigned)(rows[b] >= 0) & (unsigned)((int64_t)rows[e - 1] < K);
        for (int64_t p = b + 1; p < e; ++p) ok &= (unsigned)(rows[p] > rows[p - 1]);
        return ok == 0u;
    };
    const int64_t total = n_cols > 0 ? col_start[n_cols] : 0;
    const int64_t per_thread = int64_t(1) << 21;
    const int T = (int)std::max<int64_t>(
        1, std::min<int64_t>({(int64_t)std::max(1u, std::thread::hardware_concurrency()), total / per_thread, 16}));
    if (T == 1) {
        for (int32_t j = 0; j < n_cols; ++j)
            if (bad(j)) return j;
        return n_cols;
    }
    std::vector<int32_t> lo(T + 1, n_cols), found(T, n_cols);
    lo[0] = 0;
    for (int32_t j = 0, t = 1; j < n_cols && t < T; ++j)
        if (col_start[j + 1] >= total * t / T) lo[t++] = j + 1;
    auto walk = [&](int t) {
        for (int32_t j = lo[t]; j < lo[t + 1]; ++j)
            if (bad(j)) {
                found[t] = j;
                return;
            }
    };
    std::vector<std::thread> pool;
    int started = 0;
    try {
        for (; started < T; ++started) pool.emplace_back(walk, started);
    } catch (const std::system_error&) {  // no more threads: this one walks the rest
        for (int t = started; t < T; ++t) walk(t);
    }
    for (auto& th : pool) th.join();
    return *std::min_element(found.begin(), found.end());
}

static void validate_matrix(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                            const int64_t* val_start, const double* vals, const uint8_t* fmt) {
    require(col_start && val_start && fmt, "NULL argument");
    require(K > 0 && K < (int64_t(1) << 31) && J > 0, "bad dimensions");
    const int64_t nnz = col_start[J], nv = val_start[J];
    require(col_start[0] == 0 && val_start[0] == 0 && nnz >= 0 && nv >= 0, "bad offsets");
    require(nnz == 0 || rows, "rows is NULL");
    require(nv == 0 || vals, "vals is NULL");
    // offsets and formats column by column; the columns before the first bad
    // one have offsets within [0, nnz] and [0, nv], so their row ids can be read
    int32_t first_bad = J;
    const char* why = nullptr;
    for (int32_t j = 0; j < J && !why; ++j) {
        const int64_t nr = col_start[j + 1] - col_start[j], nvj = val_start[j + 1] - val_start[j];
        if (nr < 0 || nvj < 0 || col_start[j + 1] > nnz || val_start[j + 1] > nv) {
            why = "offsets must be non-decreasing";
        } else {
            switch (fmt[j]) {
            case F_DENSE: if (!(nr == 0 && nvj == K)) why = "DENSE column needs K values, no rows"; break;
            case F_INTERCEPT: if (!(nr == 0 && nvj == 0)) why = "INTERCEPT column takes no data"; break;
            case F_INDICATOR: if (nvj != 0) why = "INDICATOR column takes no values"; break;
            case F_SPARSE: if (nvj != nr) why = "SPARSE column needs one value per row"; break;
            default: why = "unknown column format";
            }
        }
        if (why) first_bad = j;
    }
    // a row-id error in an earlier column comes first, as in a walk in column order
    require(first_row_error(K, first_bad, col_start, rows) == first_bad, "row ids must be ascending and < K");
    require(why == nullptr, why ? why : "");
}

int ccdb_matrix_validate(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                         const int64_t* val_start, const double* vals, const uint8_t* fmt) {
    return guard([&] { validate_matrix(K, J, col_start, rows, val_start, vals, fmt); });
}

int ccdb_matrix_create(ccdb_context* ctx, int64_t K, int32_t J, const int64_t* col_start,
                       const int32_t* rows, const int64_t* val_start, const double* vals,
                       const uint8_t* fmt, ccdb_matrix** out) {
    return guard([&] {
        require(ctx && out, "NULL argument");
        validate_matrix(K, J, col_start, rows, val_start, vals, fmt);
        check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        std::unique_ptr<ccdb_matrix> m(new ccdb_matrix());
        m->ctx = ctx;
        m->K = K;
        m->J = J;
        m->col_start.assign(col_start, col_start + J + 1);
        m->val_start.assign(val_start, val_start + J + 1);
        m->fmt.assign(fmt, fmt + J);
        const int64_t nnz = col_start[J], nv = val_start[J];
        m->rows_h.assign(rows, rows + nnz);
        m->vals_h.assign(vals, vals + nv);
        cudaStream_t s = ctx->stream;
        m->d_col_ptr = upload(ctx, col_start, J + 1, s);
        m->d_val_ptr = upload(ctx, val_start, J + 1, s);
        m->d_fmt = upload(ctx, fmt, J, s);
        m->d_rows = upload(ctx, rows, nnz, s);
        m->d_vals = upload(ctx, vals, nv, s);
        check_cuda(ctx->wait(), "matrix upload");
        *out = m.release();
    });
}

int ccdb_matrix_destroy(ccdb_matrix* m) {
    return guard([&] { delete m; });
}

int ccdb_matrix_row_major(ccdb_matrix* m, int64_t* row_ptr, int32_t* col, double* val) {
    return guard([&] {
        require(m && row_ptr && col && val, "NULL argument");
        check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
        cudaStream_t s = m->ctx->stream;
        m->ensure_csr(s);
        int64_t total = 0;
        for (int j = 0; j < m->J; ++j) total += m->entries(j);
        check_cuda(cudaMemcpyAsync(row_ptr, m->d_row_ptr, sizeof(int64_t) * (size_t)(m->K + 1),
                                   cudaMemcpyDeviceToHost, s), "row offsets");
        if (total > 0) {
            check_cuda(cudaMemcpyAsync(col, m->d_csr_col, sizeof(int32_t) * (size_t)total, cudaMemcpyDeviceToHost, s),
                       "columns");
            check_cuda(cudaMemcpyAsync(val, m->d_csr_val, sizeof(double) * (size_t)total, cudaMemcpyDeviceToHost, s),
                       "values");
        }
        check_cuda(m->ctx->wait(), "row-major copy");
    });
}

int ccdb_fit_create(ccdb_context* ctx, const ccdb_matrix* m, const ccdb_fit_desc* d, ccdb_fit** out) {
    return guard([&] {
        require(ctx && m && d && out && d->y, "NULL argument");
        require(m->ctx == ctx, "matrix belongs to another context");
        if (d->model_type != M_LOGISTIC && d->model_type != M_POISSON && d->model_type != M_COX &&
            d->model_type != M_CLR && d->model_type != M_CPR)
            throw Error(CCDB_ERR_UNSUPPORTED, "model type not supported by this engine");
        if ((d->model_type == M_CLR || d->model_type == M_CPR) && !d->stratum)
            throw Error(CCDB_ERR_INVALID, "conditional models need stratum ids");
        if (d->model_type == M_COX && !d->time)
            throw Error(CCDB_ERR_INVALID, "Cox fits need survival times");
        if (d->precision != CCDB_PRECISION_FP64 &&
            !(d->precision == CCDB_PRECISION_MIXED &&
              (d->model_type == M_LOGISTIC || d->model_type == M_POISSON || d->model_type == M_COX)))
            throw Error(CCDB_ERR_UNSUPPORTED, "precision not supported for this model");
        check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        std::unique_ptr<ccdb_fit> f(new ccdb_fit());
        f->ctx = ctx;
        f->m = m;
        f->model = d->model_type;
        f->precision = d->precision;
        f->K = m->K;
        f->J = m->J;
        f->offset_col0 = d->offset_col0 != 0;
        f->stream = ctx->stream;
        f->y_h.assign(d->y, d->y + m->K);
        const int64_t K = m->K;
        const int J = m->J;
        if (d->time) f->time_h.assign(d->time, d->time + K);
        if (d->stratum) f->stratum_h.assign(d->stratum, d->stratum + K);
        else f->stratum_h.assign(K, 0);  // one stratum, as R's rep(1, n) for unstratified Cox
        const bool grp_engine = (f->model == M_COX || f->model == M_CLR || f->model == M_CPR);
        if (!grp_engine) f->row = static_cast<double2*>(ctx->alloc(sizeof(double2) * 2 * K));
        f->y = upload(ctx, d->y, K, f->stream);
        f->beta = static_cast<double*>(ctx->alloc(sizeof(double) * J));
        f->hdelta = static_cast<double*>(ctx->alloc(sizeof(double) * J));
        f->xjy = static_cast<double*>(ctx->alloc(sizeof(double) * J));
        f->ptype = static_cast<int32_t*>(ctx->alloc(sizeof(int32_t) * J));
        f->pvar = static_cast<double*>(ctx->alloc(sizeof(double) * J));
        f->st = static_cast<DevStatus*>(ctx->alloc(sizeof(DevStatus)));
        f->grid_bar = static_cast<unsigned*>(ctx->alloc(sizeof(unsigned)));
        f->red = static_cast<double2*>(ctx->alloc(sizeof(double2) * 4 * ctx->n_sm * 2));
        f->xb_tmp = static_cast<double*>(ctx->alloc(sizeof(double) * K));
        f->w = static_cast<double*>(ctx->alloc(sizeof(double) * K));
        f->gh_parts = static_cast<double2*>(ctx->alloc(sizeof(double2) * Fit::kGhParts));
        f->gh_out = static_cast<double2*>(ctx->alloc(sizeof(double2)));
        // CyclicCoordinateDescent::init (.cpp:200-239)
        f->beta_h.assign(J, 0.0);
        f->fixed.assign(J, 0);
        f->ptype_h.assign(J, 0);
        f->pvar_h.assign(J, 1.0);
        if (f->offset_col0) {
            f->beta_h[0] = 1.0;
            f->fixed[0] = 1;
            f->xb_known = false;
        } else {
            f->xb_known = false;  // xBeta = 0: computed (zero-filled) on first use
        }
        f->upload_beta();
        if (grp_engine) f->cox_allocate();
        check_cuda(f->ctx->wait(), "fit upload");
        *out = f.release();
    });
}

int ccdb_fit_destroy(ccdb_fit* f) {
    return guard([&] { delete f; });
}

// Mixed precision of logistic and Poisson fits is implemented by the batched
// engine; their single-fit calls compute in FP64 only and refuse a mixed fit
// rather than ignore its setting.  Cox fits take it in every call.
static void require_fp64(const ccdb_fit* f) {
    if (f->precision != CCDB_PRECISION_FP64 && f->model != M_COX)
        throw Error(CCDB_ERR_UNSUPPORTED, "mixed precision serves batched fits (ccdb_batch_find_mode) only");
}

int ccdb_set_weights(ccdb_fit* f, const double* w) {
    return guard([&] {
        require(f != nullptr, "NULL fit");
        if (w) {
            f->w_h.assign(w, w + f->K);
            f->weighted = true;
        } else {
            f->w_h.clear();
            f->weighted = false;
        }
        f->valid_weights = false;
        f->suff_known = false;
    });
}

int ccdb_set_beta(ccdb_fit* f, const double* beta) {
    return guard([&] {
        require(f && beta, "NULL argument");
        f->beta_h.assign(beta, beta + f->J);
        f->upload_beta();
        f->xb_known = false;
        f->suff_known = false;
    });
}

int ccdb_compute_xbeta(ccdb_fit* f, const double* beta) {
    return guard([&] {
        require(f && beta, "NULL argument");
        require_fp64(f);
        f->beta_h.assign(beta, beta + f->J);
        f->upload_beta();
        f->compute_xbeta_transpose();  // the statistics stay stale until computeRemainingStatistics
    });
}

int ccdb_compute_gradient_hessian(ccdb_fit* f, int32_t j, double* g, double* h) {
    return guard([&] {
        require(f && g && h, "NULL argument");
        require_fp64(f);
        require(j >= 0 && j < f->J, "column out of range");
        f->gradient_hessian(j, g, h);
    });
}

int ccdb_update_xbeta(ccdb_fit* f, int32_t j, double delta) {
    return guard([&] {
        require(f != nullptr, "NULL fit");
        require_fp64(f);
        require(j >= 0 && j < f->J, "column out of range");
        f->update_xbeta(j, delta);
    });
}

int ccdb_compute_remaining_statistics(ccdb_fit* f) {
    return guard([&] {
        require(f != nullptr, "NULL fit");
        require_fp64(f);
        f->check_lazy();
        f->remaining_statistics();
        check_cuda(f->ctx->wait(), "sync");
    });
}

int ccdb_get_log_likelihood(ccdb_fit* f, double* ll) {
    return guard([&] {
        require(f && ll, "NULL argument");
        require_fp64(f);
        *ll = f->log_likelihood();
    });
}

int ccdb_get_xbeta(ccdb_fit* f, double* out) {
    return guard([&] {
        require(f && out, "NULL argument");
        require_fp64(f);
        f->check_lazy();
        const int stride = f->group_engine() ? 1 : 2;
        const double2* src = f->group_engine() ? f->cox.xbe : f->row;
        std::vector<double2> r(stride * f->K);
        check_cuda(cudaMemcpyAsync(r.data(), src, sizeof(double2) * stride * f->K, cudaMemcpyDeviceToHost,
                                   f->stream), "xbeta copy");
        check_cuda(f->ctx->wait(), "sync");
        for (int64_t k = 0; k < f->K; ++k) out[k] = r[stride * k].x;
    });
}

int ccdb_get_gradient_objective(ccdb_fit* f, double* out) {
    return guard([&] {
        require(f && out, "NULL argument");
        require_fp64(f);
        double t[4];
        f->objective_terms(t);
        *out = t[2];
    });
}

int ccdb_fisher_information(ccdb_fit* f, const int32_t* indices, int32_t n, double* out) {
    return guard([&] {
        require(f != nullptr, "NULL fit");
        require(n >= 0, "negative column count");
        require(n == 0 || (indices && out), "NULL argument");
        require_fp64(f);
        for (int32_t i = 0; i < n; ++i) require(indices[i] >= 0 && indices[i] < f->J, "column out of range");
        if (f->weighted)
            throw Error(CCDB_ERR_UNSUPPORTED, "Weights are not yet implemented in Fisher Information calculations");
        f->fisher_information(indices, n, out);
    });
}

int ccdb_compute_mm_gradient_hessian(ccdb_fit* f, const uint8_t* fixed, double* gradient, double* hessian) {
    return guard([&] {
        require(f && gradient && hessian, "NULL argument");
        require_fp64(f);
        if (!f->group_engine())
            throw Error(CCDB_ERR_UNSUPPORTED, f->model == M_POISSON ? "Not model-specific"
                                                                    : "the MM algorithm needs stratified data");
        std::vector<double2> gh(f->J);
        f->mm_gradient_hessian(fixed, gh.data());
        for (int j = 0; j < f->J; ++j) {
            gradient[j] = gh[j].x;
            hessian[j] = gh[j].y;
        }
    });
}

int ccdb_get_predictive_log_likelihood(ccdb_fit* f, const double* weights, double* out) {
    return guard([&] {
        require(f && weights && out, "NULL argument");
        require_fp64(f);
        *out = f->predictive_log_likelihood(weights);
    });
}

int ccdb_get_predictive_estimates(ccdb_fit* f, const double* weights, double* y) {
    return guard([&] {
        require(f && y, "NULL argument");
        require_fp64(f);
        std::vector<double> p(f->K);
        f->predictive_estimates(p.data());
        for (int64_t k = 0; k < f->K; ++k)
            if (!weights || weights[k] != 0.0) y[k] = p[k];
    });
}

int ccdb_set_fixed(ccdb_fit* f, const uint8_t* fixed) {
    return guard([&] {
        require(f && fixed, "NULL argument");
        for (int j = 0; j < f->J; ++j) f->fixed[j] = (fixed[j] != 0 || (f->offset_col0 && j == 0)) ? 1 : 0;
    });
}

int ccdb_fit_set_wait_limit(ccdb_fit* f, int64_t nanoseconds) {
    return guard([&] {
        require(f != nullptr, "NULL fit");
        require(nanoseconds >= 0, "the wait limit must be >= 0");
        f->wait_limit_ns = nanoseconds ? nanoseconds : Fit::kDefaultWaitNs;
        f->xch_wait_ns = nanoseconds ? nanoseconds : Fit::kDefaultXchWaitNs;
    });
}

int ccdb_get_last_call_seconds(const ccdb_fit* f, double* seconds) {
    return guard([&] {
        require(f && seconds, "NULL argument");
        *seconds = f->last_call_seconds;
    });
}

int ccdb_get_beta(ccdb_fit* f, double* out) {
    return guard([&] {
        require(f && out, "NULL argument");
        std::copy(f->beta_h.begin(), f->beta_h.end(), out);
    });
}

int ccdb_find_mode(ccdb_fit* f, const ccdb_mode_args* args, double* beta_inout, ccdb_fit_result* res) {
    return guard([&] {
        require(f && args, "NULL argument");
        require_fp64(f);
        check_cuda(cudaSetDevice(f->ctx->device), "cudaSetDevice");
        f->find_mode(*args, beta_inout, res);
    });
}

int ccdb_fit_model(ccdb_context* ctx, int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                   const int64_t* val_start, const double* vals, const uint8_t* fmt,
                   const ccdb_fit_desc* desc, const double* weights, const ccdb_mode_args* args,
                   double* beta_out, ccdb_fit_result* result) {
    ccdb_matrix* m = nullptr;
    ccdb_fit* f = nullptr;
    if (!ctx) {
        g_last_error = "NULL context";
        return CCDB_ERR_INVALID;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess || cudaEventRecord(ctx->ev_a, ctx->stream) != cudaSuccess) {
        g_last_error = "cannot record on the context stream";
        return CCDB_ERR_CUDA;
    }
    int rc = ccdb_matrix_create(ctx, K, J, col_start, rows, val_start, vals, fmt, &m);
    if (rc == CCDB_OK) rc = ccdb_fit_create(ctx, m, desc, &f);
    if (rc == CCDB_OK && weights) rc = ccdb_set_weights(f, weights);
    if (rc == CCDB_OK) rc = ccdb_find_mode(f, args, nullptr, result);
    if (rc == CCDB_OK && beta_out) rc = ccdb_get_beta(f, beta_out);
    if (rc == CCDB_OK && result) {
        float ms = 0.f;
        if (cudaEventRecord(ctx->ev_b, ctx->stream) == cudaSuccess &&
            cudaEventSynchronize(ctx->ev_b) == cudaSuccess &&
            cudaEventElapsedTime(&ms, ctx->ev_a, ctx->ev_b) == cudaSuccess)
            result->device_seconds = ms * 1e-3;
    }
    std::string err = g_last_error;
    if (f) ccdb_fit_destroy(f);
    if (m) ccdb_matrix_destroy(m);
    g_last_error = err;
    return rc;
}

// Lockstep group size of the mixed-precision batched engine.  G = 4 packs the
// group's state for one row into one 32-byte sector (a quarter of the DRAM
// sectors G = 1 moves per instance), but gives one CTA G times the per-column
// arithmetic and leaves ceil(n / G) CTAs for the SMs.  Take the largest G that
// still gives every third SM a CTA.
static int batch_group_size(const Matrix* m, int n, int n_sm) {
    (void)m;
    const int want = std::max(1, n_sm / 3);
    for (int G : {4, 2})
        if ((n + G - 1) / G >= want) return G;
    return 1;
}

// Longest slice of a row-indexed column when C CTAs split the rows evenly.
static int64_t batch_max_slice(const Matrix* m, int64_t K, int C) {
    int64_t mx = 0;
    for (int j = 0; j < m->J; ++j) {
        if (m->fmt[j] != F_SPARSE && m->fmt[j] != F_INDICATOR) continue;
        const int32_t* r0 = m->rows_h.data() + m->col_start[j];
        const int32_t* r1 = m->rows_h.data() + m->col_start[j + 1];
        const int32_t* lo = r0;
        for (int r = 1; r <= C; ++r) {
            const int32_t* hi = (r == C) ? r1 : std::lower_bound(lo, r1, K * r / C);
            mx = std::max<int64_t>(mx, hi - lo);
            lo = hi;
        }
    }
    return mx;
}

// CTAs per group of the mixed engine.  The per-column critical path shrinks
// when a column's rows are split over more SMs (each gathers and updates only
// its slice), and the kernel's registers suffice without spills for the small
// stage (1024 entries per slice).  Take the smallest power of two that both
// fits every slice in the small stage and puts a CTA on every SM; at most 8.
static int batch_cluster_size(const Matrix* m, int64_t K, int n_groups, int n_sm) {
    for (int C = 1; C <= 8; C *= 2)
        if ((int64_t)n_groups * C >= n_sm && batch_max_slice(m, K, C) <= 1024) return C;
    for (int C = 1; C <= 8; C *= 2)
        if (batch_max_slice(m, K, C) <= 1024) return C;
    return 8;
}

int ccdb_batch_find_mode(ccdb_fit* f, const ccdb_batch_desc* b, const ccdb_mode_args* a, double* beta_out,
                         ccdb_batch_result* results, double* device_seconds) {
    return guard([&] {
        require(f && b && a && a->prior_type && b->variance && b->n_instances > 0, "NULL argument");
        if (f->model != M_LOGISTIC && f->model != M_POISSON)
            throw Error(CCDB_ERR_UNSUPPORTED, "batched fits support logistic and Poisson models");
        if (a->convergence_type < C_GRADIENT || a->convergence_type > C_MITTAL)
            throw Error(CCDB_ERR_UNSUPPORTED, "convergence type");
        Context* ctx = f->ctx;
        check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        const int n = b->n_instances;
        const int64_t K = f->K;
        const int J = f->J;
        const Matrix* m = f->m;
        cudaStream_t s = f->stream;
        std::vector<void*> owned;
        auto keep = [&](void* p) { owned.push_back(p); return p; };
        struct Release {
            Context* c;
            std::vector<void*>* v;
            ~Release() { for (void* p : *v) c->release(p); }
        } rel{ctx, &owned};
        BatchParams P{};
        P.col_ptr = m->d_col_ptr;
        P.rows = m->d_rows;
        P.val_ptr = m->d_val_ptr;
        P.vals = m->d_vals;
        P.fmt = m->d_fmt;
        P.K = K;
        P.J = J;
        P.model = f->model;
        P.n_inst = n;
        P.conv = a->convergence_type;
        P.max_iter = a->max_iterations;
        P.tol = a->tolerance;
        P.initial_bound = a->initial_bound;
        P.y = f->y;
        if (b->row_fold) P.row_fold = (const int32_t*)keep(upload(ctx, b->row_fold, (size_t)K, s));
        std::vector<int32_t> hold(n, -1);
        if (b->holdout) hold.assign(b->holdout, b->holdout + n);
        P.holdout = (const int32_t*)keep(upload(ctx, hold.data(), (size_t)n, s));
        P.variance = (const double*)keep(upload(ctx, b->variance, (size_t)n, s));
        P.ptype = (const int32_t*)keep(upload(ctx, a->prior_type, (size_t)J, s));
        if (f->offset_col0) {
            if (m->fmt[0] != F_DENSE) throw Error(CCDB_ERR_UNSUPPORTED, "offset column must be DENSE");
            P.offset_vals = m->d_vals + m->val_start[0];
        }
        if (f->model == M_POISSON) {  // fixed terms per instance (ModelSpecifics.h:1596-1601)
            std::vector<double> table(1, 0.0), fixed(n, 0.0);
            for (int i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int64_t k = 0; k < K; ++k) {
                    const int yi = (int)f->y_h[k];
                    while ((int)table.size() <= yi) {
                        const int c = (int)table.size();
                        table.push_back(c >= 2 ? table.back() + -std::log((double)c) : 0.0);
                    }
                    const double t = yi >= 2 ? table[yi] : 0.0;
                    const double w = (b->row_fold && hold[i] >= 0 && b->row_fold[k] == hold[i]) ? 0.0 : 1.0;
                    acc += t * w;
                }
                fixed[i] = acc;
            }
            P.ll_fixed = (const double*)keep(upload(ctx, fixed.data(), (size_t)n, s));
        }
        const bool mixed = f->precision == CCDB_PRECISION_MIXED;
        // weakest priors first: they need the most sweeps, so they start in the first wave
        // (and, in mixed precision, instances of similar variance share a group)
        std::vector<int32_t> order(n);
        for (int i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t x, int32_t y) { return b->variance[x] > b->variance[y]; });
        P.order = (const int32_t*)keep(upload(ctx, order.data(), (size_t)n, s));
        P.results = (BatchResult*)keep(ctx->alloc(sizeof(BatchResult) * n));
        int G = 1, n_groups = n;
        if (mixed) {
            G = b->group ? b->group : batch_group_size(m, n, ctx->n_sm);
            if (G != 1 && G != 2 && G != 4) throw Error(CCDB_ERR_INVALID, "batch group must be 1, 2 or 4");
            n_groups = (n + G - 1) / G;
            P.group = G;
            // the mixed engine reads each entry's fold with its row id (row | fold << 24)
            if (K > kKeyRowMask)
                throw Error(CCDB_ERR_UNSUPPORTED, "mixed batched fits: at most 16,777,215 rows");
            for (int i = 0; i < n; ++i)
                if (hold[i] >= kKeyNoFold)
                    throw Error(CCDB_ERR_UNSUPPORTED, "mixed batched fits: held-out fold ids below 127");
            const int64_t nnz = m->col_start.back();
            int32_t* keys = (int32_t*)keep(ctx->alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1)));
            check_cuda(launch_batch_keys(m->d_rows, nnz, P.row_fold, keys, s), "batch keys");
            P.keys = keys;
            // CTAs per group (a cluster splits each column's rows among its CTAs):
            // the caller's choice, else the tuner's
            int C = b->cluster ? b->cluster : batch_cluster_size(m, K, n_groups, ctx->n_sm);
            if (C < 1 || C > 16) throw Error(CCDB_ERR_INVALID, "batch cluster size must be 1..16");
            P.cluster = C;
            // per row-indexed column, where its rows cross the CTAs' row boundaries;
            // the stage capacity is the small variant when every slice fits it
            std::vector<int32_t> split((size_t)J * (C + 1), 0);
            int64_t max_slice = 0;
            for (int j = 0; j < J; ++j) {
                const int64_t cb = m->col_start[j], ce = m->col_start[j + 1];
                const int32_t* r0 = m->rows_h.data() + cb;
                const int32_t* r1 = m->rows_h.data() + ce;
                int32_t* sp = split.data() + (size_t)j * (C + 1);
                for (int r = 0; r <= C; ++r)
                    sp[r] = (r == C) ? (int32_t)(ce - cb) : (int32_t)(std::lower_bound(r0, r1, K * r / C) - r0);
                if (m->fmt[j] == F_SPARSE || m->fmt[j] == F_INDICATOR)
                    for (int r = 0; r < C; ++r) max_slice = std::max<int64_t>(max_slice, sp[r + 1] - sp[r]);
            }
            if (C > 1) P.split = (const int32_t*)keep(upload(ctx, split.data(), split.size(), s));
            P.stage_cap = max_slice <= 1024 ? 1024 : 3072;
            P.queue = (int32_t*)keep(ctx->alloc(sizeof(int32_t) * 2));
            P.abort = P.queue + 1;
            P.xch_wait_ns = f->xch_wait_ns;
            check_cuda(cudaMemsetAsync(P.queue, 0, sizeof(int32_t) * 2, s), "batch queue");
            P.xg = (double*)keep(ctx->alloc(sizeof(double) * (size_t)K * G * n_groups));
            P.beta_g = (double*)keep(ctx->alloc(sizeof(double) * (size_t)J * G * n_groups));
            P.hd_g = (double*)keep(ctx->alloc(sizeof(double) * (size_t)J * G * n_groups));
            P.xjy_g = (double*)keep(ctx->alloc(sizeof(double) * (size_t)J * G * n_groups));
        } else {
            P.row = (double2*)keep(ctx->alloc(sizeof(double2) * 2 * (size_t)K * n));
            P.beta = (double*)keep(ctx->alloc(sizeof(double) * (size_t)J * n));
            P.hdelta = (double*)keep(ctx->alloc(sizeof(double) * (size_t)J * n));
            P.xjy = (double*)keep(ctx->alloc(sizeof(double) * (size_t)J * n));
        }
        // CCDB_BATCH_TRACE_FILE: per-column phase clocks of CTA 0 in one sweep
        // (CCDB_BATCH_TRACE_SWEEP, default 1) of the mixed engine, written as int64 [J][6]
        const char* trace_path = mixed ? std::getenv("CCDB_BATCH_TRACE_FILE") : nullptr;
        if (trace_path) {
            const char* sw = std::getenv("CCDB_BATCH_TRACE_SWEEP");
            P.trace_sweep = sw ? std::atoi(sw) : 1;
            P.trace = (long long*)keep(ctx->alloc(sizeof(long long) * 6 * (size_t)J));
            check_cuda(cudaMemsetAsync(P.trace, 0, sizeof(long long) * 6 * (size_t)J, s), "trace");
        }
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "event");
        check_cuda(cudaEventCreate(&e1), "event");
        check_cuda(cudaEventRecord(e0, s), "event");
        if (mixed) check_cuda(launch_batch_mixed(P, s), "batch sweep (mixed)");
        else check_cuda(launch_batch_sweep(P, s), "batch sweep");
        check_cuda(cudaEventRecord(e1, s), "event");
        check_cuda(f->ctx->wait(), "batch sync");  // the sweep is done before a copy is queued behind it
        std::vector<BatchResult> res(n);
        check_cuda(cudaMemcpyAsync(res.data(), P.results, sizeof(BatchResult) * n, cudaMemcpyDeviceToHost, s),
                   "results");
        int32_t aborted = 0;
        if (P.abort)
            check_cuda(cudaMemcpyAsync(&aborted, P.abort, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "abort word");
        std::vector<double> bg;
        if (beta_out && mixed) {
            bg.resize((size_t)J * G * n_groups);
            check_cuda(cudaMemcpyAsync(bg.data(), P.beta_g, sizeof(double) * bg.size(), cudaMemcpyDeviceToHost, s),
                       "beta");
        } else if (beta_out) {
            check_cuda(cudaMemcpyAsync(beta_out, P.beta, sizeof(double) * (size_t)J * n, cudaMemcpyDeviceToHost, s),
                       "beta");
        }
        check_cuda(f->ctx->wait(), "batch sync");
        if (trace_path) {
            std::vector<long long> tr(6 * (size_t)J);
            check_cuda(cudaMemcpy(tr.data(), P.trace, sizeof(long long) * tr.size(), cudaMemcpyDeviceToHost),
                       "trace copy");
            if (FILE* fh = std::fopen(trace_path, "wb")) {
                std::fwrite(tr.data(), sizeof(long long), tr.size(), fh);
                std::fclose(fh);
            }
        }
        if (beta_out && mixed)  // [group][J][G] -> [instance][J]
            for (int q = 0; q < n; ++q) {
                const int grp = q / G, gi = q % G, inst = order[q];
                for (int j = 0; j < J; ++j) beta_out[(size_t)inst * J + j] = bg[((size_t)grp * J + j) * G + gi];
            }
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (device_seconds) *device_seconds = ms * 1e-3;
        bool timed_out = aborted != 0;
        for (int i = 0; i < n; ++i) timed_out |= (res[i].flag == kBatchTimeoutFlag);
        if (timed_out)
            throw Error(CCDB_ERR_TIMEOUT, "batched fits: a bounded wait for the other CTAs of a cluster ran out");
        if (results)
            for (int i = 0; i < n; ++i) {
                results[i].return_flag = res[i].flag;
                results[i].iterations = res[i].iterations;
                results[i].log_likelihood = res[i].loglik;
                results[i].objective = res[i].objective;
                results[i].predictive_loglik = res[i].pred_loglik;
                results[i].steps = res[i].steps;
                results[i].updates = res[i].updates;
                results[i].update_entries = res[i].update_entries;
                results[i].gradient_entries = res[i].sweep_entries;
            }
    });
}

int ccdb_sweep_levels(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                      const uint8_t* fmt, const uint8_t* fixed, int32_t* level_out, int32_t* n_levels) {
    return guard([&] {
        require(col_start && fmt && level_out && n_levels && K > 0 && J > 0, "bad argument");
        std::vector<int64_t> entries(J);
        for (int j = 0; j < J; ++j)
            entries[j] = (fmt[j] == F_DENSE || fmt[j] == F_INTERCEPT) ? K : col_start[j + 1] - col_start[j];
        ScheduleParams sp;
        const Schedule s = build_schedule(K, J, col_start, rows, fmt, fixed, nullptr, K, entries.data(), sp);
        std::copy(s.level_of.begin(), s.level_of.end(), level_out);
        *n_levels = s.n_levels;
    });
}

}  // extern "C"
