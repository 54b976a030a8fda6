// postfit_host.cu -- host side of the calls on a fitted state outside the
// coordinate-descent loop: Fisher information, predictive log-likelihood on
// held-out weights, per-row predictions.
#include <algorithm>
#include <vector>

#include "engine.h"
#include "postfit.h"

namespace ccdb {
namespace {

// Device scratch of one call, released (stream-ordered) however the call ends.
struct Scratch {
    Context* ctx;
    std::vector<void*> held;
    explicit Scratch(Context* c) : ctx(c) {}
    template <typename T>
    T* get(size_t n) {
        void* p = ctx->alloc(sizeof(T) * std::max<size_t>(n, 1));
        held.push_back(p);
        return static_cast<T*>(p);
    }
    ~Scratch() {
        for (void* p : held) ctx->release(p);
    }
};

}  // namespace

// CyclicCoordinateDescent::computeFisherInformation(indices) (.cpp:1288-1299)
// over ModelSpecifics::computeFisherInformation (ModelSpecifics.hpp:1203-1337),
// on the current state.  The caller refuses weighted fits, as the reference does.
void Fit::fisher_information(const int32_t* idx, int n, double* out) {
    check_lazy();
    if (n <= 0) return;
    Scratch s(ctx);
    const bool grouped = group_engine();
    FisherParams P{};
    P.col_ptr = m->d_col_ptr;
    P.rows = m->d_rows;
    P.val_ptr = m->d_val_ptr;
    P.vals = m->d_vals;
    P.fmt = m->d_fmt;
    P.K = K;
    P.model = model;
    P.grouped = grouped ? 1 : 0;
    P.row = row;
    if (grouped) {
        P.xbe = cox.xbe;
        P.grp = cox.grp;
        P.gden = cox.denom;
        P.N = cox.N;
    }
    const size_t u_bytes = sizeof(double) * (size_t)K * kFisherSlots;
    const size_t c_bytes = grouped ? sizeof(double) * (size_t)(cox.N + 1) * kFisherSlots : 0;
    P.U = s.get<double>((size_t)K * kFisherSlots);
    P.C = grouped ? s.get<double>((size_t)(cox.N + 1) * kFisherSlots) : nullptr;
    int32_t* d_idx = s.get<int32_t>(n);
    check_cuda(cudaMemcpyAsync(d_idx, idx, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream), "fisher idx");
    P.idx = d_idx;
    P.n = n;
    P.out = s.get<double>((size_t)n * n);
    check_cuda(cudaEventRecord(ctx->fev[2], stream), "event");
    for (int p0 = 0; p0 < n; p0 += kFisherSlots) {
        const int ns = std::min(kFisherSlots, n - p0);
        int64_t most = 0;
        for (int t = 0; t < ns; ++t) most = std::max(most, m->entries(idx[p0 + t]));
        check_cuda(cudaMemsetAsync(P.U, 0, u_bytes, stream), "fisher U");
        if (grouped) check_cuda(cudaMemsetAsync(P.C, 0, c_bytes, stream), "fisher C");
        check_cuda(launch_fisher_scatter(P, p0, ns, most, stream), "fisher scatter");
        check_cuda(launch_fisher_gather(P, p0, ns, stream), "fisher gather");
        launches += 2;
    }
    check_cuda(cudaEventRecord(ctx->fev[3], stream), "event");
    check_cuda(cudaMemcpyAsync(out, P.out, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost, stream),
               "fisher copy");
    check_cuda(ctx->wait(), "fisher sync");
    float ms = 0.f;
    check_cuda(cudaEventElapsedTime(&ms, ctx->fev[2], ctx->fev[3]), "elapsed");
    last_call_seconds = ms * 1e-3;
}

// CyclicCoordinateDescent::getNewPredictiveLogLikelihood (.cpp:319-355): xBeta
// again from beta, the remaining statistics, then
// ModelSpecifics::getPredictiveLogLikelihood (ModelSpecifics.hpp:652-690),
// which for the Cox model regroups the rows with the held-out weights, takes the
// accumulated denominators under them, and restores the fit's own weights.
double Fit::predictive_log_likelihood(const double* weights) {
    xb_known = false;
    suff_known = false;
    check_lazy();
    if (!is_cox()) return predictive_sum(weights);
    const bool saved_weighted = weighted;
    std::vector<double> saved_w = w_h;
    auto restore = [&] {
        w_h = saved_w;
        weighted = saved_weighted;
        valid_weights = false;
        suff_known = false;
    };
    double ll = 0.0;
    try {
        w_h.assign(weights, weights + K);
        weighted = true;
        valid_weights = false;
        suff_known = false;
        check_lazy();
        ll = predictive_sum(weights);
    } catch (...) {
        restore();
        throw;
    }
    restore();
    check_lazy();
    check_cuda(ctx->wait(), "restore sync");
    return ll;
}

// Sum of logPredLikeContrib over the rows on the current state.
double Fit::predictive_sum(const double* weights) {
    Scratch s(ctx);
    const int nb = ctx->n_sm;
    double* d_w = s.get<double>(K);
    double* part = s.get<double>(nb);
    check_cuda(cudaMemcpyAsync(d_w, weights, sizeof(double) * K, cudaMemcpyHostToDevice, stream),
               "held-out weights");
    PredictParams P{};
    P.K = K;
    P.model = model;
    P.grouped = group_engine() ? 1 : 0;
    P.row = row;
    if (group_engine()) {
        P.xbe = cox.xbe;
        P.grp = cox.grp;
        P.gden = is_cox() ? cox.D : cox.denom;
        P.N = cox.N;
    }
    P.y = y;
    P.w = d_w;
    check_cuda(launch_predictive_loglik(P, part, nb, stream), "predictive loglik");
    ++launches;
    std::vector<double> h(nb);
    check_cuda(cudaMemcpyAsync(h.data(), part, sizeof(double) * nb, cudaMemcpyDeviceToHost, stream),
               "predictive copy");
    check_cuda(ctx->wait(), "predictive sync");
    double ll = 0.0;
    for (int b = 0; b < nb; ++b) ll += h[b];
    return ll;
}

// ModelSpecifics::getPredictiveEstimates (ModelSpecifics.hpp:692-705):
// predictEstimate of every row's xBeta into out (K entries).
void Fit::predictive_estimates(double* out) {
    check_lazy();
    Scratch s(ctx);
    double* d_out = s.get<double>(K);
    PredictParams P{};
    P.K = K;
    P.model = model;
    P.grouped = group_engine() ? 1 : 0;
    P.row = row;
    P.xbe = group_engine() ? cox.xbe : nullptr;
    check_cuda(launch_predictive_estimates(P, d_out, stream), "predictive estimates");
    ++launches;
    check_cuda(cudaMemcpyAsync(out, d_out, sizeof(double) * K, cudaMemcpyDeviceToHost, stream),
               "estimates copy");
    check_cuda(ctx->wait(), "estimates sync");
}

}  // namespace ccdb
