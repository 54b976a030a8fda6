// modes_host.cu -- host drivers of two mode-finding variants of
// CyclicCoordinateDescent::update: the MM algorithm (AlgorithmType::MM) and the
// KKT swindle (ModeFindingArguments::useKktSwindle).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "engine.h"
#include "mm.h"

namespace ccdb {
namespace {

double conv_objective(const double* t4, double ll_fixed, int conv) {
    const double ll = (t4[0] - t4[1]) + ll_fixed;
    if (conv == C_GRADIENT) return t4[2];
    if (conv == C_MITTAL) return ll;
    return ll + t4[3];
}

}  // namespace

// ModelSpecifics::computeMMGradientAndHessian (ModelSpecifics.hpp:776-889) on
// the current state, without a step.
void Fit::mm_gradient_hessian(const uint8_t* fixed_flags, double2* out) {
    check_lazy();
    uint8_t* d_fixed = nullptr;
    double2* d_gh = static_cast<double2*>(ctx->alloc(sizeof(double2) * std::max(1, J)));
    try {
        if (fixed_flags) {
            d_fixed = static_cast<uint8_t*>(ctx->alloc(std::max(1, J)));
            check_cuda(cudaMemcpyAsync(d_fixed, fixed_flags, J, cudaMemcpyHostToDevice, stream), "mm fixed");
        }
        MMParams P{};
        P.col_ptr = m->d_col_ptr;
        P.rows = m->d_rows;
        P.val_ptr = m->d_val_ptr;
        P.vals = m->d_vals;
        P.fmt = m->d_fmt;
        P.K = K;
        P.J = J;
        P.step = 0;
        P.xbe = cox.xbe;
        P.grp = cox.grp;
        P.nEv = cox.nEv;
        P.denom = cox.denom;
        P.xjy = xjy;
        P.fixed = d_fixed;
        P.beta = beta;
        P.ptype = ptype;
        P.pvar = pvar;
        P.gh = d_gh;
        check_cuda(launch_mm_gradient_hessian(P, stream), "mm gradient");
        ++launches;
        check_cuda(cudaMemcpyAsync(out, d_gh, sizeof(double2) * J, cudaMemcpyDeviceToHost, stream), "mm copy");
        check_cuda(ctx->wait(), "mm sync");
    } catch (...) {
        ctx->release(d_gh);
        ctx->release(d_fixed);
        throw;
    }
    ctx->release(d_gh);
    ctx->release(d_fixed);
}

// xBeta from the device beta as ModelSpecifics::computeXBeta(double* beta, bool)
// (ModelSpecifics.hpp:313-361) forms it: row by row over hX.transpose(), whose
// rows all take one format (CompressedDataMatrix.cpp:151-209), INDICATOR when
// some column is INDICATOR and none is DENSE.  That transpose keeps no values,
// so a SPARSE column then counts 1 for each of its non-zero entries; the
// product here follows the same rule (unit_values).
void Fit::compute_xbeta_transpose() {
    bool any_indicator = false, any_dense = false;
    for (int j = 0; j < J; ++j) {
        any_indicator |= m->fmt[j] == F_INDICATOR;
        any_dense |= m->fmt[j] == F_DENSE;
    }
    const_cast<Matrix*>(m)->ensure_csr(stream);
    check_cuda(launch_xbeta_csr(m->d_row_ptr, m->d_csr_col, m->d_csr_val, beta, K, xb_tmp, stream,
                                any_indicator && !any_dense),
               "xbeta (transpose)");
    ++launches;
    xb_pending = true;
    xb_known = true;
    suff_known = false;
}

// findMode with AlgorithmType::MM (CyclicCoordinateDescent.cpp:957-1001 and
// the MM check :1032-1048): per cycle, every free coordinate steps from one
// all-coordinate (g, h) (mmUpdateAllBeta, .cpp:1354-1391), xBeta is recomputed
// from beta (compute_xbeta_transpose) and the remaining statistics follow; a
// log posterior that decreases is the reference's "Non-increasing!" error.
// Convergence as findMode's performCheckConvergence.
void Fit::find_mode_mm(const ccdb_mode_args& a, int* flag, int* iters, double* obj) {
    uint8_t* d_fixed = static_cast<uint8_t*>(ctx->alloc(std::max(1, J)));
    double2* d_gh = static_cast<double2*>(ctx->alloc(sizeof(double2) * std::max(1, J)));
    try {
        check_cuda(cudaMemcpyAsync(d_fixed, fixed.data(), J, cudaMemcpyHostToDevice, stream), "mm fixed");
        const_cast<Matrix*>(m)->ensure_csr(stream);
        MMParams P{};
        P.col_ptr = m->d_col_ptr;
        P.rows = m->d_rows;
        P.val_ptr = m->d_val_ptr;
        P.vals = m->d_vals;
        P.fmt = m->d_fmt;
        P.K = K;
        P.J = J;
        P.step = 1;
        P.xjy = xjy;
        P.fixed = d_fixed;
        P.beta = beta;
        P.ptype = ptype;
        P.pvar = pvar;
        P.gh = d_gh;
        double t[4];
        objective_terms(t);
        double last = conv_objective(t, ll_fixed, a.convergence_type);
        double last_lp = -10E10;
        int iteration = 0;
        for (;;) {
            // the row/group tables may move when weights regroup: read them each cycle
            P.xbe = cox.xbe;
            P.grp = cox.grp;
            P.nEv = cox.nEv;
            P.denom = cox.denom;
            check_cuda(launch_mm_gradient_hessian(P, stream), "mm step");
            ++launches;
            compute_xbeta_transpose();
            remaining_statistics();
            download_beta();
            ++iteration;
            objective_terms(t);
            const double lp = (t[0] - t[1]) + ll_fixed + t[3];
            if (iteration > 1 && lp - last_lp < 0.0) throw Error(CCDB_ERR_INVALID, "Non-increasing!");
            last_lp = lp;
            const double cur = conv_objective(t, ll_fixed, a.convergence_type);
            double c;
            bool ill = false;
            if (cur != cur) {
                c = 0.0;
                ill = true;
            } else {
                c = std::fabs(cur - last) / (std::fabs(cur) + 1.0);
            }
            last = cur;
            if (a.tolerance > 0 && c < a.tolerance) {
                *flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
                break;
            }
            if (iteration == a.max_iterations) {
                *flag = R_MAX_ITERATIONS;
                break;
            }
        }
        *iters = iteration;
        *obj = last;
    } catch (...) {
        ctx->release(d_fixed);
        ctx->release(d_gh);
        throw;
    }
    ctx->release(d_fixed);
    ctx->release(d_gh);
}

// CyclicCoordinateDescent::kktSwindle (.cpp:636-807) with computeKktConditions
// (.cpp:809-826): Laplace columns start inactive at beta = 0 (the intercept
// and columns of other priors start active); findMode runs over the active
// set; the inactive columns' |gradient| is compared with their Laplace lambda
// (getKktBoundary, priors/CovariatePrior.h:235-238), and the violators move
// into the active set, largest first, until none is left.  The gradients of a
// pass come from batched launches against one state.
void Fit::kkt_swindle(const ccdb_mode_args& a, double bound, int* flag, int* iters, double* obj,
                      float* ms) {
    check_lazy();
    struct Score {
        int idx;
        double score;
        bool force;
    };
    bool has_intercept = false;
    for (int j = 0; j < J; ++j) has_intercept |= (m->fmt[j] == F_INTERCEPT);
    const int intercept = has_intercept ? (offset_col0 ? 1 : 0) : -1;
    const std::vector<uint8_t> exclude = fixed;
    std::vector<Score> active, inactive;
    for (int j = 0; j < J; ++j) {
        if (fixed[j]) continue;
        if (j == intercept || ptype_h[j] != 1) active.push_back({j, 0.0, true});
        else inactive.push_back({j, 0.0, false});
    }
    // The active set's findMode runs the resident sweep when the rows fit it,
    // else the fused dependency-level sweep, unless the caller chose a strategy:
    // its columns are the ones that violated their KKT condition, so most of them
    // move, and a fixed set that changes each pass costs one schedule build
    // instead of a launch per nonzero step.
    ccdb_mode_args inner = a;
    if (inner.strategy == CCDB_SWEEP_AUTO && !use_resident(inner)) inner.strategy = CCDB_SWEEP_LEVELS;
    auto lambda = [&](int j) { return std::sqrt(2.0 / pvar_h[j]); };
    auto meets = [&](const Score& s) { return s.score <= lambda(s.idx); };
    try {
        bool done = false;
        int count = 1;
        while (!done) {
            for (const Score& s : inactive)  // setBeta(i, 0.0): an incremental step of -beta
                if (beta_h[s.idx] != 0.0) update_xbeta(s.idx, 0.0 - beta_h[s.idx]);
            *flag = R_SUCCESS;
            if (!active.empty()) {
                std::fill(fixed.begin(), fixed.end(), uint8_t(1));
                for (const Score& s : active) fixed[s.idx] = 0;
                float t = 0.f;
                find_mode_once(inner, bound, flag, iters, obj, &t);
                *ms += t;
                if (beta_dirty_host) {
                    download_beta();
                    beta_dirty_host = false;
                }
            }
            if (inactive.empty() || *flag != R_SUCCESS) {
                done = true;
            } else if (count == a.max_iterations) {
                *flag = R_MAX_ITERATIONS;
                done = true;
            } else {
                std::vector<int32_t> cols(inactive.size());
                for (size_t q = 0; q < inactive.size(); ++q) cols[q] = inactive[q].idx;
                std::vector<double2> gh(cols.size());
                for (size_t q0 = 0; q0 < cols.size(); q0 += kBatchMax) {
                    const int nb = (int)std::min<size_t>(kBatchMax, cols.size() - q0);
                    gh_batch(cols.data() + q0, nb, gh.data() + q0);
                }
                for (size_t q = 0; q < inactive.size(); ++q) inactive[q].score = std::fabs(gh[q].x);
                std::stable_sort(inactive.begin(), inactive.end(), [](const Score& l, const Score& r) {
                    return (l.force == r.force) ? (r.score < l.score) : l.force;
                });
                if (std::all_of(inactive.begin(), inactive.end(), meets)) {
                    done = true;
                } else {
                    size_t moved = 0;
                    while (moved < inactive.size() && !meets(inactive[moved])) {
                        active.push_back(inactive[moved]);
                        ++moved;
                    }
                    inactive.erase(inactive.begin(), inactive.begin() + moved);
                }
            }
            ++count;
        }
    } catch (...) {
        fixed = exclude;
        throw;
    }
    fixed = exclude;  // restore fixBeta
}

}  // namespace ccdb
