// batch.cu -- many fits over one shared CompressedDataMatrix in one launch
// (the cross-validation grid: folds x prior variances).
//
// Each CTA owns one instance: its row weights (0 on the held-out fold, as
// CrossValidationSelector::getWeights sets them, drivers/CrossValidationSelector.cpp:72-130),
// its prior variance, coefficients, bounds and its own row state
// {xBeta, exp(xBeta)}, {denominator, weight} (32 bytes per row, the plain
// fit's layout).  A CTA runs the sequential coordinate-descent sweep of its
// instance exactly as a standalone fit would -- same visiting order, same
// per-column step -- with no synchronisation with other CTAs: the
// instances' latency chains overlap, and the memory system sees hundreds of
// independent gathers in flight.  Every instance starts cold (beta = 0) and
// stops on its own convergence test.  After convergence each instance also
// reports the predictive log-likelihood of its held-out rows
// (getPredictiveLogLikelihood, ModelSpecifics.hpp:652-690), the quantity the
// CV driver averages over folds (AbstractCrossValidationDriver.cpp:131-240).
#include <cstdint>

#include "batch.h"
#include "common.cuh"

namespace ccdb {

namespace {

constexpr int kBT = 256;
constexpr int kBW = kBT / 32;

template <int FMT>
__device__ __forceinline__ int64_t b_row(const int32_t* rows, int64_t cb, int64_t p) {
    if (FMT == F_SPARSE || FMT == F_INDICATOR) return (int64_t)__ldg(rows + cb + p);
    return p;
}
template <int FMT>
__device__ __forceinline__ double b_val(const double* vals, int64_t vb, int64_t p) {
    if (FMT == F_SPARSE || FMT == F_DENSE) return __ldg(vals + vb + p);
    return 1.0;
}

// Per-entry contributions: Logistic / Poisson incrementGradientAndHessian
// (ModelSpecifics.h:541-568, :1509-1543), weighted by the instance's row weight.
template <int MODEL, int FMT>
__device__ __forceinline__ void b_gh(const BatchParams& P, const double2* row, int j, int64_t n,
                                     double& g, double& h) {
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    constexpr bool ind = (FMT == F_INDICATOR || FMT == F_INTERCEPT);
#pragma unroll 4
    for (int64_t p = threadIdx.x; p < n; p += kBT) {
        const int64_t k = b_row<FMT>(P.rows, cb, p);
        const double x = b_val<FMT>(P.vals, vb, p);
        const double2 a = row[2 * k];
        const double2 b = row[2 * k + 1];
        const double n1 = a.y * x;
        if (MODEL == M_LOGISTIC) {
            const double gg = n1 / b.x;
            g += b.y * gg;
            if (ind) h += b.y * gg * (1.0 - gg);
            else h += b.y * ((n1 * x) / b.x - gg * gg);
        } else {
            if (ind) {
                const double v = b.y * n1;
                g += v;
                h += v;
            } else {
                g += b.y * n1;
                h += b.y * (n1 * x);
            }
        }
    }
}

template <int FMT>
__device__ __forceinline__ void b_update(const BatchParams& P, double2* row, int j, int64_t n,
                                         double delta) {
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
#pragma unroll 4
    for (int64_t p = threadIdx.x; p < n; p += kBT) {
        const int64_t k = b_row<FMT>(P.rows, cb, p);
        const double x = b_val<FMT>(P.vals, vb, p);
        const double2 a = row[2 * k];
        const double dn0 = row[2 * k + 1].x;
        const double xb = a.x + delta * x;
        const double en = exp(xb);
        row[2 * k] = make_double2(xb, en);
        reinterpret_cast<double*>(row + 2 * k + 1)[0] = dn0 + (en - a.y);
    }
}

// XjY of the instance (ModelSpecifics.hpp:486-524, CV weights): x * y * w per entry.
template <int FMT>
__device__ __forceinline__ double b_xjy(const BatchParams& P, const double2* row, int j, int64_t n) {
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    double s = 0.0;
    for (int64_t p = threadIdx.x; p < n; p += kBT) {
        const int64_t k = b_row<FMT>(P.rows, cb, p);
        const double x = b_val<FMT>(P.vals, vb, p);
        s += x * P.y[k] * row[2 * k + 1].y;
    }
    return s;
}

template <int MODEL>
__global__ void __launch_bounds__(kBT, 2) batch_sweep_kernel(BatchParams P) {
    __shared__ double2 s_red2[kBW];
    __shared__ double4 s_red4[kBW];
    __shared__ double s_delta;
    __shared__ int32_t s_done;
    const int inst = blockIdx.x;
    if (inst >= P.n_inst) return;
    double2* row = P.row + (size_t)inst * 2 * P.K;
    double* beta = P.beta + (size_t)inst * P.J;
    double* hd = P.hdelta + (size_t)inst * P.J;
    double* xjy = P.xjy + (size_t)inst * P.J;
    const int hold = P.holdout ? P.holdout[inst] : -1;
    const double var = P.variance[inst];
    const double null_denom = (MODEL == M_LOGISTIC) ? 1.0 : 0.0;

    // state: xBeta from the offset (if any), exp, denominator, weight
    for (int64_t k = threadIdx.x; k < P.K; k += kBT) {
        const double xb = P.offset_vals ? 0.0 + 1.0 * P.offset_vals[k] : 0.0;
        const double e = exp(xb);
        const double w = (P.row_fold && P.row_fold[k] == hold) ? 0.0 : 1.0;
        row[2 * k] = make_double2(xb, e);
        row[2 * k + 1] = make_double2(null_denom + e, w);
    }
    for (int j = threadIdx.x; j < P.J; j += kBT) {
        beta[j] = (P.offset_vals && j == 0) ? 1.0 : 0.0;
        hd[j] = P.initial_bound;
    }
    __syncthreads();
    for (int j = 0; j < P.J; ++j) {
        const uint8_t f = P.fmt[j];
        const int64_t n = (f == F_DENSE || f == F_INTERCEPT) ? P.K : P.col_ptr[j + 1] - P.col_ptr[j];
        double s;
        switch (f) {
        case F_INDICATOR: s = b_xjy<F_INDICATOR>(P, row, j, n); break;
        case F_SPARSE: s = b_xjy<F_SPARSE>(P, row, j, n); break;
        case F_DENSE: s = b_xjy<F_DENSE>(P, row, j, n); break;
        default: s = b_xjy<F_INTERCEPT>(P, row, j, n); break;
        }
        const double2 t = block_sum2<kBW>(make_double2(s, 0.0), s_red2);
        if (threadIdx.x == 0) xjy[j] = t.x;
    }
    __syncthreads();

    auto objective = [&](double& ll_out, double& lp_out) -> double {
        double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int64_t k = threadIdx.x; k < P.K; k += kBT) {
            const double2 a = row[2 * k];
            const double2 dw = row[2 * k + 1];
            const double yk = P.y[k];
            acc.x += (double)((int)yk) * a.x * dw.y;
            if (MODEL == M_LOGISTIC) acc.y += dw.y * log(dw.x);
            else acc.y += dw.y * dw.x;
            acc.z += a.x * yk * dw.y;
        }
        for (int j = threadIdx.x; j < P.J; j += kBT) {
            const int pt = P.ptype[j];
            acc.w += log_prior_one(beta[j], pt, pt == 0 ? 1.0 : var);
        }
        const double4 t = block_sum4<kBW>(acc, s_red4);
        double fixed = 0.0;
        if (MODEL == M_POISSON && P.ll_fixed) fixed = P.ll_fixed[inst];
        ll_out = (t.x - t.y) + fixed;
        lp_out = t.w;
        if (P.conv == C_GRADIENT) return t.z;
        if (P.conv == C_MITTAL) return ll_out;
        return ll_out + t.w;
    };

    double ll = 0.0, lp = 0.0;
    double last = objective(ll, lp);
    int iteration = 0, flag = R_FAIL;
    for (int it = 0; it < P.max_iter; ++it) {
        for (int j = (P.offset_vals ? 1 : 0); j < P.J; ++j) {
            const uint8_t f = P.fmt[j];
            const int64_t n = (f == F_DENSE || f == F_INTERCEPT) ? P.K : P.col_ptr[j + 1] - P.col_ptr[j];
            double g = 0.0, h = 0.0;
            switch (f) {
            case F_INDICATOR: b_gh<MODEL, F_INDICATOR>(P, row, j, n, g, h); break;
            case F_SPARSE: b_gh<MODEL, F_SPARSE>(P, row, j, n, g, h); break;
            case F_DENSE: b_gh<MODEL, F_DENSE>(P, row, j, n, g, h); break;
            default: b_gh<MODEL, F_INTERCEPT>(P, row, j, n, g, h); break;
            }
            const double2 s = block_sum2<kBW>(make_double2(g, h), s_red2);
            if (threadIdx.x == 0) {
                double G = 0.0, H = 0.0;
                if (n > 0) {
                    G = s.x - xjy[j];
                    H = s.y;
                }
                const int pt = P.ptype[j];
                double d = newton_prior_delta(G, H, beta[j], pt, pt == 0 ? 1.0 : var);
                double b = hd[j];
                d = apply_bounds(d, b);
                hd[j] = b;
                if (d != 0.0) beta[j] = beta[j] + d;
                s_delta = d;
            }
            __syncthreads();
            const double d = s_delta;
            if (d != 0.0) {
                switch (f) {
                case F_INDICATOR: b_update<F_INDICATOR>(P, row, j, n, d); break;
                case F_SPARSE: b_update<F_SPARSE>(P, row, j, n, d); break;
                case F_DENSE: b_update<F_DENSE>(P, row, j, n, d); break;
                default: b_update<F_INTERCEPT>(P, row, j, n, d); break;
                }
                __syncthreads();
            }
        }
        iteration = it + 1;
        const double cur = objective(ll, lp);
        if (threadIdx.x == 0) {
            double conv;
            bool ill = false;
            if (cur != cur) {
                conv = 0.0;
                ill = true;
            } else {
                conv = fabs(cur - last) / (fabs(cur) + 1.0);
            }
            int done = 0;
            if (P.tol > 0 && conv < P.tol) {
                flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
                done = 1;
            } else if (iteration == P.max_iter) {
                flag = R_MAX_ITERATIONS;
                done = 1;
            }
            s_done = done;
        }
        last = cur;
        __syncthreads();
        if (s_done) break;
    }
    // predictive log-likelihood of the held-out rows (weights 1 - w)
    double pred = 0.0;
    for (int64_t k = threadIdx.x; k < P.K; k += kBT) {
        const double2 a = row[2 * k];
        const double2 dw = row[2 * k + 1];
        const double wo = 1.0 - dw.y;
        if (MODEL == M_LOGISTIC) pred += P.y[k] * wo * (a.x - log(dw.x));
        else pred += (P.y[k] * a.x - exp(a.x)) * wo;
    }
    const double2 pt = block_sum2<kBW>(make_double2(pred, 0.0), s_red2);
    if (threadIdx.x == 0) {
        BatchResult r;
        r.flag = flag;
        r.iterations = iteration;
        r.loglik = ll;
        r.objective = last;
        r.pred_loglik = pt.x;
        P.results[inst] = r;
    }
}

}  // namespace

cudaError_t launch_batch_sweep(const BatchParams& P, cudaStream_t stream) {
    if (P.model == M_LOGISTIC) batch_sweep_kernel<M_LOGISTIC><<<P.n_inst, kBT, 0, stream>>>(P);
    else batch_sweep_kernel<M_POISSON><<<P.n_inst, kBT, 0, stream>>>(P);
    return cudaGetLastError();
}

}  // namespace ccdb
