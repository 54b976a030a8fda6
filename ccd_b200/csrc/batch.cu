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

constexpr int kBT = 512;
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

// One column of the sweep with its entries staged in shared memory (row ids,
// values) and the gathered row state kept in registers between the gradient
// and the update.  Columns longer than kBT * kBE entries take the loop path.
constexpr int kBE = 6;  // staged entries per thread: columns up to 3,072 entries

struct ColStage {
    int32_t k[kBT * kBE];
    double x[kBT * kBE];
};

__device__ __forceinline__ void stage_column(const BatchParams& P, const double2* row, int j,
                                             ColStage& st, int64_t n) {
    const uint8_t f = P.fmt[j];
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    for (int p = threadIdx.x; p < n; p += kBT) {
        const int32_t k = has_rows ? __ldg(P.rows + cb + p) : p;
        st.k[p] = k;
        st.x[p] = has_vals ? __ldg(P.vals + vb + p) : 1.0;
        // L2 is the point of coherence: the lines are current when read later
        asm volatile("prefetch.global.L2 [%0];" ::"l"(row + 2 * (int64_t)k));
    }
}

template <int MODEL>
__global__ void __launch_bounds__(kBT, 1) batch_sweep_kernel(BatchParams P) {
    __shared__ double2 s_red2[kBW];
    __shared__ double4 s_red4[kBW];
    __shared__ double s_delta;
    __shared__ int32_t s_done;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    ColStage* s_stage = reinterpret_cast<ColStage*>(s_dyn);  // two stages (double buffer)
    const int inst = P.order ? P.order[blockIdx.x] : blockIdx.x;
    if (blockIdx.x >= P.n_inst) return;
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
        const double w = (P.row_fold && hold >= 0 && P.row_fold[k] == hold) ? 0.0 : 1.0;
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

    auto col_len = [&](int j) -> int64_t {
        const uint8_t f = P.fmt[j];
        return (f == F_DENSE || f == F_INTERCEPT) ? P.K : P.col_ptr[j + 1] - P.col_ptr[j];
    };
    const int j0 = P.offset_vals ? 1 : 0;
    constexpr int64_t kStageMax = kBT * kBE;

    double ll = 0.0, lp = 0.0;
    double last = objective(ll, lp);
    int iteration = 0, flag = R_FAIL;
    long long steps = 0, updates = 0, upd_entries = 0, gh_entries = 0;
    for (int it = 0; it < P.max_iter; ++it) {
        int buf = 0;
        if (j0 < P.J && col_len(j0) <= kStageMax) stage_column(P, row, j0, s_stage[0], col_len(j0));
        __syncthreads();
        for (int j = j0; j < P.J; ++j) {
            const uint8_t f = P.fmt[j];
            const int64_t n = col_len(j);
            const bool staged = n <= kStageMax;
            // metadata of this column (thread 0) and staging of the next one
            double m_beta = 0.0, m_hd = 0.0, m_xjy = 0.0;
            if (threadIdx.x == 0) {
                m_beta = beta[j];
                m_hd = hd[j];
                m_xjy = xjy[j];
            }
            if (j + 1 < P.J && col_len(j + 1) <= kStageMax)
                stage_column(P, row, j + 1, s_stage[buf ^ 1], col_len(j + 1));
            double g = 0.0, h = 0.0;
            double2 A[kBE];
            double Dn[kBE];
            const ColStage& st = s_stage[buf];
            const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
            if (staged) {
                double Wt[kBE];
#pragma unroll
                for (int i = 0; i < kBE; ++i) {
                    const int p = threadIdx.x + i * kBT;
                    if (p < n) {
                        const int64_t k = st.k[p];
                        A[i] = row[2 * k];
                        const double2 b = row[2 * k + 1];
                        Dn[i] = b.x;
                        Wt[i] = b.y;
                    }
                }
#pragma unroll
                for (int i = 0; i < kBE; ++i) {
                    const int p = threadIdx.x + i * kBT;
                    if (p >= n) continue;
                    const double x = st.x[p];
                    const double n1 = A[i].y * x;
                    if (MODEL == M_LOGISTIC) {
                        const double gg = n1 / Dn[i];
                        g += Wt[i] * gg;
                        if (ind) h += Wt[i] * gg * (1.0 - gg);
                        else h += Wt[i] * ((n1 * x) / Dn[i] - gg * gg);
                    } else {
                        if (ind) {
                            const double v = Wt[i] * n1;
                            g += v;
                            h += v;
                        } else {
                            g += Wt[i] * n1;
                            h += Wt[i] * (n1 * x);
                        }
                    }
                }
            } else {
                switch (f) {
                case F_INDICATOR: b_gh<MODEL, F_INDICATOR>(P, row, j, n, g, h); break;
                case F_SPARSE: b_gh<MODEL, F_SPARSE>(P, row, j, n, g, h); break;
                case F_DENSE: b_gh<MODEL, F_DENSE>(P, row, j, n, g, h); break;
                default: b_gh<MODEL, F_INTERCEPT>(P, row, j, n, g, h); break;
                }
            }
            const double2 s = block_sum2<kBW>(make_double2(g, h), s_red2);
            if (threadIdx.x == 0) {
                double G = 0.0, H = 0.0;
                if (n > 0) {
                    G = s.x - m_xjy;
                    H = s.y;
                }
                const int pt = P.ptype[j];
                double d = newton_prior_delta(G, H, m_beta, pt, pt == 0 ? 1.0 : var);
                double b = m_hd;
                d = apply_bounds(d, b);
                hd[j] = b;
                if (d != 0.0) {
                    beta[j] = m_beta + d;
                    ++updates;
                    upd_entries += n;
                }
                ++steps;
                gh_entries += n;
                s_delta = d;
            }
            __syncthreads();
            const double d = s_delta;
            if (d != 0.0) {
                if (staged) {
#pragma unroll
                    for (int i = 0; i < kBE; ++i) {
                        const int p = threadIdx.x + i * kBT;
                        if (p >= n) continue;
                        const int64_t k = st.k[p];
                        const double xb = A[i].x + d * st.x[p];
                        const double en = exp(xb);
                        row[2 * k] = make_double2(xb, en);
                        reinterpret_cast<double*>(row + 2 * k + 1)[0] = Dn[i] + (en - A[i].y);
                    }
                } else {
                    switch (f) {
                    case F_INDICATOR: b_update<F_INDICATOR>(P, row, j, n, d); break;
                    case F_SPARSE: b_update<F_SPARSE>(P, row, j, n, d); break;
                    case F_DENSE: b_update<F_DENSE>(P, row, j, n, d); break;
                    default: b_update<F_INTERCEPT>(P, row, j, n, d); break;
                    }
                }
            }
            __syncthreads();
            buf ^= 1;
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
        r.steps = steps;
        r.updates = updates;
        r.update_entries = upd_entries;
        r.sweep_entries = gh_entries;
        P.results[inst] = r;
    }
}

}  // namespace

cudaError_t launch_batch_sweep(const BatchParams& P, cudaStream_t stream) {
    const size_t smem = sizeof(ColStage) * 2;
    static std::atomic<uint64_t> done{0};
    cudaError_t e = once_per_device(done, [&] {
        cudaError_t r = cudaFuncSetAttribute(batch_sweep_kernel<M_LOGISTIC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (r != cudaSuccess) return r;
        return cudaFuncSetAttribute(batch_sweep_kernel<M_POISSON>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem);
    });
    if (e != cudaSuccess) return e;
    if (P.model == M_LOGISTIC) batch_sweep_kernel<M_LOGISTIC><<<P.n_inst, kBT, smem, stream>>>(P);
    else batch_sweep_kernel<M_POISSON><<<P.n_inst, kBT, smem, stream>>>(P);
    return cudaGetLastError();
}

}  // namespace ccdb
