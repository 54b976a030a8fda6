// batch_common.cuh -- pieces shared by the two mixed-precision batched
// kernels (batch_mixed.cu: thread gathers; batch_tma.cu: TMA gathers).
#pragma once

#include <cstdint>

#include "batch.h"
#include "common.cuh"
#include "step.h"

namespace ccdb {
namespace bm {

constexpr int kMT = 512;           // threads per CTA
constexpr int kMW = kMT / 32;      // warps per CTA
constexpr int kStageN = 3072;      // entries of a staged column; longer columns stream

struct MStage {
    int32_t k[kStageN];  // keys: row | fold code << 24
    double x[kStageN];
};

struct MMeta {
    int64_t cb, vb;
    int32_t n, fmt;
};

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// all but the most recent group complete
__device__ __forceinline__ void cp_async_wait_but_last() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Knuth's TwoSum: s + c carries the running sum with the rounding error of
// every addition kept in c.
__device__ __forceinline__ void two_sum(float& s, float& c, float v) {
    const float t = s + v;
    const float bp = t - s;
    c += (s - (t - bp)) + (v - bp);
    s = t;
}

__device__ __forceinline__ MMeta load_meta(const BatchParams& P, int j) {
    MMeta m;
    const int f = P.fmt[j];
    m.fmt = f;
    m.cb = P.col_ptr[j];
    m.vb = P.val_ptr[j];
    m.n = (f == F_DENSE || f == F_INTERCEPT) ? (int32_t)P.K : (int32_t)(P.col_ptr[j + 1] - m.cb);
    return m;
}

__device__ __forceinline__ bool stageable(const MMeta& m) {
    return (m.fmt == F_SPARSE || m.fmt == F_INDICATOR) && m.n <= kStageN;
}

// FP32 gradient / Hessian terms of one entry with value x at xBeta xb.
// Logistic: t = sigma(xb), u = 1 - t, evaluated as 1/(1+a) and a/(1+a) with
// a = exp(-|xb|) so that neither overflows; g = t x, h = t u x^2.
// Poisson: e = exp(xb); g = e x, h = e x^2.
template <int MODEL>
__device__ __forceinline__ void entry_terms(double xb, float x, bool ind, float& gt, float& ht) {
    const float xf = (float)xb;
    if (MODEL == M_LOGISTIC) {
        const float a = expf(-fabsf(xf));
        const float r = __frcp_rn(1.0f + a);
        const float ar = a * r;
        const float t = (xf >= 0.0f) ? r : ar;
        const float u = (xf >= 0.0f) ? ar : r;
        gt = ind ? t : t * x;
        ht = ind ? t * u : (t * u) * (x * x);
    } else {
        const float e = expf(xf);
        gt = ind ? e : e * x;
        ht = ind ? e : e * (x * x);
    }
}

// Sum of v over the kMT / G threads of each instance of the group (threads with
// the same threadIdx % G): butterfly within the warp, then a fixed-order sum of
// the per-warp values.  One barrier; `red` alternates between two buffers so
// that consecutive calls need no second barrier.  Every thread of the instance
// gets the same value.
// group_sum whose barrier also returns whether any thread of the CTA passed
// `pred` true (the barrier is __syncthreads_or).
template <int G, int NV>
__device__ __forceinline__ bool group_sum_or(double (&v)[NV], double (*red)[kMW][4][NV], int& rb, bool pred) {
#pragma unroll
    for (int off = G; off < 32; off <<= 1)
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = threadIdx.x % G;
    if (lane < G)
#pragma unroll
        for (int q = 0; q < NV; ++q) red[rb][wid][lane][q] = v[q];
    const bool any = __syncthreads_or(pred);
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kMW; ++w) t += red[rb][w][g][q];
        v[q] = t;
    }
    rb ^= 1;
    return any;
}

template <int G, int NV>
__device__ __forceinline__ void group_sum(double (&v)[NV], double (*red)[kMW][4][NV], int& rb) {
#pragma unroll
    for (int off = G; off < 32; off <<= 1)
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = threadIdx.x % G;
    if (lane < G)
#pragma unroll
        for (int q = 0; q < NV; ++q) red[rb][wid][lane][q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kMW; ++w) t += red[rb][w][g][q];
        v[q] = t;
    }
    rb ^= 1;
}

// One thread's view of its instance: which instance of the group it serves,
// that instance's slices of the group arrays, prior and held-out fold.
template <int G>
struct Inst {
    static constexpr int S = kMT / G;  // threads per instance
    int grp, g, sl, inst, hold, J;
    bool exists;
    int64_t K;
    double *X, *Bt, *Hd, *Xy;
    double var, lambda;
    const int32_t* fold;  // NULL when the instance holds nothing out

    __device__ explicit Inst(const BatchParams& P) {
        grp = blockIdx.x;
        g = threadIdx.x % G;
        sl = threadIdx.x / G;
        const int pos = grp * G + g;
        exists = pos < P.n_inst;
        inst = exists ? (P.order ? P.order[pos] : pos) : -1;
        K = P.K;
        J = P.J;
        X = P.xg + (size_t)grp * (size_t)K * G;
        Bt = P.beta_g + (size_t)grp * (size_t)J * G;
        Hd = P.hd_g + (size_t)grp * (size_t)J * G;
        Xy = P.xjy_g + (size_t)grp * (size_t)J * G;
        hold = (exists && P.holdout) ? P.holdout[inst] : -1;
        var = exists ? P.variance[inst] : 1.0;
        lambda = sqrt(2.0 / var);
        fold = (hold >= 0) ? P.row_fold : nullptr;  // a negative holdout holds out nothing
    }
    __device__ bool held(int64_t k) const { return fold && __ldg(fold + k) == hold; }
};

// Initial state: xBeta from the offset column (computeXBeta with beta_0 = 1),
// coefficients, bounds, and each instance's XjY (ModelSpecifics.hpp:486-524).
template <int G>
__device__ void inst_setup(const BatchParams& P, const Inst<G>& I, double (*red2)[kMW][4][2], int& rb2) {
    constexpr int S = Inst<G>::S;
    for (int64_t k = I.sl; k < I.K; k += S)
        I.X[k * G + I.g] = P.offset_vals ? 0.0 + 1.0 * P.offset_vals[k] : 0.0;
    for (int j = I.sl; j < I.J; j += S) {
        I.Bt[(size_t)j * G + I.g] = (P.offset_vals && j == 0) ? 1.0 : 0.0;
        I.Hd[(size_t)j * G + I.g] = P.initial_bound;
    }
    for (int j = 0; j < I.J; ++j) {
        const MMeta m = load_meta(P, j);
        const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
        const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
        double acc[2] = {0.0, 0.0};
        if (I.exists)
            for (int64_t p = I.sl; p < m.n; p += S) {
                const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : p;
                const double x = has_vals ? __ldg(P.vals + m.vb + p) : 1.0;
                acc[0] += x * P.y[k] * (I.held(k) ? 0.0 : 1.0);
            }
        group_sum<G, 2>(acc, red2, rb2);
        if (I.sl == 0) I.Xy[(size_t)j * G + I.g] = acc[0];
    }
    __syncthreads();
}

// Per-sweep objective in FP64 (getLogLikelihood, ModelSpecifics.hpp:605-650;
// the gradient objective, :103-120); the LL terms only when they are needed.
template <int MODEL, int G>
__device__ double inst_objective(const BatchParams& P, const Inst<G>& I, bool active, bool need_ll,
                                 double& ll_out, double (*red4)[kMW][4][4], int& rb4) {
    constexpr int S = Inst<G>::S;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (active)
        for (int64_t k = I.sl; k < I.K; k += S) {
            const double xb = I.X[k * G + I.g];
            const double w = I.held(k) ? 0.0 : 1.0;
            const double yk = P.y[k];
            acc[2] += xb * yk * w;
            if (need_ll) {
                acc[0] += (double)((int)yk) * xb * w;
                const double e = exp(xb);
                if (MODEL == M_LOGISTIC) acc[1] += w * log(1.0 + e);
                else acc[1] += w * e;
            }
        }
    if (active && P.conv == C_LANGE)
        for (int j = I.sl; j < I.J; j += S) {
            const int pt = P.ptype[j];
            acc[3] += log_prior_one(I.Bt[(size_t)j * G + I.g], pt, pt == 0 ? 1.0 : I.var);
        }
    group_sum<G, 4>(acc, red4, rb4);
    const double fixed = (MODEL == M_POISSON && P.ll_fixed && I.exists) ? P.ll_fixed[I.inst] : 0.0;
    ll_out = (acc[0] - acc[1]) + fixed;
    if (P.conv == C_GRADIENT) return acc[2];
    if (P.conv == C_MITTAL) return ll_out;
    return ll_out + acc[3];
}

struct InstCounters {
    long long steps = 0, updates = 0, upd_entries = 0, gh_entries = 0;
};

// The coordinate step of one instance (ccdUpdateBeta + applyBounds), computed
// identically by every thread of the instance; thread 0 of the instance stores
// the bound and coefficient.  An empty column gives (0, 0)
// (ModelSpecifics.hpp:720-723).
template <int G>
__device__ __forceinline__ double inst_step(const Inst<G>& I, int j, int n, double gsum, double hsum,
                                            double b0, double hd0, double xjy0, int pt, InstCounters& c) {
    double Gv = 0.0, Hv = 0.0;
    if (n > 0) {
        Gv = gsum - xjy0;
        Hv = hsum;
    }
    double d = newton_prior_delta_l(Gv, Hv, b0, pt, pt == 0 ? 1.0 : I.var, I.lambda);
    double bnd = hd0;
    d = apply_bounds(d, bnd);
    if (I.sl == 0) {
        I.Hd[(size_t)j * G + I.g] = bnd;
        if (d != 0.0) {
            I.Bt[(size_t)j * G + I.g] = b0 + d;
            ++c.updates;
            c.upd_entries += n;
        }
        ++c.steps;
        c.gh_entries += n;
    }
    return d;
}

// Convergence test after a sweep (CyclicCoordinateDescent.cpp:541-558, 839-906).
__device__ __forceinline__ void inst_converge(const BatchParams& P, double cur, double& last, int iteration,
                                              int& flag, bool& active) {
    const bool ill = (cur != cur);
    const double conv = ill ? 0.0 : fabs(cur - last) / (fabs(cur) + 1.0);
    if (P.tol > 0 && conv < P.tol) {
        flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
        active = false;
    } else if (iteration == P.max_iter) {
        flag = R_MAX_ITERATIONS;
        active = false;
    }
    last = cur;
}

// Training log-likelihood and the predictive log-likelihood of the held-out
// rows (getPredictiveLogLikelihood, ModelSpecifics.hpp:652-690), FP64; result.
template <int MODEL, int G>
__device__ void inst_finish(const BatchParams& P, const Inst<G>& I, int flag, int iteration, double last,
                            const InstCounters& c, double (*red4)[kMW][4][4], int& rb4) {
    constexpr int S = Inst<G>::S;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (I.exists)
        for (int64_t k = I.sl; k < I.K; k += S) {
            const double xb = I.X[k * G + I.g];
            const double w = I.held(k) ? 0.0 : 1.0, wo = 1.0 - w;
            const double yk = P.y[k];
            const double e = exp(xb);
            acc[0] += (double)((int)yk) * xb * w;
            if (MODEL == M_LOGISTIC) {
                const double lg = log(1.0 + e);
                acc[1] += w * lg;
                acc[2] += yk * wo * (xb - lg);
            } else {
                acc[1] += w * e;
                acc[2] += (yk * xb - e) * wo;
            }
        }
    group_sum<G, 4>(acc, red4, rb4);
    if (I.exists && I.sl == 0) {
        const double fixed = (MODEL == M_POISSON && P.ll_fixed) ? P.ll_fixed[I.inst] : 0.0;
        BatchResult r;
        r.flag = flag;
        r.iterations = iteration;
        r.loglik = (acc[0] - acc[1]) + fixed;
        r.objective = last;
        r.pred_loglik = acc[2];
        r.steps = c.steps;
        r.updates = c.updates;
        r.update_entries = c.upd_entries;
        r.sweep_entries = c.gh_entries;
        P.results[I.inst] = r;
    }
}

}  // namespace bm
}  // namespace ccdb
