// batch_mixed.cu -- the cross-validation grid in mixed precision, with the
// instances of a CTA stepping through the columns in lockstep.
//
// A CTA runs a group of G instances (G = 1, 2 or 4; consecutive in the launch
// order, which sorts by prior variance, so a group's instances need similar
// numbers of sweeps).  Every instance keeps its own weights, coefficients,
// bounds and xBeta and runs the sequential coordinate-descent sweep of a
// standalone fit -- same visiting order, same per-column step -- but the G
// instances visit column j together.  Their row state is interleaved
// instance-minor (xBeta[row][G], FP64), so a gathered row is one 32-byte
// DRAM sector for the whole group at G = 4 instead of one sector per instance,
// and the column's row ids are read once per group.  Each entry's row id
// carries the row's fold in its top bits (row | fold << 24), so the instance
// weight (0 on the held-out fold) costs no extra load.
//
// Precision: the row state xBeta and every coefficient stay FP64.  exp(xBeta),
// the logistic ratio and the per-entry gradient/Hessian terms run in FP32, each
// thread sums its terms with a compensated (two-sum) accumulator, and the
// per-column reduction across threads, the Newton step with its prior and
// bound, the convergence objective and the reported log-likelihoods are FP64.
// The per-entry terms follow Logistic / Poisson incrementGradientAndHessian
// (ModelSpecifics.h:541-568, :1509-1543); the step follows ccdUpdateBeta +
// applyBounds (CyclicCoordinateDescent.cpp:1394-1413, :1503-1520).
//
// Pipeline per column j (one CTA, two barriers), deep enough that no DRAM
// round trip of a later column falls on column j's critical path:
//   * the keys (and values) of column j+4 are copied into shared memory with
//     cp.async (completion is awaited two columns later);
//   * the row state of column j+2 is prefetched into L2;
//   * the coefficient, bound and XjY of column j+1 are loaded into registers;
//   * column j's state is gathered into registers, reduced, stepped, and the
//     updated xBeta written back from the same registers.
#include <cstdint>

#include "batch.h"
#include "common.cuh"
#include "step.h"

namespace ccdb {

namespace {

constexpr int kMT = 512;           // threads per CTA
constexpr int kMW = kMT / 32;      // warps per CTA
constexpr int kStageN = 3072;      // entries of a staged column; longer columns stream
constexpr int kAhead = 4;          // column j stages column j + kAhead
constexpr int kPf = 2;             // column j prefetches the rows of column j + kPf
constexpr int kNBuf = kAhead + 1;  // stage buffers: columns j .. j + kAhead
constexpr int kRing = 8;           // column metadata ring: columns j .. j + kAhead + 1

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

template <int MODEL, int G>
__global__ void __launch_bounds__(kMT, 1) batch_mixed_kernel(BatchParams P) {
    constexpr int S = kMT / G;       // threads per instance
    constexpr int kE = kStageN / S;  // staged entries per thread
    __shared__ double s_red2[2][kMW][4][2];
    __shared__ double s_red4[2][kMW][4][4];
    __shared__ MMeta s_meta[kRing];
    extern __shared__ __align__(16) unsigned char s_dyn[];
    MStage* st = reinterpret_cast<MStage*>(s_dyn);

    const int grp = blockIdx.x;
    const int g = threadIdx.x % G;
    const int sl = threadIdx.x / G;
    const int pos = grp * G + g;
    const bool exists = pos < P.n_inst;
    const int inst = exists ? (P.order ? P.order[pos] : pos) : -1;
    const int64_t K = P.K;
    const int J = P.J;
    double* X = P.xg + (size_t)grp * (size_t)K * G;
    double* Bt = P.beta_g + (size_t)grp * (size_t)J * G;
    double* Hd = P.hd_g + (size_t)grp * (size_t)J * G;
    double* Xy = P.xjy_g + (size_t)grp * (size_t)J * G;
    const int hold = (exists && P.holdout) ? P.holdout[inst] : -1;
    const double var = exists ? P.variance[inst] : 1.0;
    const double lambda = sqrt(2.0 / var);
    const int32_t* fold = (hold >= 0) ? P.row_fold : nullptr;  // a negative holdout holds out nothing
    int rb2 = 0, rb4 = 0;

    // state: xBeta from the offset column (computeXBeta with beta_0 = 1), coefficients, bounds
    for (int64_t k = sl; k < K; k += S) X[k * G + g] = P.offset_vals ? 0.0 + 1.0 * P.offset_vals[k] : 0.0;
    for (int j = sl; j < J; j += S) {
        Bt[(size_t)j * G + g] = (P.offset_vals && j == 0) ? 1.0 : 0.0;
        Hd[(size_t)j * G + g] = P.initial_bound;
    }
    // XjY of each instance (ModelSpecifics.hpp:486-524): x * y * w over the column
    for (int j = 0; j < J; ++j) {
        const MMeta m = load_meta(P, j);
        const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
        const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
        double acc[2] = {0.0, 0.0};
        if (exists)
            for (int64_t p = sl; p < m.n; p += S) {
                const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : p;
                const double x = has_vals ? __ldg(P.vals + m.vb + p) : 1.0;
                const double w = (fold && __ldg(fold + k) == hold) ? 0.0 : 1.0;
                acc[0] += x * P.y[k] * w;
            }
        group_sum<G, 2>(acc, s_red2, rb2);
        if (sl == 0) Xy[(size_t)j * G + g] = acc[0];
    }
    __syncthreads();

    // per-sweep objective in FP64 (getLogLikelihood, ModelSpecifics.hpp:605-650;
    // the gradient objective, :103-120); the LL terms only when they are needed
    auto objective = [&](bool active, bool need_ll, double& ll_out) -> double {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (active)
            for (int64_t k = sl; k < K; k += S) {
                const double xb = X[k * G + g];
                const double w = (fold && __ldg(fold + k) == hold) ? 0.0 : 1.0;
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
            for (int j = sl; j < J; j += S) {
                const int pt = P.ptype[j];
                acc[3] += log_prior_one(Bt[(size_t)j * G + g], pt, pt == 0 ? 1.0 : var);
            }
        group_sum<G, 4>(acc, s_red4, rb4);
        const double fixed = (MODEL == M_POISSON && P.ll_fixed && exists) ? P.ll_fixed[inst] : 0.0;
        ll_out = (acc[0] - acc[1]) + fixed;
        if (P.conv == C_GRADIENT) return acc[2];
        if (P.conv == C_MITTAL) return ll_out;
        return ll_out + acc[3];
    };

    const int j0 = P.offset_vals ? 1 : 0;
    const bool need_ll = P.conv != C_GRADIENT;
    bool active = exists;
    double ll = 0.0;
    double last = objective(active, need_ll, ll);
    int iteration = 0, flag = R_FAIL;
    long long steps = 0, updates = 0, upd_entries = 0, gh_entries = 0;

    auto stage = [&](int col) {
        const MMeta m = s_meta[col & (kRing - 1)];
        if (!stageable(m)) return;
        MStage& b = st[col % kNBuf];
        for (int p = threadIdx.x; p < m.n; p += kMT) {
            cp_async4(&b.k[p], P.keys + m.cb + p);
            if (m.fmt == F_SPARSE) cp_async8(&b.x[p], P.vals + m.vb + p);
        }
    };
    auto prefetch = [&](int col) {
        const MMeta m1 = s_meta[col & (kRing - 1)];
        if (!stageable(m1)) return;
        const MStage& b = st[col % kNBuf];
        for (int p = threadIdx.x; p < m1.n; p += kMT)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(X + (int64_t)(b.k[p] & kKeyRowMask) * G));
    };

    while (__syncthreads_or(active)) {
        // sweep prologue: metadata of the first kAhead + 1 columns, stage the first kAhead
        if (threadIdx.x <= kAhead && j0 + (int)threadIdx.x < J)
            s_meta[(j0 + threadIdx.x) & (kRing - 1)] = load_meta(P, j0 + threadIdx.x);
        __syncthreads();
        for (int q = 0; q < kAhead; ++q)
            if (j0 + q < J) stage(j0 + q);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        if (P.prefetch)
            for (int q = 0; q < kPf; ++q)
                if (j0 + q < J) prefetch(j0 + q);
        // coefficient, bound, XjY and prior of the next column, one column ahead
        double nb0 = 0.0, nhd0 = 0.0, nxjy0 = 0.0;
        int npt = 0;
        if (j0 < J) {
            if (active) {
                nb0 = Bt[(size_t)j0 * G + g];
                nhd0 = Hd[(size_t)j0 * G + g];
                nxjy0 = Xy[(size_t)j0 * G + g];
            }
            npt = P.ptype[j0];
        }
        long long* tr = (P.trace && blockIdx.x == 0 && threadIdx.x == 0 && iteration == P.trace_sweep)
                            ? P.trace : nullptr;

        for (int j = j0; j < J; ++j) {
            if (tr) tr[6 * j] = clock64();
            const MMeta m = s_meta[j & (kRing - 1)];
            const int n = m.n;
            const bool ind = (m.fmt == F_INDICATOR || m.fmt == F_INTERCEPT);
            const bool staged = stageable(m);
            const double b0 = nb0, hd0 = nhd0, xjy0 = nxjy0;
            const int pt = npt;
            if (j + 1 < J) {
                if (active) {
                    nb0 = Bt[(size_t)(j + 1) * G + g];
                    nhd0 = Hd[(size_t)(j + 1) * G + g];
                    nxjy0 = Xy[(size_t)(j + 1) * G + g];
                }
                npt = P.ptype[j + 1];
            }
            MMeta nm{};
            if (threadIdx.x == 0 && j + kAhead + 1 < J) nm = load_meta(P, j + kAhead + 1);
            if (j + kAhead < J) stage(j + kAhead);
            cp_async_commit();
            if (P.prefetch && j + kPf < J) prefetch(j + kPf);
            if (tr) tr[6 * j + 1] = clock64();

            // gather and FP32 terms with compensated sums
            float gs = 0.f, gc = 0.f, hs = 0.f, hc = 0.f;
            double xr[kE];
            const MStage& c = st[j % kNBuf];
            if (staged) {
                if (active) {
                    // loads only: every gather of the column is in flight at once
#pragma unroll
                    for (int i = 0; i < kE; ++i) {
                        const int p = sl + i * S;
                        if (p < n) xr[i] = X[(int64_t)(c.k[p] & kKeyRowMask) * G + g];
                    }
#pragma unroll
                    for (int i = 0; i < kE; ++i) {
                        const int p = sl + i * S;
                        if (p < n && (c.k[p] >> kKeyRowBits) != hold) {
                            const float x = (m.fmt == F_SPARSE) ? (float)c.x[p] : 1.0f;
                            float gt, ht;
                            entry_terms<MODEL>(xr[i], x, ind, gt, ht);
                            two_sum(gs, gc, gt);
                            two_sum(hs, hc, ht);
                        }
                    }
                }
            } else if (active) {
                const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
                const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
                for (int64_t p = sl; p < n; p += S) {
                    const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : p;
                    if (fold && __ldg(fold + k) == hold) continue;
                    const float x = has_vals ? (float)__ldg(P.vals + m.vb + p) : 1.0f;
                    float gt, ht;
                    entry_terms<MODEL>(X[k * G + g], x, ind, gt, ht);
                    two_sum(gs, gc, gt);
                    two_sum(hs, hc, ht);
                }
            }
            double gh[2] = {(double)gs + (double)gc, (double)hs + (double)hc};
            if (tr) tr[6 * j + 2] = clock64();
            group_sum<G, 2>(gh, s_red2, rb2);
            if (tr) tr[6 * j + 3] = clock64();

            // the step, computed identically by every thread of the instance
            double d = 0.0;
            if (active) {
                double Gv = 0.0, Hv = 0.0;
                if (n > 0) {  // an empty column gives (0, 0) (ModelSpecifics.hpp:720-723)
                    Gv = gh[0] - xjy0;
                    Hv = gh[1];
                }
                d = newton_prior_delta_l(Gv, Hv, b0, pt, pt == 0 ? 1.0 : var, lambda);
                double bnd = hd0;
                d = apply_bounds(d, bnd);
                if (sl == 0) {
                    Hd[(size_t)j * G + g] = bnd;
                    if (d != 0.0) {
                        Bt[(size_t)j * G + g] = b0 + d;
                        ++updates;
                        upd_entries += n;
                    }
                    ++steps;
                    gh_entries += n;
                }
            }
            // update xBeta (FP64) from the gathered registers
            if (d != 0.0) {
                if (staged) {
#pragma unroll
                    for (int i = 0; i < kE; ++i) {
                        const int p = sl + i * S;
                        if (p < n) {
                            const double x = (m.fmt == F_SPARSE) ? c.x[p] : 1.0;
                            X[(int64_t)(c.k[p] & kKeyRowMask) * G + g] = xr[i] + d * x;
                        }
                    }
                } else {
                    const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
                    const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
                    for (int64_t p = sl; p < n; p += S) {
                        const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : p;
                        const double x = has_vals ? __ldg(P.vals + m.vb + p) : 1.0;
                        X[k * G + g] += d * x;
                    }
                }
            }
            if (threadIdx.x == 0 && j + kAhead + 1 < J) s_meta[(j + kAhead + 1) & (kRing - 1)] = nm;
            if (tr) tr[6 * j + 4] = clock64();
            cp_async_wait_but_last();
            __syncthreads();
            if (tr) tr[6 * j + 5] = clock64();
        }
        cp_async_wait_all();

        // convergence, per instance (CyclicCoordinateDescent.cpp:541-558, 839-906)
        if (active) ++iteration;
        const double cur = objective(active, need_ll, ll);
        if (active) {
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
    }

    // log-likelihood on the training rows and the predictive log-likelihood of
    // the held-out rows (getPredictiveLogLikelihood, ModelSpecifics.hpp:652-690), FP64
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (exists)
        for (int64_t k = sl; k < K; k += S) {
            const double xb = X[k * G + g];
            const bool out = fold && __ldg(fold + k) == hold;
            const double w = out ? 0.0 : 1.0, wo = 1.0 - w;
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
    group_sum<G, 4>(acc, s_red4, rb4);
    if (exists && sl == 0) {
        const double fixed = (MODEL == M_POISSON && P.ll_fixed) ? P.ll_fixed[inst] : 0.0;
        BatchResult r;
        r.flag = flag;
        r.iterations = iteration;
        r.loglik = (acc[0] - acc[1]) + fixed;
        r.objective = last;
        r.pred_loglik = acc[2];
        r.steps = steps;
        r.updates = updates;
        r.update_entries = upd_entries;
        r.sweep_entries = gh_entries;
        P.results[inst] = r;
    }
}

__global__ void batch_keys_kernel(const int32_t* rows, int64_t nnz, const int32_t* fold, int32_t* keys) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = rows[e];
        int32_t f = fold ? fold[k] : -1;
        if (f < 0 || f >= kKeyNoFold) f = kKeyNoFold;
        keys[e] = k | (f << kKeyRowBits);
    }
}

template <int MODEL, int G>
cudaError_t launch_g(const BatchParams& P, cudaStream_t stream) {
    const size_t smem = sizeof(MStage) * kNBuf;
    cudaError_t e = cudaFuncSetAttribute(batch_mixed_kernel<MODEL, G>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int n_groups = (P.n_inst + G - 1) / G;
    batch_mixed_kernel<MODEL, G><<<n_groups, kMT, smem, stream>>>(P);
    return cudaGetLastError();
}

template <int MODEL>
cudaError_t launch_m(const BatchParams& P, cudaStream_t stream) {
    switch (P.group) {
    case 1: return launch_g<MODEL, 1>(P, stream);
    case 2: return launch_g<MODEL, 2>(P, stream);
    case 4: return launch_g<MODEL, 4>(P, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_batch_keys(const int32_t* rows, int64_t nnz, const int32_t* fold, int32_t* keys,
                              cudaStream_t stream) {
    if (nnz <= 0) return cudaSuccess;
    batch_keys_kernel<<<148 * 4, 256, 0, stream>>>(rows, nnz, fold, keys);
    return cudaGetLastError();
}

cudaError_t launch_batch_mixed(const BatchParams& P, cudaStream_t stream) {
    return (P.model == M_LOGISTIC) ? launch_m<M_LOGISTIC>(P, stream) : launch_m<M_POISSON>(P, stream);
}

}  // namespace ccdb
