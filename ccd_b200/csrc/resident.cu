// resident.cu -- one findMode of an independent-row fit (logistic, Poisson)
// in one CTA whose shared memory holds the row state (or, for a fit with more
// rows than that, a global array only this CTA touches).
//
// A fit of up to resident_max_rows() rows keeps {xBeta, denominator} of every
// row in shared memory for the whole launch.  offsExpXBeta is not stored: every
// value the engine ever holds for it is exp(xBeta) of the same xBeta (set by
// computeRemainingStatistics and by every update, ModelSpecifics.hpp:1548-1571),
// so it is recomputed where it is used.  The weights stay in global memory and
// are read only by weighted fits (an unweighted fit's weights are 1.0, whose
// products are exact).  With no other CTA to wait for, a coordinate costs
// shared-memory latency and the L2 round trips of its column's entries, not a
// grid or cluster barrier.
//
// The sweep is the sequential cycle (CyclicCoordinateDescent.cpp:1008-1021) run
// as speculative batches: the warps compute the gradients of consecutive short
// columns (one each) against one state, the first nonzero step in visiting
// order is applied by its warp, and the batch restarts after it -- every zero
// step leaves the state untouched, so each gradient is the one the sequential
// cycle computes.  A long column (more than kLong entries: the intercept, dense
// columns) is taken by the whole CTA on its own.  Bounds (hDelta) change with
// every visited coordinate, zero steps included, as applyBounds does.  The
// per-position column records (row offset, value offset, entry count, format)
// are built by the host, so a batch reads one record per column before its
// entries.  The convergence test runs on the device after each cycle from the
// same objective terms as the other sweeps; at exit the row state is written
// back to global memory.
//
// A fit with more rows than shared memory holds runs the same sweep with the
// row state in a global array (GL): only this CTA touches it, so the block
// barriers order its reads and writes and L1 keeps what fits.  Warps then take
// columns of up to kResidentWarpMaxGlobal entries, in chunks of 256: a large
// L1-penalised fit, whose steps are mostly zero and whose columns share rows,
// moves a whole batch of columns per round instead of one dependency level a
// column.
//
// No wait spans CTAs (there is one), so the kernel has no wait to bound.
#include <cstdint>

#include "common.cuh"
#include "indep.h"
#include "resident.h"
#include "step.h"

namespace ccdb {

namespace {

constexpr int kRT = 512;              // threads
constexpr int kRW = kRT / 32;         // warps = columns per speculative batch
constexpr int kLong = 256;            // longer columns run on the whole CTA
constexpr int kLanePer = kLong / 32;  // entries per lane of a warp's column

// One entry's gradient and Hessian terms (ModelSpecifics.h:541-568 logistic,
// Poisson ModelSpecifics.h:1509-1530), accumulated in entry order.
template <int MODEL>
__device__ __forceinline__ void entry_gh(bool ind, double x, double e, double dn, double w, double& g,
                                         double& h) {
    const double n1 = e * x;
    if (MODEL == M_LOGISTIC) {
        const double gg = n1 / dn;
        g += w * gg;
        if (ind) h += w * gg * (1.0 - gg);
        else h += w * ((n1 * x) / dn - gg * gg);
    } else {
        if (ind) {
            const double v = w * n1;
            g += v;
            h += v;
        } else {
            g += w * n1;
            h += w * (n1 * x);
        }
    }
}

// updateXBeta for one entry: xBeta += delta x, offsExpXBeta = exp, the
// denominator changed by the difference (ModelSpecifics.hpp:1548-1571).
__device__ __forceinline__ void entry_update(double2* s_rs, int k, double x, double delta) {
    const double2 xd = s_rs[k];
    const double xb = xd.x + delta * x;
    const double en = exp(xb);
    s_rs[k] = make_double2(xb, xd.y + (en - exp(xd.x)));
}

// The step of column j from its (g, h) sums: Newton step with the prior,
// then the bound (meta_step of the other sweeps).
__device__ __forceinline__ double col_step(int64_t n, double gsum, double hsum, double xjy, double beta,
                                           int ptype, double pvar, double& hd) {
    double g = 0.0, h = 0.0;
    if (n > 0) {
        g = gsum - xjy;
        h = hsum;
    }
    const double d = newton_prior_delta(g, h, beta, ptype, pvar);
    return apply_bounds(d, hd);
}

// CTA sum of (g, h) in a fixed order, the same bits in every thread.
__device__ __forceinline__ double2 cta_sum2_all(double2 v, double2* s_red) {
    v = warp_sum2(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_red[wid] = v;
    __syncthreads();
    double2 t = (lane < kRW) ? s_red[lane] : make_double2(0.0, 0.0);
#pragma unroll
    for (int o = kRW / 2; o > 0; o >>= 1) {
        t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
    }
    t.x = __shfl_sync(0xffffffffu, t.x, 0);
    t.y = __shfl_sync(0xffffffffu, t.y, 0);
    __syncthreads();  // s_red is free again
    return t;
}

// The objective terms {LL numerator, LL denominator, gradient objective, log
// prior} over all rows and columns (objective_share of the other sweeps),
// valid in every thread.
template <int MODEL>
__device__ double4 objective_terms(const ResidentParams& R, const double2* s_rs, double4* s_red4) {
    const IndepParams& P = R.P;
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int64_t k = threadIdx.x; k < P.K; k += blockDim.x) {
        const double2 xd = s_rs[k];
        const double w = R.weighted ? P.row[2 * k + 1].y : 1.0;
        const double yk = P.y[k];
        acc.x += (double)((int)yk) * xd.x * w;
        if (MODEL == M_LOGISTIC) acc.y += w * log(xd.y);
        else acc.y += w * xd.y;
        acc.z += xd.x * yk * w;
    }
    for (int64_t j = threadIdx.x; j < P.J; j += blockDim.x) acc.w += log_prior_one(P.beta[j], P.ptype[j], P.pvar[j]);
    return block_sum4<kRW>(acc, s_red4);
}

// The convergence objective of findMode from the objective terms.
__device__ __forceinline__ double conv_objective(int conv, const double4& t, double ll_fixed, double& ll) {
    ll = (t.x - t.y) + ll_fixed;
    return (conv == C_GRADIENT) ? t.z : (conv == C_MITTAL ? ll : ll + t.w);
}

__device__ __forceinline__ ResCol shfl_rec(const ResCol& r, int src) {
    ResCol o;
    o.j = __shfl_sync(0xffffffffu, r.j, src);
    o.flags = __shfl_sync(0xffffffffu, r.flags, src);
    o.n = __shfl_sync(0xffffffffu, r.n, src);
    o.cb = __shfl_sync(0xffffffffu, r.cb, src);
    o.vb = __shfl_sync(0xffffffffu, r.vb, src);
    return o;
}

template <int MODEL, bool GL>
__global__ void __launch_bounds__(kRT, 1) resident_sweep_kernel(ResidentParams R) {
    extern __shared__ __align__(16) double2 s_dyn[];  // {xBeta, denominator} of every row (shared form)
    __shared__ double2 s_red2[kRW];
    __shared__ double4 s_red4[kRW];
    __shared__ double s_delta[kRW], s_hd[kRW], s_beta[kRW];

    const IndepParams& P = R.P;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double2* const s_rs = GL ? R.rs : s_dyn;
    const int64_t warp_max = GL ? kResidentWarpMaxGlobal : kLong;
    for (int64_t k = tid; k < P.K; k += kRT) s_rs[k] = make_double2(P.row[2 * k].x, P.row[2 * k + 1].x);
    __syncthreads();

    double ll;
    double last = conv_objective(P.conv, objective_terms<MODEL>(R, s_rs, s_red4), P.ll_fixed, ll);
    unsigned long long moved = 0;
    long long* tr = (R.trace && tid == 0) ? R.trace : nullptr;
    int trn = R.trace_n;

    for (int it = 0; it < P.max_iter; ++it) {
        int pos = 0;
        while (pos < R.n_active) {
            const long long tb0 = tr ? clock64() : 0;
            // the column records of the next 32 positions (lanes kRW.. hold the batch
            // after this one); the run of short ones among the first kRW
            ResCol rec{-1, 0, 0, 0, 0};
            const int q = pos + lane;
            if (q < R.n_active) rec = R.recs[q];
            const bool short_col = lane < kRW && rec.j >= 0 && rec.n <= warp_max;
            const unsigned run = __ballot_sync(0xffffffffu, short_col);
            const int nb = (~run == 0u) ? 32 : __ffs(~run) - 1;  // at most kRW: lanes >= kRW are false
            if (nb == 0) {
                // ---- a long column: the whole CTA
                const ResCol c = shfl_rec(rec, 0);
                const int j = c.j;
                const bool has_rows = c.flags & 1, has_vals = c.flags & 2, ind = c.flags & 4;
                const double xjy = P.xjy[j], pvar = P.pvar[j], b0 = P.beta[j];
                const int ptype = P.ptype[j];
                double hd = P.hdelta[j];
                double g = 0.0, h = 0.0;
                for (int64_t p = tid; p < c.n; p += kRT) {
                    const int k = has_rows ? __ldg(P.rows + c.cb + p) : (int)p;
                    const double x = has_vals ? __ldg(P.vals + c.vb + p) : 1.0;
                    const double w = R.weighted ? P.row[2 * (int64_t)k + 1].y : 1.0;
                    const double2 xd = s_rs[k];
                    entry_gh<MODEL>(ind, x, exp(xd.x), xd.y, w, g, h);
                }
                const double2 s = cta_sum2_all(make_double2(g, h), s_red2);
                const double d = col_step(c.n, s.x, s.y, xjy, b0, ptype, pvar, hd);
                if (d != 0.0) {
                    for (int64_t p = tid; p < c.n; p += kRT) {
                        const int k = has_rows ? __ldg(P.rows + c.cb + p) : (int)p;
                        const double x = has_vals ? __ldg(P.vals + c.vb + p) : 1.0;
                        entry_update(s_rs, k, x, d);
                    }
                }
                if (tid == 0) {
                    P.hdelta[j] = hd;
                    if (d != 0.0) {
                        P.beta[j] = b0 + d;
                        ++moved;
                    }
                }
                __syncthreads();  // the state is read by the next columns
                pos += 1;
                if (tr) {
                    tr[0] = tb0;
                    tr[4] = clock64();
                    tr[5] = -1;  // a long column
                    tr += kResidentTraceWords;
                    if (--trn <= 0) tr = nullptr;
                }
                continue;
            }
            // ---- a batch of nb short columns, one per warp, against the same state
            const ResCol c = shfl_rec(rec, wid < nb ? wid : 0);
            const bool has_rows = c.flags & 1, has_vals = c.flags & 2, ind = c.flags & 4;
            // the warp's column in chunks of kLong entries, kLanePer a lane (one
            // chunk in the shared form); the last chunk stays in registers
            int k[kLanePer];
            double x[kLanePer];
            auto load_chunk = [&](int64_t base) {
#pragma unroll
                for (int i = 0; i < kLanePer; ++i) {
                    const int64_t p = base + lane + 32 * i;
                    k[i] = -1;
                    x[i] = 1.0;
                    if (p < c.n) {
                        k[i] = has_rows ? __ldg(P.rows + c.cb + p) : (int)p;
                        if (has_vals) x[i] = __ldg(P.vals + c.vb + p);
                    }
                }
            };
            double g = 0.0, h = 0.0;
            auto add_chunk = [&]() {
#pragma unroll
                for (int i = 0; i < kLanePer; ++i)
                    if (k[i] >= 0) {
                        const double w = R.weighted ? P.row[2 * (int64_t)k[i] + 1].y : 1.0;
                        const double2 xd = s_rs[k[i]];
                        entry_gh<MODEL>(ind, x[i], exp(xd.x), xd.y, w, g, h);
                    }
            };
#pragma unroll
            for (int i = 0; i < kLanePer; ++i) k[i] = -1;
            if (wid < nb) {
                const int j = c.j;
                load_chunk(0);  // the entries' loads go out before the column's scalars
                const double xjy = P.xjy[j], pvar = P.pvar[j], b0 = P.beta[j];
                const int ptype = P.ptype[j];
                double hd = P.hdelta[j];
                add_chunk();
                if (GL)
                    for (int64_t base = kLong; base < c.n; base += kLong) {
                        load_chunk(base);
                        add_chunk();
                    }
                // the butterfly leaves the same sums in every lane
                const double2 s = warp_sum2(make_double2(g, h));
                const double d = col_step(c.n, s.x, s.y, xjy, b0, ptype, pvar, hd);
                if (lane == 0) {
                    s_delta[wid] = d;
                    s_hd[wid] = hd;
                    s_beta[wid] = b0;
                }
            }
            const long long tb1 = tr ? clock64() : 0;
            __syncthreads();
            const long long tb2 = tr ? clock64() : 0;
            // the first nonzero step in visiting order; the columns up to it are visited
            const unsigned nz = __ballot_sync(0xffffffffu, lane < nb && s_delta[lane] != 0.0);
            const int first = nz ? __ffs(nz) - 1 : nb;
            const int walked = (first < nb) ? first + 1 : nb;
            if (wid < walked && lane == 0) {
                P.hdelta[c.j] = s_hd[wid];
                if (wid == first) {
                    P.beta[c.j] = s_beta[wid] + s_delta[wid];
                    ++moved;
                }
            }
            if (wid == first && first < nb) {
                const double d = s_delta[wid];
                if (GL && c.n > kLong) {  // a column of several chunks: read them again
                    for (int64_t base = 0; base < c.n; base += kLong) {
                        load_chunk(base);
#pragma unroll
                        for (int i = 0; i < kLanePer; ++i)
                            if (k[i] >= 0) entry_update(s_rs, k[i], x[i], d);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < kLanePer; ++i)
                        if (k[i] >= 0) entry_update(s_rs, k[i], x[i], d);
                }
            }
            const long long tb3 = tr ? clock64() : 0;
            __syncthreads();
            pos += walked;
            if (tr) {
                tr[0] = tb0;
                tr[1] = tb1;
                tr[2] = tb2;
                tr[3] = tb3;
                tr[4] = clock64();
                tr[5] = nb;
                tr[6] = first;
                tr += kResidentTraceWords;
                if (--trn <= 0) tr = nullptr;
            }
        }
        // ---- the cycle is complete: convergence (findMode, CyclicCoordinateDescent.cpp:1023-1056)
        const double4 t = objective_terms<MODEL>(R, s_rs, s_red4);
        const double cur = conv_objective(P.conv, t, P.ll_fixed, ll);
        const int iteration = it + 1;
        double conv;
        bool ill = false;
        if (cur != cur) {
            conv = 0.0;
            ill = true;
        } else {
            conv = fabs(cur - last) / (fabs(cur) + 1.0);
        }
        last = cur;
        int done = 0, flag = R_SUCCESS;
        if (P.tol > 0 && conv < P.tol) {
            flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
            done = 1;
        } else if (iteration == P.max_iter) {
            flag = R_MAX_ITERATIONS;
            done = 1;
        }
        if (tid == 0) {
            P.st->iterations = iteration;
            P.st->objective = cur;
            P.st->loglik = ll;
            P.st->log_prior = t.w;
            if (done) P.st->flag = flag;
        }
        if (done) break;
    }
    // the row state back to global memory for the calls that follow
    for (int64_t k = tid; k < P.K; k += kRT) {
        const double2 xd = s_rs[k];
        P.row[2 * k] = make_double2(xd.x, exp(xd.x));
        P.row[2 * k + 1].x = xd.y;
    }
    if (moved) atomicAdd(&P.st->nonzero_steps, moved);
}

constexpr size_t kStaticSmemBound = 4096;  // the kernel's static shared memory stays below this

}  // namespace

int resident_threads() { return kRT; }

cudaError_t resident_max_rows(int model, int64_t* rows) {
    (void)model;
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const size_t avail = (size_t)optin > kStaticSmemBound ? (size_t)optin - kStaticSmemBound : 0;
    *rows = (int64_t)(avail / sizeof(double2));
    return cudaSuccess;
}

cudaError_t launch_resident_sweep(const ResidentParams& R, cudaStream_t stream) {
    // the dynamic shared memory limit is raised once to the most a CTA can hold
    static std::atomic<uint64_t> done{0};
    cudaError_t e = once_per_device(done, [] {
        int dev = 0, optin = 0;
        cudaError_t r = cudaGetDevice(&dev);
        if (r == cudaSuccess) r = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (r != cudaSuccess) return r;
        const int dyn = optin - (int)kStaticSmemBound;
        r = cudaFuncSetAttribute(resident_sweep_kernel<M_LOGISTIC, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
        if (r != cudaSuccess) return r;
        return cudaFuncSetAttribute(resident_sweep_kernel<M_POISSON, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    });
    if (e != cudaSuccess) return e;
    if (R.rs) {  // the row state in global memory
        if (R.P.model == M_LOGISTIC) resident_sweep_kernel<M_LOGISTIC, true><<<1, kRT, 0, stream>>>(R);
        else resident_sweep_kernel<M_POISSON, true><<<1, kRT, 0, stream>>>(R);
        return cudaGetLastError();
    }
    const size_t smem = sizeof(double2) * (size_t)R.P.K;
    if (R.P.model == M_LOGISTIC) resident_sweep_kernel<M_LOGISTIC, false><<<1, kRT, smem, stream>>>(R);
    else resident_sweep_kernel<M_POISSON, false><<<1, kRT, smem, stream>>>(R);
    return cudaGetLastError();
}

}  // namespace ccdb
