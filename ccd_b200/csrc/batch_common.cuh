// batch_common.cuh -- the per-instance pieces of the mixed-precision batched
// engine (batch_mixed.cu): instance context, slices of a column owned by one
// CTA of a cluster, cluster-wide sums, setup, objective, step and results.
#pragma once

#include <cooperative_groups.h>

#include <cstdint>

#include "batch.h"
#include "common.cuh"
#include "step.h"

namespace ccdb {
namespace bm {

constexpr int kMT = 512;           // threads per CTA
constexpr int kMW = kMT / 32;      // warps per CTA
// A CTA stages the keys (and values) of its slice of a column when the slice
// has at most SN entries; longer slices stream from global memory.
template <int SN>
struct MStage {
    int32_t k[SN];  // keys: row | fold code << 24
    double x[SN];
};

// The part of column j one CTA owns: entries [cb, cb + n) of the row-indexed
// arrays (rows, keys, vals at [vb, vb + n)) for SPARSE / INDICATOR columns; rows
// [cb, cb + n) (values at [vb, vb + n)) for DENSE / INTERCEPT columns.  ntot is
// the whole column's entry count.
struct MMeta {
    int64_t cb, vb;
    int32_t n, fmt, ntot, pad;
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

// Slice of column j owned by CTA `rank` of a cluster of C, which owns rows
// [rlo, rhi); P.split holds, per row-indexed column, the C + 1 entry offsets
// where the column's rows cross the ranks' row boundaries.
__device__ __forceinline__ MMeta load_meta(const BatchParams& P, int j, int rank, int C, int64_t rlo,
                                           int64_t rhi) {
    MMeta m;
    const int f = P.fmt[j];
    m.fmt = f;
    m.pad = 0;
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    if (f == F_DENSE || f == F_INTERCEPT) {
        m.ntot = (int32_t)P.K;
        m.cb = rlo;
        m.vb = vb + rlo;
        m.n = (int32_t)(rhi - rlo);
    } else {
        m.ntot = (int32_t)(P.col_ptr[j + 1] - cb);
        int32_t lo = 0, hi = m.ntot;
        if (C > 1) {
            lo = P.split[(size_t)j * (C + 1) + rank];
            hi = P.split[(size_t)j * (C + 1) + rank + 1];
        }
        m.cb = cb + lo;
        m.vb = vb + lo;
        m.n = hi - lo;
    }
    return m;
}

// load_meta in two halves: the loads (issued early, nothing waits on them)
// and the arithmetic (done once they have landed).
struct RawMeta {
    int64_t c0, c1, v;
    int32_t lo, hi, f;
};

__device__ __forceinline__ RawMeta raw_meta(const BatchParams& P, int j, int rank, int C) {
    RawMeta r;
    r.f = P.fmt[j];
    r.c0 = P.col_ptr[j];
    r.c1 = P.col_ptr[j + 1];
    r.v = P.val_ptr[j];
    r.lo = (C > 1) ? P.split[(size_t)j * (C + 1) + rank] : 0;
    r.hi = (C > 1) ? P.split[(size_t)j * (C + 1) + rank + 1] : 0;
    return r;
}

__device__ __forceinline__ MMeta cook_meta(const RawMeta& r, int64_t K, int C, int64_t rlo, int64_t rhi) {
    MMeta m;
    m.fmt = r.f;
    m.pad = 0;
    if (r.f == F_DENSE || r.f == F_INTERCEPT) {
        m.ntot = (int32_t)K;
        m.cb = rlo;
        m.vb = r.v + rlo;
        m.n = (int32_t)(rhi - rlo);
    } else {
        m.ntot = (int32_t)(r.c1 - r.c0);
        const int32_t lo = (C > 1) ? r.lo : 0, hi = (C > 1) ? r.hi : m.ntot;
        m.cb = r.c0 + lo;
        m.vb = r.v + lo;
        m.n = hi - lo;
    }
    return m;
}

template <int SN>
__device__ __forceinline__ bool stageable(const MMeta& m) {
    return (m.fmt == F_SPARSE || m.fmt == F_INDICATOR) && m.n <= SN;
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

// One thread's view of its instance: which instance of the group it serves,
// that instance's slices of the group arrays, prior and held-out fold, and the
// rows [rlo, rhi) that this CTA owns within its cluster of C CTAs.
template <int G>
struct Inst {
    static constexpr int S = kMT / G;  // threads per instance
    int grp, g, sl, inst, hold, J, rank, C;
    bool exists;
    int64_t K, rlo, rhi;
    double *X, *Bt, *Hd, *Xy;
    double var, lambda;
    const int32_t* fold;  // NULL when the instance holds nothing out

    __device__ Inst(const BatchParams& P, int cluster, int group, int cta_rank) {
        C = cluster;
        grp = group;
        rank = cta_rank;
        g = threadIdx.x % G;
        sl = threadIdx.x / G;
        const int pos = grp * G + g;
        exists = pos < P.n_inst;
        inst = exists ? (P.order ? P.order[pos] : pos) : -1;
        K = P.K;
        J = P.J;
        rlo = K * rank / C;
        rhi = K * (rank + 1) / C;
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
    __device__ MMeta meta(const BatchParams& P, int j) const { return load_meta(P, j, rank, C, rlo, rhi); }
    __device__ RawMeta raw(const BatchParams& P, int j) const { return raw_meta(P, j, rank, C); }
    __device__ MMeta cook(const RawMeta& r) const { return cook_meta(r, K, C, rlo, rhi); }
};

// Sum over the instance's threads in the CTA, then over the CTAs of the
// cluster: each CTA publishes its sums in its shared memory, and after the
// cluster barrier every thread adds the C values in rank order, so every CTA
// gets the same bits.  `xch` alternates between two buffers (a CTA can reuse
// one only after every CTA passed the next cluster barrier, i.e. after all
// have read it).
template <int G, int NV>
__device__ __forceinline__ void inst_sum(const Inst<G>& I, double (&v)[NV], double (*red)[kMW][4][NV], int& rb,
                                         double (*xch)[4][NV], int& xb) {
    group_sum<G, NV>(v, red, rb);
    if (I.C == 1) return;
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    if (I.sl == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) xch[xb][I.g][q] = v[q];
    cl.sync();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double t = 0.0;
        for (int r = 0; r < I.C; ++r) t += *cl.map_shared_rank(&xch[xb][I.g][q], r);
        v[q] = t;
    }
    xb ^= 1;
}

// --- per-column cluster exchange without a cluster barrier -------------------
// Each CTA pushes its per-instance (g, h) sums into every other CTA's shared
// memory with st.async, which completes on the receiver's mbarrier; a CTA
// waits only for its own mbarrier.  Slots alternate by column parity: a CTA
// cannot send column j + 2 before it has received every CTA's column j + 1,
// which each sends only after consuming column j.

constexpr int kMaxCluster = 16;
// After a wait has run past the caller's bound (BatchParams::xch_wait_ns) and
// raised the abort word, it keeps waiting up to this much longer before giving
// up: peers that are slow but running still deliver, so every CTA of the
// cluster finishes the sweep's exchanges in step and no st.async is left in
// flight towards a CTA that leaves.
constexpr unsigned long long kXchGiveUpNs = 2000000000ull;

struct __align__(16) ColXch {  // st.async of two doubles needs 16-byte aligned slots
    double part[2][kMaxCluster][4][2];  // [slot][rank][instance][g, h]
    uint64_t bar[2];
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void xch_init(ColXch& x) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&x.bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&x.bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ unsigned long long xch_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Cluster-wide (g, h) of column j for the thread's instance.  A wait that runs
// past `limit_ns` raises the launch's abort word (the caller then stops
// stepping and reports a timeout) and goes on waiting up to kXchGiveUpNs;
// false only when even that ran out (the sums are then not valid).
template <int G>
__device__ __forceinline__ bool xch_sum(const Inst<G>& I, double (&v)[2], ColXch& x, int j, unsigned& phase_bits,
                                        unsigned long long limit_ns, int32_t* abort) {
    const int slot = j & 1;
    if (I.sl == 0)
        for (int r = 0; r < I.C; ++r) {
            if (r == I.rank) continue;
            unsigned ra, rb;
            asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                         : "=r"(ra)
                         : "r"(smem_addr(&x.part[slot][I.rank][I.g][0])), "r"(r));
            asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rb) : "r"(smem_addr(&x.bar[slot])), "r"(r));
            asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(ra),
                         "d"(v[0]), "d"(v[1]), "r"(rb)
                         : "memory");
        }
    if (threadIdx.x == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&x.bar[slot])),
                     "r"((unsigned)((I.C - 1) * G * 2 * sizeof(double)))
                     : "memory");
    const unsigned parity = (phase_bits >> slot) & 1u;
    phase_bits ^= 1u << slot;
    const unsigned a = smem_addr(&x.bar[slot]);
    const unsigned long long t0 = xch_now();
    bool raised = false;
    for (unsigned n = 0;; ++n) {
        unsigned done;
        // test_wait returns at once (try_wait may suspend the thread in hardware
        // until the phase completes, which would hide the bound from this loop)
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) break;
        if (n > 8) __nanosleep(32);
        const unsigned long long dt = xch_now() - t0;
        if (!raised && dt > limit_ns) {
            atomicExch(abort, 1);
            __threadfence();
            raised = true;
        }
        if (dt > limit_ns + kXchGiveUpNs) return false;
    }
    double sg = 0.0, sh = 0.0;  // rank order, own sums in place: the same bits in every CTA
    for (int r = 0; r < I.C; ++r) {
        sg += (r == I.rank) ? v[0] : x.part[slot][r][I.g][0];
        sh += (r == I.rank) ? v[1] : x.part[slot][r][I.g][1];
    }
    v[0] = sg;
    v[1] = sh;
    return true;
}

// Initial state: xBeta from the offset column (computeXBeta with beta_0 = 1),
// coefficients, bounds, and each instance's XjY (ModelSpecifics.hpp:486-524).
// Each CTA sets its own rows; rank 0 the coefficients and bounds.
template <int G>
__device__ void inst_setup(const BatchParams& P, const Inst<G>& I, double (*red2)[kMW][4][2], int& rb2,
                           double (*xch2)[4][2], int& xb2) {
    constexpr int S = Inst<G>::S;
    for (int64_t k = I.rlo + I.sl; k < I.rhi; k += S)
        I.X[k * G + I.g] = P.offset_vals ? 0.0 + 1.0 * P.offset_vals[k] : 0.0;
    if (I.rank == 0)
        for (int j = I.sl; j < I.J; j += S) {
            I.Bt[(size_t)j * G + I.g] = (P.offset_vals && j == 0) ? 1.0 : 0.0;
            I.Hd[(size_t)j * G + I.g] = P.initial_bound;
        }
    for (int j = 0; j < I.J; ++j) {
        const MMeta m = I.meta(P, j);
        const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
        const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
        double acc[2] = {0.0, 0.0};
        if (I.exists)
            for (int64_t p = I.sl; p < m.n; p += S) {
                const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : m.cb + p;
                const double x = has_vals ? __ldg(P.vals + m.vb + p) : 1.0;
                acc[0] += x * P.y[k] * (I.held(k) ? 0.0 : 1.0);
            }
        inst_sum<G, 2>(I, acc, red2, rb2, xch2, xb2);
        if (I.sl == 0 && I.rank == 0) I.Xy[(size_t)j * G + I.g] = acc[0];
    }
    if (I.C > 1) cooperative_groups::this_cluster().sync();  // coefficients and XjY are set
    __syncthreads();
}

// Per-sweep objective in FP64 (getLogLikelihood, ModelSpecifics.hpp:605-650;
// the gradient objective, :103-120); the LL terms only when they are needed.
template <int MODEL, int G>
__device__ double inst_objective(const BatchParams& P, const Inst<G>& I, bool active, bool need_ll,
                                 double& ll_out, double (*red4)[kMW][4][4], int& rb4, double (*xch4)[4][4],
                                 int& xb4) {
    constexpr int S = Inst<G>::S;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (active)
        for (int64_t k = I.rlo + I.sl; k < I.rhi; k += S) {
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
    if (active && P.conv == C_LANGE && I.rank == 0)
        for (int j = I.sl; j < I.J; j += S) {
            const int pt = P.ptype[j];
            acc[3] += log_prior_one(I.Bt[(size_t)j * G + I.g], pt, pt == 0 ? 1.0 : I.var);
        }
    inst_sum<G, 4>(I, acc, red4, rb4, xch4, xb4);
    const double fixed = (MODEL == M_POISSON && P.ll_fixed && I.exists) ? P.ll_fixed[I.inst] : 0.0;
    ll_out = (acc[0] - acc[1]) + fixed;
    if (P.conv == C_GRADIENT) return acc[2];
    if (P.conv == C_MITTAL) return ll_out;
    return ll_out + acc[3];
}

struct InstCounters {  // kept in shared memory, updated by one thread per instance
    long long steps, updates, upd_entries, gh_entries;
};

// The coordinate step of one instance (ccdUpdateBeta + applyBounds), computed
// identically by every thread of the instance in every CTA of the cluster;
// thread 0 of the instance in rank 0 stores the bound and coefficient.  An
// empty column gives (0, 0) (ModelSpecifics.hpp:720-723).
template <int G>
__device__ __forceinline__ double inst_step(const Inst<G>& I, int j, int ntot, double gsum, double hsum,
                                            double b0, double hd0, double xjy0, int pt, InstCounters& c) {
    double Gv = 0.0, Hv = 0.0;
    if (ntot > 0) {
        Gv = gsum - xjy0;
        Hv = hsum;
    }
    double d = newton_prior_delta_l(Gv, Hv, b0, pt, pt == 0 ? 1.0 : I.var, I.lambda);
    double bnd = hd0;
    d = apply_bounds(d, bnd);
    if (I.sl == 0 && I.rank == 0) {
        I.Hd[(size_t)j * G + I.g] = bnd;
        if (d != 0.0) {
            I.Bt[(size_t)j * G + I.g] = b0 + d;
            ++c.updates;
            c.upd_entries += ntot;
        }
        ++c.steps;
        c.gh_entries += ntot;
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
// rows (getPredictiveLogLikelihood, ModelSpecifics.hpp:652-690), FP64; rank 0
// writes the result.
template <int MODEL, int G>
__device__ void inst_finish(const BatchParams& P, const Inst<G>& I, int flag, int iteration, double last,
                            const InstCounters& c, double (*red4)[kMW][4][4], int& rb4, double (*xch4)[4][4],
                            int& xb4) {
    constexpr int S = Inst<G>::S;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (I.exists)
        for (int64_t k = I.rlo + I.sl; k < I.rhi; k += S) {
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
    inst_sum<G, 4>(I, acc, red4, rb4, xch4, xb4);
    if (I.exists && I.sl == 0 && I.rank == 0) {
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
    // no CTA leaves while another may still read its shared memory
    if (I.C > 1) cooperative_groups::this_cluster().sync();
}
}  // namespace bm
}  // namespace ccdb
