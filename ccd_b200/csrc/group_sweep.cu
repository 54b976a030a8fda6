// group_sweep.cu -- one findMode of the group engine in one persistent launch.
//
// The Breslow Cox model and the grouped models (conditional logistic /
// Poisson) share rows through their risk sets or strata, so their sweep is
// the speculative one of the per-call path, now driven by the device: the
// gradients of a batch of consecutive coordinates are computed together
// against one state (one CTA per column); walking them in visiting order every
// zero step leaves the state unchanged, so each is the gradient the
// sequential cycle (CyclicCoordinateDescent.cpp:1008-1021) would see, and the
// first nonzero step is applied and the batch restarts after it.  Every CTA
// takes the same decision from the same published gradients, so the control
// flow (and every grid barrier) is uniform.
//
// A nonzero step of column j:
//   * the column's rows are split over the CTAs: xBeta += delta x, e = exp,
//     and each row's (weighted) change of e is recorded with its group;
//   * after a barrier, the first row of each group's run adds the run's
//     changes to the group denominator in row order, as updateXBetaImpl does
//     (ModelSpecifics.hpp:1548-1571);
//   * Cox: the accumulated denominators D (a segmented prefix scan within
//     strata, computeAccumlatedDenominator, ModelSpecifics.hpp:1670-1715) and
//     the suffix sums S1 = sum nEv/D, S2 = sum nEv/D^2 behind the O(nnz)
//     gradient are rebuilt by a reduce-then-scan over contiguous group ranges
//     of the CTAs: aggregates, barrier, carry-in in CTA order, barrier.
// A column's bound (hDelta) changes with every step, zero or not; the writes
// of a decision (bounds of the walked columns, the moved coefficient) are
// held back by CTA 0 until the next grid barrier, after every CTA has read
// the old values.  Convergence is tested on the device after each sweep, in
// every CTA from the same partial sums.
//
// Fits a few SMs cover run as one thread-block cluster whose barriers are the
// hardware cluster barrier (no wait to bound); otherwise as a cooperative grid
// whose every wait is a grid barrier bounded by wait_limit_ns (common.cuh): a
// wait that runs out records an error, raises the abort word and all CTAs
// return.
#include <cstdint>

#include "common.cuh"
#include "group_common.cuh"
#include "group_sweep.h"
#include "step.h"

namespace ccdb {

namespace {

using namespace grp;


// Exclusive scan of one Seg3 per thread in thread order (REV: in reverse
// thread order), fixed combination order; *total gets the block aggregate.
template <bool REV>
__device__ __forceinline__ Seg3 block_excl_scan3(Seg3 x, Seg3* s_w, Seg3* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    Seg3 inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        Seg3 y;
        if (!REV) {
            y.f = __shfl_up_sync(0xffffffffu, inc.f, o);
            y.a = __shfl_up_sync(0xffffffffu, inc.a, o);
            y.b = __shfl_up_sync(0xffffffffu, inc.b, o);
            if (lane >= o) inc = seg3_combine(y, inc);
        } else {
            y.f = __shfl_down_sync(0xffffffffu, inc.f, o);
            y.a = __shfl_down_sync(0xffffffffu, inc.a, o);
            y.b = __shfl_down_sync(0xffffffffu, inc.b, o);
            if (lane + o < 32) inc = seg3_combine(y, inc);
        }
    }
    // exclusive within the warp: the neighbour's inclusive value
    Seg3 ex;
    if (!REV) {
        ex.f = __shfl_up_sync(0xffffffffu, inc.f, 1);
        ex.a = __shfl_up_sync(0xffffffffu, inc.a, 1);
        ex.b = __shfl_up_sync(0xffffffffu, inc.b, 1);
    } else {
        ex.f = __shfl_down_sync(0xffffffffu, inc.f, 1);
        ex.a = __shfl_down_sync(0xffffffffu, inc.a, 1);
        ex.b = __shfl_down_sync(0xffffffffu, inc.b, 1);
    }
    const bool first_in_warp = REV ? (lane == 31) : (lane == 0);
    const bool last_in_warp = REV ? (lane == 0) : (lane == 31);
    if (last_in_warp) s_w[wid] = inc;
    __syncthreads();
    if (wid == 0) {  // warp 0: exclusive scan of the warp aggregates in scan order
        const int w = REV ? (kW - 1 - lane) : lane;  // lane q holds the q-th warp in scan order
        Seg3 a = (lane < kW) ? s_w[w] : Seg3{0, 0.0, 0.0};
#pragma unroll
        for (int o = 1; o < kW; o <<= 1) {
            Seg3 y;
            y.f = __shfl_up_sync(0xffffffffu, a.f, o);
            y.a = __shfl_up_sync(0xffffffffu, a.a, o);
            y.b = __shfl_up_sync(0xffffffffu, a.b, o);
            if (lane >= o) a = seg3_combine(y, a);
        }
        Seg3 e;
        e.f = __shfl_up_sync(0xffffffffu, a.f, 1);
        e.a = __shfl_up_sync(0xffffffffu, a.a, 1);
        e.b = __shfl_up_sync(0xffffffffu, a.b, 1);
        if (lane < kW) s_w[w] = (lane == 0) ? Seg3{0, 0.0, 0.0} : e;
        if (lane == kW - 1) *total = a;
    }
    __syncthreads();
    const Seg3 wpre = s_w[wid];
    const bool first_warp = REV ? (wid == kW - 1) : (wid == 0);
    Seg3 out;
    if (first_in_warp) out = first_warp ? Seg3{0, 0.0, 0.0} : wpre;
    else out = first_warp ? ex : seg3_combine(wpre, ex);
    __syncthreads();
    return out;
}

// The CTA aggregates agg[q], q in [lo, hi), combined in ascending q (REV:
// descending q, the suffix direction) by one warp: each lane combines a
// contiguous run of them in scan order, its loads issued together, then the
// lanes' results are combined in lane order by a tree (lane l takes lane
// l + o, o = 1, 2, 4, ...).  Valid in lane 0.  The empty range gives {0, 0, 0}.
template <bool REV>
__device__ __forceinline__ Seg3 warp_agg_combine(const SegAgg* agg, int64_t lo, int64_t hi, bool two) {
    const int lane = threadIdx.x & 31;
    const int64_t n = hi - lo;
    const int64_t m = (n + 31) / 32;
    const int64_t s0 = lane * m, s1 = (s0 + m < n) ? s0 + m : n;
    Seg3 run{0, 0.0, 0.0};
    for (int64_t s = s0; s < s1; s += 4) {
        Seg3 e[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (s + i < s1) {
                const int64_t q = REV ? (hi - 1 - (s + i)) : (lo + s + i);
                e[i] = Seg3{__ldcg(&agg[q].f), __ldcg(&agg[q].v0), two ? __ldcg(&agg[q].v1) : 0.0};
            }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (s + i < s1) run = (s + i == s0) ? e[i] : seg3_combine(run, e[i]);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        Seg3 y;
        y.f = __shfl_down_sync(0xffffffffu, run.f, o);
        y.a = __shfl_down_sync(0xffffffffu, run.a, o);
        y.b = __shfl_down_sync(0xffffffffu, run.b, o);
        if ((lane & (2 * o - 1)) == 0 && lane + o < 32) run = seg3_combine(run, y);
    }
    return run;
}

// Thread t's contiguous share of a CTA's range [lo, hi).
__device__ __forceinline__ void thread_share(int64_t lo, int64_t hi, int64_t& a, int64_t& b) {
    const int64_t len = hi - lo;
    a = lo + len * threadIdx.x / blockDim.x;
    b = lo + len * (threadIdx.x + 1) / blockDim.x;
}

// Up to kCh consecutive groups of a thread's share are loaded before they are
// combined, so a thread has kCh independent loads in flight instead of one
// dependent load per group.
constexpr int kCh = 4;


// Hint the cache lines of elements [a, b) of an array into L1: a thread's
// share of a phase is contiguous, so its lines are all requested at once and
// the phase's loads hit L1 instead of waiting on L2 a chunk at a time.  The
// arrays are read with plain loads after a grid barrier, whose acquire orders
// them after every CTA's writes.
template <typename T>
__device__ __forceinline__ void prefetch_l1(const T* p, int64_t a, int64_t b) {
    if (a >= b) return;
    const uintptr_t lo = reinterpret_cast<uintptr_t>(p + a) & ~(uintptr_t)127;
    const uintptr_t hi = reinterpret_cast<uintptr_t>(p + b);
    for (uintptr_t q = lo; q < hi; q += 128) asm volatile("prefetch.global.L1 [%0];" ::"l"(q));
}

// The forward (prefix) elements {gfirst, denominator} of groups [g, g + n).
__device__ __forceinline__ void load_fwd(const CoxParams& P, int64_t g, int n, int (&f)[kCh], double (&v)[kCh]) {
#pragma unroll
    for (int i = 0; i < kCh; ++i)
        if (i < n) {
            f[i] = P.gfirst[g + i];
            v[i] = P.denom[g + i];
        }
}

// The suffix elements {glast, nEv/D, nEv/D^2} of groups [g, g + n).
__device__ __forceinline__ void load_rev(const CoxParams& P, int64_t g, int n, int (&f)[kCh], double (&a)[kCh],
                                         double (&c)[kCh]) {
    double D[kCh], ne[kCh];
#pragma unroll
    for (int i = 0; i < kCh; ++i)
        if (i < n) {
            f[i] = P.glast[g + i];
            D[i] = P.D[g + i];
            ne[i] = P.nEv[g + i];
        }
#pragma unroll
    for (int i = 0; i < kCh; ++i)
        if (i < n) {
            a[i] = ne[i] / D[i];
            c[i] = ne[i] / (D[i] * D[i]);
        }
}

// Every CTA's writes before it are visible to every CTA after it.  CL: the
// launch is one thread-block cluster and the hardware cluster barrier (release
// / acquire at cluster scope) does it; there is no wait to bound, and no CTA
// leaves the kernel before the others.  Otherwise the bounded grid barrier of
// a cooperative launch; false when its wait ran out.
template <bool CL>
__device__ __forceinline__ bool sync_all(const GroupSweepParams& Q, unsigned& epoch, int32_t* s_fail) {
    if (CL) {
        asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::: "memory");
        return true;
    }
    return grid_barrier(Q.grid_bar, epoch, Q.wait_limit_ns, Q.st, s_fail);
}

// D, S1, S2 rebuilt from the group denominators (Cox).  Three phases separated
// by grid barriers; false when a barrier wait ran out.
template <bool CL>
__device__ bool cox_rebuild(const GroupSweepParams& Q, unsigned& epoch, int32_t* s_fail, Seg3* s_w,
                            Seg3* s_tot, Seg3* s_carry, unsigned long long* trc) {
    const CoxParams& P = Q.P;
    const int64_t G = gridDim.x, b = blockIdx.x;
    const int64_t g0 = P.N * b / G, g1 = P.N * (b + 1) / G;
    int64_t t0, t1;
    thread_share(g0, g1, t0, t1);
    int fl[kCh];
    double va[kCh], vb[kCh];
    // phase 1: aggregate of the CTA's range (prefix direction)
    prefetch_l1(P.gfirst, t0, t1);
    prefetch_l1(P.denom, t0, t1);
    Seg3 mine{0, 0.0, 0.0};
    for (int64_t g = t0; g < t1; g += kCh) {
        const int n = (int)(int)(t1 - g < kCh ? t1 - g : kCh);
        load_fwd(P, g, n, fl, va);
#pragma unroll
        for (int i = 0; i < kCh; ++i)
            if (i < n) {
                const Seg3 e{fl[i], va[i], 0.0};
                mine = (g + i == t0) ? e : seg3_combine(mine, e);
            }
    }
    block_excl_scan3<false>(mine, s_w, s_tot);
    if (threadIdx.x == 0) {
        __stcg(&Q.agg[b].f, s_tot->f);
        __stcg(&Q.agg[b].v0, s_tot->a);
    }
    if (!sync_all<CL>(Q, epoch, s_fail)) return false;
    if (trc) trc[4] = global_ns();
    // phase 2: carry-in from the CTAs before, D of the range; suffix aggregates
    if (threadIdx.x < 32) {
        const Seg3 c = warp_agg_combine<false>(Q.agg, 0, b, false);
        if (threadIdx.x == 0) *s_carry = c;
    }
    __syncthreads();
    Seg3 pre = block_excl_scan3<false>(mine, s_w, s_tot);
    {
        // running value entering this thread's first group
        Seg3 run = (b == 0) ? pre : (threadIdx.x == 0 ? *s_carry : seg3_combine(*s_carry, pre));
        const bool has_run = (b > 0) || (threadIdx.x > 0);
        prefetch_l1(P.glast, t0, t1);
        prefetch_l1(P.nEv, t0, t1);
        // the suffix aggregate of the share from the D just computed: the element of
        // group g is the highest of [t0, g], so it is combined in front
        Seg3 rs{0, 0.0, 0.0};
        for (int64_t g = t0; g < t1; g += kCh) {
            const int n = (int)(int)(t1 - g < kCh ? t1 - g : kCh);
            load_fwd(P, g, n, fl, va);
            int fr[kCh];
            double ne[kCh];
#pragma unroll
            for (int i = 0; i < kCh; ++i)
                if (i < n) {
                    fr[i] = P.glast[g + i];
                    ne[i] = P.nEv[g + i];
                }
#pragma unroll
            for (int i = 0; i < kCh; ++i)
                if (i < n) {
                    const Seg3 e{fl[i], va[i], 0.0};
                    run = (!has_run && g + i == t0) ? e : seg3_combine(run, e);
                    __stcg(P.D + g + i, run.a);
                    const double D = run.a;
                    const Seg3 r{fr[i], ne[i] / D, ne[i] / (D * D)};
                    rs = (g + i == t0) ? r : seg3_combine(r, rs);
                }
        }
        mine = rs;
    }
    block_excl_scan3<true>(mine, s_w, s_tot);
    if (threadIdx.x == 0) {
        __stcg(&Q.agg[G + b].f, s_tot->f);
        __stcg(&Q.agg[G + b].v0, s_tot->a);
        __stcg(&Q.agg[G + b].v1, s_tot->b);
    }
    if (!sync_all<CL>(Q, epoch, s_fail)) return false;
    if (trc) trc[5] = global_ns();
    // phase 3: carry-in from the CTAs after (suffix direction), S1 and S2 of the range
    prefetch_l1(P.D, t0, t1);
    if (threadIdx.x < 32) {
        const Seg3 c = warp_agg_combine<true>(Q.agg + G, b + 1, G, true);
        if (threadIdx.x == 0) *s_carry = c;
    }
    __syncthreads();
    Seg3 suf = block_excl_scan3<true>(mine, s_w, s_tot);
    {
        const bool last_cta = (b == G - 1);
        Seg3 run = last_cta ? suf : (threadIdx.x == kT - 1 ? *s_carry : seg3_combine(*s_carry, suf));
        const bool has_run = !last_cta || (threadIdx.x < kT - 1);
        for (int64_t hi = t1; hi > t0; hi -= kCh) {
            const int64_t g = (hi - kCh > t0 ? hi - kCh : t0);
            const int n = (int)(hi - g);
            load_rev(P, g, n, fl, va, vb);
#pragma unroll
            for (int i = kCh - 1; i >= 0; --i)
                if (i < n) {
                    const Seg3 e{fl[i], va[i], vb[i]};
                    run = (!has_run && g + i == t1 - 1) ? e : seg3_combine(run, e);
                    __stcg(P.S1 + g + i, run.a);
                    __stcg(P.S2 + g + i, run.b);
                }
        }
    }
    return sync_all<CL>(Q, epoch, s_fail);
}

// The staged rebuild: a CTA whose group range holds at most kStageCap groups
// copies the range's inputs into shared memory with coalesced loads (one group
// per thread a step) once, walks its thread-contiguous shares there, and
// writes D, S1, S2 back with coalesced stores.  The direct form above reads
// and writes a thread's contiguous share straight from global memory: each
// warp access then touches 32 lines, and the CTA's load/store transactions,
// not bytes, bound it.
constexpr int kStageCap = 6144;
struct RbStage {
    double a[kStageCap];   // denominators, then D, then S1
    double b[kStageCap];   // nEv, then S2
    int32_t f[kStageCap];  // gfirst
    int32_t g[kStageCap];  // glast
};

template <bool CL>
__device__ bool cox_rebuild_staged(const GroupSweepParams& Q, unsigned& epoch, int32_t* s_fail, Seg3* s_w,
                                   Seg3* s_tot, Seg3* s_carry, RbStage& T, unsigned long long* trc) {
    const CoxParams& P = Q.P;
    const int64_t G = gridDim.x, b = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t g0 = P.N * b / G, g1 = P.N * (b + 1) / G;
    const int n = (int)(g1 - g0);
    int64_t a0, a1;
    thread_share(0, n, a0, a1);  // this thread's contiguous share, as offsets into the range
    const int t0 = (int)a0, t1 = (int)a1;

    // phase 1: the range's inputs into shared memory; the CTA's prefix aggregate
    for (int i = tid; i < n; i += kT) {
        T.f[i] = P.gfirst[g0 + i];
        T.a[i] = P.denom[g0 + i];
        T.g[i] = P.glast[g0 + i];
        T.b[i] = P.nEv[g0 + i];
    }
    __syncthreads();
    Seg3 mine{0, 0.0, 0.0};
    for (int i = t0; i < t1; ++i) {
        const Seg3 e{T.f[i], T.a[i], 0.0};
        mine = (i == t0) ? e : seg3_combine(mine, e);
    }
    block_excl_scan3<false>(mine, s_w, s_tot);
    if (tid == 0) {
        __stcg(&Q.agg[b].f, s_tot->f);
        __stcg(&Q.agg[b].v0, s_tot->a);
    }
    if (!sync_all<CL>(Q, epoch, s_fail)) return false;
    if (trc) trc[4] = global_ns();

    // phase 2: carry-in from the CTAs before, D of the range; suffix aggregates
    if (tid < 32) {
        const Seg3 c = warp_agg_combine<false>(Q.agg, 0, b, false);
        if (tid == 0) *s_carry = c;
    }
    __syncthreads();
    const Seg3 pre = block_excl_scan3<false>(mine, s_w, s_tot);
    {
        Seg3 run = (b == 0) ? pre : (tid == 0 ? *s_carry : seg3_combine(*s_carry, pre));
        const bool has_run = (b > 0) || (tid > 0);
        Seg3 rs{0, 0.0, 0.0};  // the share's suffix aggregate: each group is the highest so far
        for (int i = t0; i < t1; ++i) {
            const Seg3 e{T.f[i], T.a[i], 0.0};
            run = (!has_run && i == t0) ? e : seg3_combine(run, e);
            const double D = run.a;
            T.a[i] = D;
            const double ne = T.b[i];
            const Seg3 r{T.g[i], ne / D, ne / (D * D)};
            rs = (i == t0) ? r : seg3_combine(r, rs);
        }
        mine = rs;
    }
    block_excl_scan3<true>(mine, s_w, s_tot);  // its barriers also order the D written above
    if (tid == 0) {
        __stcg(&Q.agg[G + b].f, s_tot->f);
        __stcg(&Q.agg[G + b].v0, s_tot->a);
        __stcg(&Q.agg[G + b].v1, s_tot->b);
    }
    for (int i = tid; i < n; i += kT) __stcg(P.D + g0 + i, T.a[i]);
    if (!sync_all<CL>(Q, epoch, s_fail)) return false;
    if (trc) trc[5] = global_ns();

    // phase 3: carry-in from the CTAs after (suffix direction), S1 and S2 of the range
    if (tid < 32) {
        const Seg3 c = warp_agg_combine<true>(Q.agg + G, b + 1, G, true);
        if (tid == 0) *s_carry = c;
    }
    __syncthreads();
    const Seg3 suf = block_excl_scan3<true>(mine, s_w, s_tot);
    {
        const bool last_cta = (b == G - 1);
        Seg3 run = last_cta ? suf : (tid == kT - 1 ? *s_carry : seg3_combine(*s_carry, suf));
        const bool has_run = !last_cta || (tid < kT - 1);
        for (int i = t1 - 1; i >= t0; --i) {
            const double D = T.a[i], ne = T.b[i];
            const Seg3 e{T.g[i], ne / D, ne / (D * D)};
            run = (!has_run && i == t1 - 1) ? e : seg3_combine(run, e);
            T.a[i] = run.a;
            T.b[i] = run.b;
        }
    }
    __syncthreads();
    for (int i = tid; i < n; i += kT) {
        __stcg(P.S1 + g0 + i, T.a[i]);
        __stcg(P.S2 + g0 + i, T.b[i]);
    }
    return sync_all<CL>(Q, epoch, s_fail);
}

// This CTA's objective partials {LL numerator, LL denominator, gradient
// objective, log prior} (ModelSpecifics.hpp:103-120, 605-650; JointPrior.h:121-128).
template <bool COX>
__device__ double4 objective_share(const GroupSweepParams& Q, double4* s_red4) {
    const CoxParams& P = Q.P;
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    const int64_t G = gridDim.x, b = blockIdx.x;
    const int64_t k0 = P.K * b / G, k1 = P.K * (b + 1) / G;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const double xb = __ldcg(P.xbe + k).x;
        const double yk = P.y[k];
        const int yi = (int)yk;
        if (COX) {
            const double w = P.weighted ? P.w[k] : 1.0;
            const double c = (yi != 1) ? 0.0 : xb;
            acc.x += P.weighted ? c * w : c;
            acc.z += P.weighted ? xb * yk * w : xb * yk;
        } else {
            acc.x += P.weighted ? (yi * xb) * P.w[k] : yi * xb;
            acc.z += P.weighted ? xb * yk * P.w[k] : xb * yk;
        }
    }
    const int64_t n0 = P.N * b / G, n1 = P.N * (b + 1) / G;
    for (int64_t g = n0 + threadIdx.x; g < n1; g += blockDim.x)
        acc.y += P.nEv[g] * log(__ldcg((COX ? P.D : P.denom) + g));
    const int64_t j0 = (int64_t)Q.J * b / G, j1 = (int64_t)Q.J * (b + 1) / G;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x)
        acc.w += log_prior_one(__ldcg(Q.beta + j), Q.ptype[j], Q.pvar[j]);
    return block_sum4<kW>(acc, s_red4);
}

template <bool COX, bool CL>
__device__ bool objective_all(const GroupSweepParams& Q, unsigned& epoch, int32_t* s_fail, double4* s_red4,
                              double& obj, double& ll, double& lp) {
    const double4 o = objective_share<COX>(Q, s_red4);
    if (threadIdx.x == 0) {
        __stcg(Q.red + 2 * blockIdx.x, make_double2(o.x, o.y));
        __stcg(Q.red + 2 * blockIdx.x + 1, make_double2(o.z, o.w));
    }
    if (!sync_all<CL>(Q, epoch, s_fail)) return false;
    double4 t = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int c = 0; c < (int)gridDim.x; ++c) {
        const double2 u = __ldcg(Q.red + 2 * c), v = __ldcg(Q.red + 2 * c + 1);
        t.x += u.x;
        t.y += u.y;
        t.z += v.x;
        t.w += v.y;
    }
    ll = (t.x - t.y) + Q.ll_fixed;
    lp = t.w;
    obj = (Q.conv == C_GRADIENT) ? t.z : (Q.conv == C_MITTAL ? ll : ll + t.w);
    // every CTA has read the partials before any of them writes the next ones
    return sync_all<CL>(Q, epoch, s_fail);
}

template <bool COX, bool CL>
__global__ void __launch_bounds__(kT, 1) group_sweep_kernel(GroupSweepParams Q) {
    __shared__ GhShared S;
    __shared__ double4 s_red4[kW];
    __shared__ Seg3 s_w3[kW];
    __shared__ Seg3 s_tot, s_carry;
    __shared__ int32_t s_fail;
    __shared__ int32_t s_first;
    __shared__ double s_delta, s_newbeta;
    __shared__ double s_pend_hd[kGroupBatchMax];  // CTA 0: bounds of the last decision
    extern __shared__ __align__(16) unsigned char s_dyn[];  // Cox: the staged rebuild's range (RbStage)

    const CoxParams& P = Q.P;
    const int tid = threadIdx.x;
    const int64_t G = gridDim.x, b = blockIdx.x;
    unsigned epoch = 0;
    int pend_pos = 0, pend_n = 0, pend_col = -1;  // CTA 0's writes held back to the next barrier
    long long n_updates = 0, n_batches = 0;
    unsigned long long* trc = (Q.trace && Q.trace_steps > 0 && b == 0 && tid == 0) ? Q.trace : nullptr;
    int trn = Q.trace_steps;

    // grid barrier, then CTA 0 applies the held-back writes of the last decision
    auto barrier = [&]() -> bool {
        if (!sync_all<CL>(Q, epoch, &s_fail)) return false;
        if (b == 0 && pend_n > 0) {
            for (int i = tid; i < pend_n; i += blockDim.x) Q.hdelta[Q.cols[pend_pos + i]] = s_pend_hd[i];
            if (tid == 0 && pend_col >= 0) Q.beta[pend_col] = s_newbeta;
            __syncthreads();
        }
        pend_n = 0;
        pend_col = -1;
        return true;
    };

    double last, ll, lp;
    if (!objective_all<COX, CL>(Q, epoch, &s_fail, s_red4, last, ll, lp)) return;

    // a batch opens with at most one column per CTA (and at most 32): a CTA's
    // columns are evaluated one after another, and after a nonzero step the
    // next one usually comes within a few columns, so a wider opening batch on
    // a few CTAs mostly computes gradients that are thrown away; a batch of
    // zero steps doubles the next one
    const int batch0 = (int)min((int64_t)32, G);
    int iteration = 0;
    for (int it = 0; it < Q.max_iter; ++it) {
        int pos = 0, batch = batch0;
        while (pos < Q.n_active) {
            const int nb = min(batch, Q.n_active - pos);
            // optional timestamps of the first nonzero steps (CTA 0): batch start, decided,
            // rows updated, denominators updated, rebuild phases 1 and 2 done, rebuilt, next
            if (trc) trc[0] = global_ns();
            // gradients of the batch, one CTA per column; the two halves of gh
            // alternate by batch, so a CTA that is on to the next batch never
            // overwrites values another CTA is still deciding from
            double2* gh = Q.gh + (n_batches & 1) * kGroupBatchMax;
            ++n_batches;
            for (int c = (int)b; c < nb; c += (int)G) {
                const double2 r = COX ? cox_column_gh(P, Q.cols[pos + c], S) : grouped_column_gh(P, Q.cols[pos + c], S);
                if (tid == 0) __stcg(gh + c, r);
            }
            if (!barrier()) return;
            if (trc) trc[1] = global_ns();
            // the decision, in every CTA from the same values: the first nonzero step
            if (tid == 0) s_first = nb;
            __syncthreads();
            double hd_r[kGroupBatchMax / kT];
#pragma unroll
            for (int r = 0; r < kGroupBatchMax / kT; ++r) {
                const int i = tid + r * kT;
                hd_r[r] = 0.0;
                if (i < nb) {
                    const int j = Q.cols[pos + i];
                    const double2 ghv = __ldcg(gh + i);
                    const double b0 = __ldcg(Q.beta + j);
                    double hd = __ldcg(Q.hdelta + j);
                    double d = newton_prior_delta(ghv.x, ghv.y, b0, Q.ptype[j], Q.pvar[j]);
                    d = apply_bounds(d, hd);
                    hd_r[r] = hd;
                    if (d != 0.0) atomicMin(&s_first, i);
                }
            }
            __syncthreads();
            const int first = s_first;
#pragma unroll
            for (int r = 0; r < kGroupBatchMax / kT; ++r) {
                const int i = tid + r * kT;
                if (i < nb && i <= first) {
                    if (b == 0) s_pend_hd[i] = hd_r[r];
                    if (i == first) {  // recompute the step of the moving column: same inputs, same bits
                        const int j = Q.cols[pos + i];
                        const double2 ghv = __ldcg(gh + i);
                        const double b0 = __ldcg(Q.beta + j);
                        double hd = __ldcg(Q.hdelta + j);
                        double d = newton_prior_delta(ghv.x, ghv.y, b0, Q.ptype[j], Q.pvar[j]);
                        d = apply_bounds(d, hd);
                        s_delta = d;
                        s_newbeta = b0 + d;
                    }
                }
            }
            __syncthreads();
            if (b == 0) {
                pend_pos = pos;
                pend_n = (first < nb) ? first + 1 : nb;
                pend_col = (first < nb) ? Q.cols[pos + first] : -1;
            }
            if (first >= nb) {  // every step of the batch was zero: the state is unchanged
                pos += nb;
                batch = min(2 * batch, Q.batch_max);
                continue;
            }
            // ---- the nonzero step of column j: the rows, then the group denominators
            const int j = Q.cols[pos + first];
            const double delta = s_delta;
            ++n_updates;
            {
                const uint8_t f = P.fmt[j];
                const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
                const bool has_vals = (f == F_SPARSE || f == F_DENSE);
                const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
                const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
                // entry p: xBeta += delta x, e = exp, the (weighted) change of e and the group recorded
                auto update_entry = [&](int64_t p, int64_t k, double x, double2 xe, double w, int32_t g) {
                    const double xb = xe.x + delta * x;
                    const double en = row_exp(xb, P.mixed);
                    __stcg(P.xbe + k, make_double2(xb, en));
                    const double dd = (COX && P.weighted) ? w * en - w * xe.y : en - xe.y;
                    __stcg(Q.dd + p, dd);
                    __stcg(Q.ddg + p, g);
                };
                // the first row of each group's run adds the run's changes in row order;
                // rows dropped by a zero weight (group N) may sit inside a run
                auto add_runs = [&](int64_t p0, int64_t p1) {
                    for (int64_t p = p0 + tid; p < p1; p += blockDim.x) {
                        const int32_t g = __ldcg(Q.ddg + p);
                        if (g == P.N) continue;
                        int64_t q = p - 1;
                        while (q >= 0 && __ldcg(Q.ddg + q) == P.N) --q;
                        if (q >= 0 && __ldcg(Q.ddg + q) == g) continue;
                        double d = __ldcg(P.denom + g);
                        for (q = p; q < n; ++q) {
                            const int32_t gq = __ldcg(Q.ddg + q);
                            if (gq == P.N) continue;
                            if (gq != g) break;
                            d = d + __ldcg(Q.dd + q);
                        }
                        __stcg(P.denom + g, d);
                    }
                };
                // rows split over the CTAs
                const int64_t p0 = n * b / G, p1 = n * (b + 1) / G;
                for (int64_t p = p0 + tid; p < p1; p += blockDim.x) {
                    const int64_t k = has_rows ? (int64_t)__ldg(P.rows + cb + p) : p;
                    const double x = has_vals ? __ldg(P.vals + vb + p) : 1.0;
                    update_entry(p, k, x, __ldcg(P.xbe + k), (COX && P.weighted) ? P.w[k] : 1.0, P.grp[k]);
                }
                if (!barrier()) return;
                if (trc) trc[2] = global_ns();
                add_runs(p0, p1);
                if (!barrier()) return;
                if (trc) trc[3] = global_ns();
            }
            if (COX) {
                const bool ok = ((P.N + G - 1) / G <= kStageCap)
                                    ? cox_rebuild_staged<CL>(Q, epoch, &s_fail, s_w3, &s_tot, &s_carry,
                                                             *reinterpret_cast<RbStage*>(s_dyn), trc)
                                    : cox_rebuild<CL>(Q, epoch, &s_fail, s_w3, &s_tot, &s_carry, trc);
                if (!ok) return;
            }
            if (trc) trc[6] = global_ns();
            pos += first + 1;
            if (trc) {
                trc[7] = global_ns();
                trc += kTraceStamps;
                if (--trn <= 0) trc = nullptr;
            }
            batch = batch0;
        }
        // the sweep is complete: held-back writes land, then the objective
        if (!barrier()) return;
        double cur;
        if (!objective_all<COX, CL>(Q, epoch, &s_fail, s_red4, cur, ll, lp)) return;
        iteration = it + 1;
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
        if (Q.tol > 0 && conv < Q.tol) {
            flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
            done = 1;
        } else if (iteration == Q.max_iter) {
            flag = R_MAX_ITERATIONS;
            done = 1;
        }
        if (b == 0 && tid == 0) {
            Q.st->iterations = iteration;
            Q.st->objective = cur;
            Q.st->loglik = ll;
            Q.st->log_prior = lp;
            if (done) Q.st->flag = flag;
        }
        if (done) break;
    }
    if (b == 0 && tid == 0) {
        if (Q.counters) {
            Q.counters[0] = n_updates;
            Q.counters[1] = n_batches;
        }
        Q.st->nonzero_steps = (unsigned long long)n_updates;
    }
}

}  // namespace

int group_sweep_threads() { return kT; }

// The Cox kernels hold the staged rebuild's range in dynamic shared memory;
// the limit is raised, and the cluster-size attribute set, once per device.
cudaError_t group_sweep_attrs() {
    static std::atomic<uint64_t> done{0};
    return once_per_device(done, [] {
        for (const void* fn : {(const void*)group_sweep_kernel<true, false>, (const void*)group_sweep_kernel<true, true>}) {
            cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RbStage));
            if (e != cudaSuccess) return e;
        }
        for (const void* fn : {(const void*)group_sweep_kernel<true, true>, (const void*)group_sweep_kernel<false, true>}) {
            cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

cudaError_t group_sweep_occupancy(int* blocks_per_sm) {
    cudaError_t e = group_sweep_attrs();
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, group_sweep_kernel<true, false>, kT,
                                                         sizeof(RbStage));
}

namespace {
cudaLaunchConfig_t cluster_cfg(int c, cudaStream_t stream, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(kT);
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}
}  // namespace

// The largest cluster (16, 8, 4, 2) of the cluster form of which one can be
// resident; 0 if none.
cudaError_t group_sweep_max_cluster(int* cluster) {
    *cluster = 0;
    cudaError_t e0 = group_sweep_attrs();
    if (e0 != cudaSuccess) return e0;
    for (int c = kMaxGroupCluster; c >= 2; c /= 2) {
        cudaLaunchAttribute attr[1];
        cudaLaunchConfig_t cfg = cluster_cfg(c, 0, attr);
        int n = 0, n2 = 0;
        cfg.dynamicSmemBytes = sizeof(RbStage);
        cudaError_t e = cudaOccupancyMaxActiveClusters(&n, group_sweep_kernel<true, true>, &cfg);
        cfg.dynamicSmemBytes = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&n2, group_sweep_kernel<false, true>, &cfg);
        if (e != cudaSuccess) {
            cudaGetLastError();  // a size the device rejects: try the next one
            continue;
        }
        if (n >= 1 && n2 >= 1) {
            *cluster = c;
            return cudaSuccess;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_group_sweep(const GroupSweepParams& Q, int n_cta, bool cluster, cudaStream_t stream) {
    cudaError_t e = group_sweep_attrs();
    if (e != cudaSuccess) return e;
    const size_t smem = Q.cox ? sizeof(RbStage) : 0;
    if (cluster) {
        cudaLaunchAttribute attr[1];
        cudaLaunchConfig_t cfg = cluster_cfg(n_cta, stream, attr);
        cfg.dynamicSmemBytes = smem;
        if (Q.cox) return cudaLaunchKernelEx(&cfg, group_sweep_kernel<true, true>, Q);
        return cudaLaunchKernelEx(&cfg, group_sweep_kernel<false, true>, Q);
    }
    void* args[] = {(void*)&Q};
    const void* fn = Q.cox ? (const void*)group_sweep_kernel<true, false> : (const void*)group_sweep_kernel<false, false>;
    return cudaLaunchCooperativeKernel(fn, dim3(n_cta), dim3(kT), args, smem, stream);
}

}  // namespace ccdb
