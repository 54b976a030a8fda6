// group_common.cuh -- device pieces shared by the group engine's per-call
// kernels (cox.cu) and its persistent sweep (group_sweep.cu): the segmented
// block scan, and the gradient/Hessian of one column for the Breslow Cox and
// the grouped (conditional logistic / Poisson) models, computed by one CTA.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "cox.h"

namespace ccdb {
namespace grp {

constexpr int kT = 256;  // threads per CTA
constexpr int kW = kT / 32;
constexpr int kPer = 4;           // groups per thread in a scan tile
constexpr int kTile = kPer * kT;  // groups per scan tile

// Segmented-sum operator on (start flag, value): the later element's value
// restarts the sum when it (or anything between) starts a segment.
struct Seg2 {
    int f;
    double v;
};
__device__ __forceinline__ Seg2 seg_combine(Seg2 a, Seg2 b) { return Seg2{a.f | b.f, b.f ? b.v : a.v + b.v}; }

// Inclusive segmented scan across the lanes of a warp, in lane order.
__device__ __forceinline__ Seg2 warp_seg_scan(Seg2 x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        Seg2 y;
        y.f = __shfl_up_sync(0xffffffffu, x.f, o);
        y.v = __shfl_up_sync(0xffffffffu, x.v, o);
        if (lane >= o) x = seg_combine(y, x);
    }
    return x;
}

// Warp 0 replaces the kW warp aggregates s_w[0..kW) by their exclusive
// prefixes (warp order, {0, 0} for warp 0) and writes the block aggregate to
// *agg.  Called by every thread between two barriers.
__device__ __forceinline__ void warps_excl_scan(Seg2* s_w, Seg2* agg) {
    const int lane = threadIdx.x & 31;
    if ((threadIdx.x >> 5) != 0) return;
    const Seg2 inc = warp_seg_scan(lane < kW ? s_w[lane] : Seg2{0, 0.0});
    Seg2 ex;
    ex.f = __shfl_up_sync(0xffffffffu, inc.f, 1);
    ex.v = __shfl_up_sync(0xffffffffu, inc.v, 1);
    if (lane < kW) s_w[lane] = (lane == 0) ? Seg2{0, 0.0} : ex;
    if (lane == kW - 1) *agg = inc;
}

// Block-wide inclusive segmented scan of one element per thread; returns the
// inclusive value and writes the block aggregate to *agg (valid after return).
__device__ __forceinline__ Seg2 block_seg_scan(Seg2 x, Seg2* s_w, Seg2* agg) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    x = warp_seg_scan(x);
    if (lane == 31) s_w[wid] = x;
    __syncthreads();
    warps_excl_scan(s_w, agg);
    __syncthreads();
    if (wid > 0) x = seg_combine(s_w[wid], x);
    __syncthreads();
    return x;
}

// Block-wide exclusive segmented scan of one element per thread ({0, 0} in
// thread 0).
__device__ __forceinline__ Seg2 block_seg_scan_excl(Seg2 x, Seg2* s_w, Seg2* agg) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const Seg2 inc = warp_seg_scan(x);
    Seg2 ex;
    ex.f = __shfl_up_sync(0xffffffffu, inc.f, 1);
    ex.v = __shfl_up_sync(0xffffffffu, inc.v, 1);
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    warps_excl_scan(s_w, agg);
    __syncthreads();
    const Seg2 wpre = s_w[wid];
    const Seg2 out = (lane == 0) ? wpre : (wid == 0 ? ex : seg_combine(wpre, ex));
    __syncthreads();
    return out;
}

// Two-channel segmented sum: (start flag, a, b).
struct Seg3 {
    int f;
    double a, b;
};
__device__ __forceinline__ Seg3 seg3_combine(Seg3 x, Seg3 y) {
    return Seg3{x.f | y.f, y.f ? y.a : x.a + y.a, y.f ? y.b : x.b + y.b};
}

// Inclusive two-channel segmented scan across the lanes of a warp, in lane order.
__device__ __forceinline__ Seg3 warp_seg3_scan(Seg3 x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        Seg3 y;
        y.f = __shfl_up_sync(0xffffffffu, x.f, o);
        y.a = __shfl_up_sync(0xffffffffu, x.a, o);
        y.b = __shfl_up_sync(0xffffffffu, x.b, o);
        if (lane >= o) x = seg3_combine(y, x);
    }
    return x;
}

// Block-wide exclusive two-channel segmented scan of one element per thread
// ({0, 0, 0} in thread 0); s_w holds kW elements.
__device__ __forceinline__ Seg3 block_seg3_scan_excl(Seg3 x, Seg3* s_w) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const Seg3 inc = warp_seg3_scan(x);
    Seg3 ex;
    ex.f = __shfl_up_sync(0xffffffffu, inc.f, 1);
    ex.a = __shfl_up_sync(0xffffffffu, inc.a, 1);
    ex.b = __shfl_up_sync(0xffffffffu, inc.b, 1);
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    if (wid == 0) {  // warp 0: exclusive scan of the warp aggregates
        const Seg3 wi = warp_seg3_scan(lane < kW ? s_w[lane] : Seg3{0, 0.0, 0.0});
        Seg3 we;
        we.f = __shfl_up_sync(0xffffffffu, wi.f, 1);
        we.a = __shfl_up_sync(0xffffffffu, wi.a, 1);
        we.b = __shfl_up_sync(0xffffffffu, wi.b, 1);
        if (lane < kW) s_w[lane] = (lane == 0) ? Seg3{0, 0.0, 0.0} : we;
    }
    __syncthreads();
    const Seg3 wpre = s_w[wid];
    const Seg3 out = (lane == 0) ? wpre : (wid == 0 ? ex : seg3_combine(wpre, ex));
    __syncthreads();
    return out;
}

// Sums of (a, b, c) over the CTA in a fixed order, valid in thread 0: warp
// butterflies, then warp 0 combines the kW warp sums by a butterfly.
__device__ __forceinline__ double3 block_sum3(double a, double b, double c, double3* s_red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) s_red[wid] = make_double3(a, b, c);
    __syncthreads();
    double3 t = make_double3(0.0, 0.0, 0.0);
    if (wid == 0) {
        if (lane < kW) t = s_red[lane];
#pragma unroll
        for (int o = kW / 2; o > 0; o >>= 1) {
            t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
            t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
            t.z += __shfl_xor_sync(0xffffffffu, t.z, o);
        }
    }
    __syncthreads();
    return t;
}

// exp of a row's xBeta: FP64, or in the mixed precision of the Cox engine
// FP32 (expf of the rounded xBeta), kept in the FP64 row state.
__device__ __forceinline__ double row_exp(double xb, int mixed) {
    return mixed ? (double)expf((float)xb) : exp(xb);
}

// Knuth's TwoSum: s + c carries the running FP32 sum with the rounding error
// of every addition kept in c.
__device__ __forceinline__ void two_sum_f(float& s, float& c, float v) {
    const float t = s + v;
    const float bp = t - s;
    c += (s - (t - bp)) + (v - bp);
    s = t;
}

// Shared memory of one CTA computing column gradients.
struct GhShared {
    Seg2 w[kW], w2[kW];
    Seg3 w3[kW];
    Seg2 agg, agg2;
    double2 red[kW];
    double red3[kW];
    double3 sum3[kW];
    int32_t key[kT + 1];
    int32_t key0[kT + 1];
    double last, carry1, carry2;
    int32_t last_key, carry_key;
};

// Breslow Cox gradient/Hessian of column j (ModelSpecifics.hpp:904-1020 with
// BreslowTiedCoxProportionalHazards, ModelSpecifics.h:1162-1257) in O(nnz_j)
// through the suffix sums S1, S2: a segmented (by stratum) inclusive scan of
// n1 over the entries gives A(t) per entry.  The entries are walked in passes
// of kT x kIt, each thread holding kIt consecutive entries, so a thread's
// three rounds of dependent loads (row ids; the row's group, stratum, state
// and weight; the group's suffix sums) are issued for all its entries at once
// and one block scan serves the pass; the carry continues across passes.
// Result valid in thread 0.
constexpr int kIt = 4;  // column entries per thread per pass

__device__ __forceinline__ double2 cox_column_gh(const CoxParams& P, int j, GhShared& S) {
    const uint8_t f = P.fmt[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
    double g = 0.0, h2 = 0.0, hq = 0.0;
    float gs = 0.f, gc = 0.f, hs = 0.f, hc = 0.f;  // mixed: FP32 TwoSum partials of g and h2
    double carry = 0.0;
    int32_t carry_key = -1;
    for (int64_t base = 0; base < n; base += (int64_t)kT * kIt) {
        const int64_t p0 = base + (int64_t)threadIdx.x * kIt;
        int64_t k[kIt];
        double x[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            k[i] = -1;
            x[i] = 1.0;
            if (p0 + i < n) {
                k[i] = has_rows ? (int64_t)__ldg(P.rows + cb + p0 + i) : p0 + i;
                if (has_vals) x[i] = __ldg(P.vals + vb + p0 + i);
            }
        }
        int32_t grp[kIt], key[kIt];
        double e[kIt], w[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            key[i] = 0x7fffffff;  // past the end: a segment of its own
            grp[i] = 0;
            e[i] = 0.0;
            w[i] = 1.0;
            if (k[i] >= 0) {
                grp[i] = P.grp[k[i]];
                key[i] = P.rstrat[k[i]];
                e[i] = __ldcg(P.xbe + k[i]).y;
                if (P.weighted) w[i] = P.w[k[i]];
            }
        }
        double s1[kIt], s2[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            s1[i] = 0.0;
            s2[i] = 0.0;
            if (k[i] >= 0) {
                s1[i] = __ldcg(P.S1 + grp[i]);  // S1[N] = S2[N] = 0 for dropped rows
                s2[i] = __ldcg(P.S2 + grp[i]);
            }
        }
        double n1[kIt], n2[kIt];
        float n1f[kIt], n2f[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            n1[i] = n2[i] = 0.0;
            n1f[i] = n2f[i] = 0.f;
            if (k[i] < 0) continue;
            if (P.mixed) {  // the per-entry terms in FP32
                const float xf = (float)x[i], ef = (float)e[i];
                n1f[i] = P.weighted ? (float)w[i] * (ef * xf) : ef * xf;
                if (!ind) n2f[i] = n1f[i] * xf;
                n1[i] = (double)n1f[i];
                n2[i] = (double)n2f[i];
            } else {
                // incrementNumeratorForGradientImpl (ModelSpecifics.hpp:1433-1449)
                n1[i] = P.weighted ? w[i] * (e[i] * x[i]) : e[i] * x[i];
                if (!ind) n2[i] = P.weighted ? w[i] * (e[i] * x[i] * x[i]) : e[i] * x[i] * x[i];
            }
        }
        // segment starts: the stratum differs from the previous entry's
        S.key[threadIdx.x] = key[kIt - 1];
        __syncthreads();
        int32_t prev = (threadIdx.x == 0) ? carry_key : S.key[threadIdx.x - 1];
        Seg2 loc[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            const Seg2 el{key[i] != prev ? 1 : 0, n1[i]};
            prev = key[i];
            loc[i] = (i == 0) ? el : seg_combine(loc[i - 1], el);
        }
        // the thread's prefix: the previous pass's run, then the threads before
        const Seg2 ex = block_seg_scan_excl(loc[kIt - 1], S.w, &S.agg);
        const Seg2 pre = seg_combine(Seg2{0, carry}, ex);
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            if (k[i] < 0) continue;
            const double A_incl = seg_combine(pre, loc[i]).v;
            const double A_excl = A_incl - n1[i];
            if (P.mixed) {
                const float s1f = (float)s1[i];
                two_sum_f(gs, gc, n1f[i] * s1f);
                two_sum_f(hs, hc, n2f[i] * s1f);
            } else {
                g += n1[i] * s1[i];
                h2 += n2[i] * s1[i];
            }
            hq += s2[i] * (A_incl * A_incl - A_excl * A_excl);  // risk-set sums: FP64
        }
        // carry: the run value and stratum of the pass's last entry
        if (threadIdx.x == kT - 1) {
            S.last = seg_combine(pre, loc[kIt - 1]).v;
            S.last_key = key[kIt - 1];
        }
        __syncthreads();
        carry = S.last;
        carry_key = S.last_key;
        __syncthreads();
    }
    if (P.mixed) {
        g = (double)gs + (double)gc;
        h2 = (double)hs + (double)hc;
    }
    const double3 t = block_sum3(g, h2, hq, S.sum3);
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0 && n > 0) {  // empty columns give (0, 0) (ModelSpecifics.hpp:720-723)
        out.x = t.x - P.xjy[j];
        out.y = (ind ? t.x : t.y) - t.z;
    }
    return out;
}

// ConditionalLogisticRegression / ConditionalPoissonRegression gradient of
// column j (GroupedData, ModelSpecifics.hpp:1101-1179): the column's entries in
// row order, numerators accumulated per stratum; each stratum run contributes
// t = numer / denom, g += nEv t, h += nEv t (1 - t) (indicator) or
// nEv (numer2 / denom - t^2).  Numerators are not weighted; CV weights act
// through nEv and XjY only.  Passes of kT x kIt entries, kIt consecutive
// entries per thread, the loads of each dependent round issued together; one
// two-channel block scan per pass.  Result valid in thread 0.
__device__ __forceinline__ double2 grouped_column_gh(const CoxParams& P, int j, GhShared& S) {
    const uint8_t f = P.fmt[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
    double g = 0.0, h = 0.0;
    double c1 = 0.0, c2 = 0.0;
    int32_t carry_key = -1;
    for (int64_t base = 0; base < n; base += (int64_t)kT * kIt) {
        const int64_t p0 = base + (int64_t)threadIdx.x * kIt;
        int64_t k[kIt];
        double x[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            k[i] = -1;
            x[i] = 1.0;
            if (p0 + i < n) {
                k[i] = has_rows ? (int64_t)__ldg(P.rows + cb + p0 + i) : p0 + i;
                if (has_vals) x[i] = __ldg(P.vals + vb + p0 + i);
            }
        }
        int32_t key[kIt];
        double n1[kIt], n2[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            key[i] = 0x7fffffff;  // past the end: a segment of its own
            n1[i] = n2[i] = 0.0;
            if (k[i] >= 0) {
                const double e = __ldcg(P.xbe + k[i]).y;
                key[i] = P.grp[k[i]];
                n1[i] = e * x[i];
                if (!ind) n2[i] = e * x[i] * x[i];
            }
        }
        // the next pass's first stratum (a run may continue into it)
        int32_t next_pass_key = 0x7fffffff;
        if (threadIdx.x == kT - 1 && base + (int64_t)kT * kIt < n) {
            const int64_t q = base + (int64_t)kT * kIt;
            next_pass_key = P.grp[has_rows ? (int64_t)__ldg(P.rows + cb + q) : q];
        }
        S.key[threadIdx.x] = key[kIt - 1];
        S.key0[threadIdx.x] = key[0];
        __syncthreads();
        int32_t prev = (threadIdx.x == 0) ? carry_key : S.key[threadIdx.x - 1];
        const int32_t after = (threadIdx.x < kT - 1) ? S.key0[threadIdx.x + 1] : next_pass_key;
        Seg3 loc[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            const Seg3 el{key[i] != prev ? 1 : 0, n1[i], n2[i]};
            prev = key[i];
            loc[i] = (i == 0) ? el : seg3_combine(loc[i - 1], el);
        }
        const Seg3 ex = block_seg3_scan_excl(loc[kIt - 1], S.w3);
        const Seg3 pre = seg3_combine(Seg3{0, c1, c2}, ex);
        // the last entry of each stratum run: its group's denominator and event count
        bool end[kIt];
        double dn[kIt], ne[kIt];
#pragma unroll
        for (int i = 0; i < kIt; ++i) {
            const int32_t nk = (i < kIt - 1) ? key[i + 1] : after;
            end[i] = (k[i] >= 0) && (nk != key[i] || p0 + i + 1 >= n);
            if (end[i]) {
                dn[i] = __ldcg(P.denom + key[i]);
                ne[i] = P.nEv[key[i]];
            }
        }
#pragma unroll
        for (int i = 0; i < kIt; ++i)
            if (end[i]) {
                const Seg3 r = seg3_combine(pre, loc[i]);
                const double t = r.a / dn[i];
                const double gg = ne[i] * t;
                g += gg;
                if (ind) h += gg * (1.0 - t);
                else h += ne[i] * (r.b / dn[i] - t * t);
            }
        if (threadIdx.x == kT - 1) {
            const Seg3 r = seg3_combine(pre, loc[kIt - 1]);
            S.carry1 = r.a;
            S.carry2 = r.b;
            S.carry_key = key[kIt - 1];
        }
        __syncthreads();
        c1 = S.carry1;
        c2 = S.carry2;
        carry_key = S.carry_key;
        __syncthreads();
    }
    const double3 t = block_sum3(g, h, 0.0, S.sum3);
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0 && n > 0) out = make_double2(t.x - P.xjy[j], t.y);
    return out;
}

}  // namespace grp
}  // namespace ccdb
