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

constexpr int kT = 512;  // threads per CTA
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

// Block-wide inclusive segmented scan of one element per thread; returns the
// inclusive value and writes the block aggregate to *agg (valid after return).
__device__ __forceinline__ Seg2 block_seg_scan(Seg2 x, Seg2* s_w, Seg2* agg) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        Seg2 y;
        y.f = __shfl_up_sync(0xffffffffu, x.f, o);
        y.v = __shfl_up_sync(0xffffffffu, x.v, o);
        if (lane >= o) x = seg_combine(y, x);
    }
    if (lane == 31) s_w[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive scan of the warp aggregates, fixed order
        Seg2 run{0, 0.0};
        for (int w = 0; w < kW; ++w) {
            const Seg2 t = s_w[w];
            s_w[w] = run;
            run = (w == 0) ? t : seg_combine(run, t);
        }
        *agg = run;
    }
    __syncthreads();
    if (wid > 0) x = seg_combine(s_w[wid], x);
    __syncthreads();
    return x;
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
    Seg2 agg, agg2;
    double2 red[kW];
    double red3[kW];
    int32_t key[kT + 1];
    double last, carry1, carry2;
    int32_t last_key, carry_key;
};

// Breslow Cox gradient/Hessian of column j (ModelSpecifics.hpp:904-1020 with
// BreslowTiedCoxProportionalHazards, ModelSpecifics.h:1162-1257) in O(nnz_j)
// through the suffix sums S1, S2: entries are walked in tiles of kT; a
// segmented (by stratum) inclusive scan of n1 over the entries gives A(t) per
// entry; the carry continues across tiles.  Result valid in thread 0.
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
    for (int64_t base = 0; base < n; base += kT) {
        const int64_t p = base + threadIdx.x;
        double n1 = 0.0, n2 = 0.0, s1 = 0.0, s2 = 0.0;
        float n1f = 0.f, n2f = 0.f;
        int32_t key = 0x7fffffff;  // past the end: a segment of its own
        if (p < n) {
            const int64_t k = has_rows ? (int64_t)__ldg(P.rows + cb + p) : p;
            const double x = has_vals ? __ldg(P.vals + vb + p) : 1.0;
            const int32_t grp = P.grp[k];
            const double2 xe = __ldcg(P.xbe + k);
            const double w = P.w[k];
            if (P.mixed) {  // the per-entry terms in FP32
                const float xf = (float)x, ef = (float)xe.y;
                n1f = P.weighted ? (float)w * (ef * xf) : ef * xf;
                if (!ind) n2f = n1f * xf;
                n1 = (double)n1f;
                n2 = (double)n2f;
            } else {
                // incrementNumeratorForGradientImpl (ModelSpecifics.hpp:1433-1449)
                n1 = P.weighted ? w * (xe.y * x) : xe.y * x;
                if (!ind) n2 = P.weighted ? w * (xe.y * x * x) : xe.y * x * x;
            }
            key = P.rstrat[k];
            s1 = __ldcg(P.S1 + grp);  // S1[N] = S2[N] = 0 for dropped rows
            s2 = __ldcg(P.S2 + grp);
        }
        S.key[threadIdx.x] = key;
        __syncthreads();
        const int32_t prev_key = (threadIdx.x == 0) ? carry_key : S.key[threadIdx.x - 1];
        Seg2 e{(threadIdx.x == 0) ? (key != carry_key ? 1 : 0) : (key != prev_key ? 1 : 0), n1};
        if (threadIdx.x == 0 && !e.f) e.v = carry + n1;  // continue the previous tile's run
        const Seg2 r = block_seg_scan(e, S.w, &S.agg);
        const double A_incl = r.v;
        const double A_excl = A_incl - n1;
        if (p < n) {
            if (P.mixed) {
                const float s1f = (float)s1;
                two_sum_f(gs, gc, n1f * s1f);
                two_sum_f(hs, hc, n2f * s1f);
            } else {
                g += n1 * s1;
                h2 += n2 * s1;
            }
            hq += s2 * (A_incl * A_incl - A_excl * A_excl);  // risk-set sums: FP64
        }
        // carry: the value of the last element of this tile
        if (threadIdx.x == kT - 1) {
            S.last = r.v;
            S.last_key = key;
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
    double2 v = warp_sum2(make_double2(g, h2));
    double q = hq;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        S.red[wid] = v;
        S.red3[wid] = q;
    }
    __syncthreads();
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        double G = 0.0, H2 = 0.0, HQ = 0.0;
        for (int w = 0; w < kW; ++w) {
            G += S.red[w].x;
            H2 += S.red[w].y;
            HQ += S.red3[w];
        }
        if (n > 0) {  // empty columns give (0, 0) (ModelSpecifics.hpp:720-723)
            out.x = G - P.xjy[j];
            out.y = (ind ? G : H2) - HQ;
        }
    }
    __syncthreads();
    return out;
}

// ConditionalLogisticRegression / ConditionalPoissonRegression gradient of
// column j (GroupedData, ModelSpecifics.hpp:1101-1179): the column's entries in
// row order, numerators accumulated per stratum; each stratum run contributes
// t = numer / denom, g += nEv t, h += nEv t (1 - t) (indicator) or
// nEv (numer2 / denom - t^2).  Numerators are not weighted; CV weights act
// through nEv and XjY only.  Result valid in thread 0.
__device__ __forceinline__ double2 grouped_column_gh(const CoxParams& P, int j, GhShared& S) {
    const uint8_t f = P.fmt[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
    double g = 0.0, h = 0.0;
    if (threadIdx.x == 0) {
        S.carry1 = 0.0;
        S.carry2 = 0.0;
        S.carry_key = -1;
    }
    __syncthreads();
    for (int64_t base = 0; base < n; base += kT) {
        const int64_t p = base + threadIdx.x;
        double n1 = 0.0, n2 = 0.0;
        int32_t key = 0x7fffffff;
        if (p < n) {
            const int64_t k = has_rows ? (int64_t)__ldg(P.rows + cb + p) : p;
            const double x = has_vals ? __ldg(P.vals + vb + p) : 1.0;
            const double e = __ldcg(P.xbe + k).y;
            n1 = e * x;
            if (!ind) n2 = e * x * x;
            key = P.grp[k];
        }
        S.key[threadIdx.x] = key;
        if (threadIdx.x == 0) S.key[kT] = 0x7fffffff;
        __syncthreads();
        // the run continues across tiles when the next tile starts with the same key
        const int32_t carry_key = S.carry_key;
        const int32_t prev_key = (threadIdx.x == 0) ? carry_key : S.key[threadIdx.x - 1];
        const int start = (key != prev_key) ? 1 : 0;
        Seg2 e1{start, n1}, e2{start, n2};
        if (threadIdx.x == 0 && !start) {
            e1.v = S.carry1 + n1;
            e2.v = S.carry2 + n2;
        }
        __syncthreads();
        const Seg2 r1 = block_seg_scan(e1, S.w, &S.agg);
        const Seg2 r2 = block_seg_scan(e2, S.w2, &S.agg2);
        // last entry of a stratum run (the next entry, possibly in the next tile, differs)
        bool run_end = false;
        if (p < n) {
            if (threadIdx.x < kT - 1) {
                run_end = (S.key[threadIdx.x + 1] != key) || (p + 1 >= n);
            } else if (p + 1 >= n) {
                run_end = true;
            } else {
                // peek the next tile's first key
                const int64_t k2 = has_rows ? (int64_t)__ldg(P.rows + cb + p + 1) : p + 1;
                run_end = (P.grp[k2] != key);
            }
        }
        if (run_end) {
            const double numer = r1.v, numer2 = r2.v;
            const double denom = __ldcg(P.denom + key);
            const double nev = P.nEv[key];
            const double t = numer / denom;
            const double gg = nev * t;
            g += gg;
            if (ind) h += gg * (1.0 - t);
            else h += nev * (numer2 / denom - t * t);
        }
        __syncthreads();
        if (threadIdx.x == kT - 1) {
            S.carry1 = r1.v;
            S.carry2 = r2.v;
            S.carry_key = key;
        }
        __syncthreads();
    }
    double2 v = warp_sum2(make_double2(g, h));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) S.red[wid] = v;
    __syncthreads();
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        double G = 0.0, H = 0.0;
        for (int w = 0; w < kW; ++w) {
            G += S.red[w].x;
            H += S.red[w].y;
        }
        if (n > 0) out = make_double2(G - P.xjy[j], H);
    }
    __syncthreads();
    return out;
}

}  // namespace grp
}  // namespace ccdb
