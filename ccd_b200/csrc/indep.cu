// indep.cu -- coordinate descent for models with independent rows
// (LogisticRegression, PoissonRegression: IndependentData in
// src/cyclops/engine/ModelSpecifics.h:383-395).
//
// Row state lives in HBM as two 16-byte words per row, {xBeta, offsExpXBeta}
// and {denominator, weight}, so a gathered row is one 32-byte sector fetched
// with two 128-bit loads.  The fused sweep kernel is persistent and
// cooperative: each CTA walks its own list of (dependency level, tasks); a task
// reduces the gradient/Hessian of one column (warp, CTA, or a chunk of a long
// column), applies the Newton/prior/bound step on the device and scatters the
// update into xBeta, exp(xBeta) and the denominators.  Levels are ordered by
// per-level arrival counters; the convergence objective is reduced on the
// device after each sweep, so a whole findMode is one launch.
//
// Arithmetic follows the reference's per-entry expressions operation by
// operation (the file is compiled with -fmad=false so no product is fused
// into a sum); only the order of the column reductions differs (a fixed,
// deterministic tree instead of a serial loop).
#include <cstdint>

#include "common.cuh"
#include "indep.h"

namespace ccdb {

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxSplit = 64;

template <int FMT>
__device__ __forceinline__ int64_t entry_row(const int32_t* rows, int64_t cb, int64_t p) {
    if (FMT == F_SPARSE || FMT == F_INDICATOR) return (int64_t)__ldg(rows + cb + p);
    return p;
}
template <int FMT>
__device__ __forceinline__ double entry_val(const double* vals, int64_t vb, int64_t p) {
    if (FMT == F_SPARSE || FMT == F_DENSE) return __ldg(vals + vb + p);
    return 1.0;
}

// Gradient/Hessian contributions of entries [p0,p1) of column j, strided by
// nthr: ModelSpecifics.hpp:1022-1038 with Logistic::incrementGradientAndHessian
// (ModelSpecifics.h:541-568) or PoissonRegression's (ModelSpecifics.h:1509-1543).
// Unweighted fits carry weight 1.0, which leaves every product bit-identical.
template <int MODEL, int FMT>
__device__ __forceinline__ void gh_range(const IndepParams& P, int j, int64_t p0, int64_t p1, int tid,
                                         int nthr, double& g, double& h) {
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    constexpr bool ind = (FMT == F_INDICATOR || FMT == F_INTERCEPT);
#pragma unroll 4
    for (int64_t p = p0 + tid; p < p1; p += nthr) {
        const int64_t k = entry_row<FMT>(P.rows, cb, p);
        const double x = entry_val<FMT>(P.vals, vb, p);
        const double2 a = __ldcg(P.row + 2 * k);      // {xBeta, offsExpXBeta}
        const double2 b = __ldcg(P.row + 2 * k + 1);  // {denominator, weight}
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

// updateXBetaImpl for independent rows (ModelSpecifics.hpp:1561-1571):
// xBeta += delta*x; offsExpXBeta = exp(xBeta); denom += new - old.
template <int FMT>
__device__ __forceinline__ void update_range(const IndepParams& P, int j, int64_t p0, int64_t p1,
                                             int tid, int nthr, double delta) {
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
#pragma unroll 4
    for (int64_t p = p0 + tid; p < p1; p += nthr) {
        const int64_t k = entry_row<FMT>(P.rows, cb, p);
        const double x = entry_val<FMT>(P.vals, vb, p);
        const double2 a = __ldcg(P.row + 2 * k);
        const double2 b = __ldcg(P.row + 2 * k + 1);
        const double xb = a.x + delta * x;
        const double en = exp(xb);
        const double dn = b.x + (en - a.y);
        __stcg(P.row + 2 * k, make_double2(xb, en));
        __stcg(P.row + 2 * k + 1, make_double2(dn, b.y));
    }
}

template <int MODEL>
__device__ __forceinline__ void gh_dispatch(const IndepParams& P, int j, uint8_t f, int64_t p0,
                                            int64_t p1, int tid, int nthr, double& g, double& h) {
    switch (f) {
    case F_INDICATOR: gh_range<MODEL, F_INDICATOR>(P, j, p0, p1, tid, nthr, g, h); break;
    case F_SPARSE: gh_range<MODEL, F_SPARSE>(P, j, p0, p1, tid, nthr, g, h); break;
    case F_DENSE: gh_range<MODEL, F_DENSE>(P, j, p0, p1, tid, nthr, g, h); break;
    default: gh_range<MODEL, F_INTERCEPT>(P, j, p0, p1, tid, nthr, g, h); break;
    }
}

__device__ __forceinline__ void update_dispatch(const IndepParams& P, int j, uint8_t f, int64_t p0,
                                                int64_t p1, int tid, int nthr, double delta) {
    switch (f) {
    case F_INDICATOR: update_range<F_INDICATOR>(P, j, p0, p1, tid, nthr, delta); break;
    case F_SPARSE: update_range<F_SPARSE>(P, j, p0, p1, tid, nthr, delta); break;
    case F_DENSE: update_range<F_DENSE>(P, j, p0, p1, tid, nthr, delta); break;
    default: update_range<F_INTERCEPT>(P, j, p0, p1, tid, nthr, delta); break;
    }
}

// (g, h) of a whole column -> delta; writes beta[j] and hDelta[j].
// Empty columns give (0, 0) (ModelSpecifics.hpp:720-723).
__device__ __forceinline__ double column_step(const IndepParams& P, int j, int64_t entries,
                                              double gsum, double hsum, double beta, double hd,
                                              bool write) {
    double g = 0.0, h = 0.0;
    if (entries > 0) {
        g = gsum - P.xjy[j];
        h = hsum;
    }
    double delta = newton_prior_delta(g, h, beta, P.ptype[j], P.pvar[j]);
    delta = apply_bounds(delta, hd);
    if (write) {
        P.hdelta[j] = hd;
        if (delta != 0.0) P.beta[j] = beta + delta;
    }
    return delta;
}

// Objective terms of the current state: {LL numerator, LL denominator,
// gradient objective, log prior} (ModelSpecifics.hpp:103-120, 605-650;
// JointPrior.h:121-128), reduced over the grid into red[buf*G + cta].
template <int MODEL>
__device__ void objective_partials(const IndepParams& P, int buf, double4* s_red4) {
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    const int64_t G = gridDim.x, b = blockIdx.x;
    const int64_t k0 = P.K * b / G, k1 = P.K * (b + 1) / G;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const double2 a = __ldcg(P.row + 2 * k);
        const double2 dw = __ldcg(P.row + 2 * k + 1);
        const double yk = P.y[k];
        acc.x += (double)((int)yk) * a.x * dw.y;
        if (MODEL == M_LOGISTIC) acc.y += dw.y * log(dw.x);
        else acc.y += dw.y * dw.x;
        acc.z += a.x * yk * dw.y;
    }
    const int64_t j0 = (int64_t)P.J * b / G, j1 = (int64_t)P.J * (b + 1) / G;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x)
        acc.w += log_prior_one(__ldcg(P.beta + j), P.ptype[j], P.pvar[j]);
    acc = block_sum4<kWarps>(acc, s_red4);
    if (threadIdx.x == 0) {
        __stcg(P.red + 2 * (buf * G + b), make_double2(acc.x, acc.y));
        __stcg(P.red + 2 * (buf * G + b) + 1, make_double2(acc.z, acc.w));
    }
}

__device__ __forceinline__ double4 objective_total(const IndepParams& P, int buf) {
    double4 t = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int c = 0; c < (int)gridDim.x; ++c) {
        const double2 u = __ldcg(P.red + 2 * (buf * gridDim.x + c));
        const double2 v = __ldcg(P.red + 2 * (buf * gridDim.x + c) + 1);
        t.x += u.x;
        t.y += u.y;
        t.z += v.x;
        t.w += v.y;
    }
    return t;
}

__device__ __forceinline__ double objective_of(const IndepParams& P, double4 t, double& ll) {
    ll = (t.x - t.y) + P.ll_fixed;
    if (P.conv == C_GRADIENT) return t.z;
    if (P.conv == C_MITTAL) return ll;
    return ll + t.w;
}

// ---------------------------------------------------------------- staged tasks
// A task's entries are staged into registers (row id, value) before its level
// is released: they are immutable, so only the row-state gather remains on the
// dependency chain.  kE entries per thread cover every task the scheduler
// builds (warp tasks <= 32*kE entries, CTA tasks and chunks <= kThreads*kE);
// longer chunks (a column longer than n_cta * kThreads * kE) take the loop path.
constexpr int kE = 8;   // entries per thread of a CTA-level task
constexpr int kEw = 4;  // entries per lane of a warp task (warp tasks <= 128 entries)

template <int N>
struct Staged {
    int32_t k[N];
    double x[N];
};

struct ColMeta {
    double xjy, pvar, beta, hd;
    int32_t ptype;
    int32_t fmt;
};

template <int N>
__device__ __forceinline__ bool stageable(const Task& t, int nthr) {
    return (t.p1 - t.p0) <= N * nthr;
}

// Hint the task's row ids and values into L1 ahead of its level.
__device__ __forceinline__ void prefetch_entries(const IndepParams& P, const Task& t, int tid, int nthr) {
    const uint8_t f = P.fmt[t.col];
    const int64_t cb = P.col_ptr[t.col], vb = P.val_ptr[t.col];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    for (int p = t.p0 + tid * 8; p < t.p1; p += nthr * 8) {  // 8 values per 64-byte stride
        if (has_rows) asm volatile("prefetch.global.L1 [%0];" ::"l"(P.rows + cb + p));
        if (has_vals) asm volatile("prefetch.global.L1 [%0];" ::"l"(P.vals + vb + p));
    }
}

template <int N>
__device__ __forceinline__ void stage_entries(const IndepParams& P, const Task& t, int tid, int nthr,
                                              Staged<N>& s) {
    const uint8_t f = P.fmt[t.col];
    const int64_t cb = P.col_ptr[t.col], vb = P.val_ptr[t.col];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const int p = t.p0 + tid + i * nthr;
        if (p < t.p1) {
            s.k[i] = has_rows ? __ldg(P.rows + cb + p) : p;
            s.x[i] = has_vals ? __ldg(P.vals + vb + p) : 1.0;
        } else {
            s.k[i] = -1;
            s.x[i] = 0.0;
        }
    }
}

__device__ __forceinline__ ColMeta load_meta(const IndepParams& P, int j) {
    ColMeta m;
    m.xjy = P.xjy[j];
    m.pvar = P.pvar[j];
    m.ptype = P.ptype[j];
    m.beta = __ldcg(P.beta + j);
    m.hd = __ldcg(P.hdelta + j);
    m.fmt = P.fmt[j];
    return m;
}

// Hint the row state of staged entries into L2 before the level opens.  L2 is
// the point of coherence, so the lines are current when read after the wait.
template <int N>
__device__ __forceinline__ void prefetch_rows_l2(const IndepParams& P, const Staged<N>& s) {
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (s.k[i] >= 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(P.row + 2 * (int64_t)s.k[i]));
}

// gather + gradient/Hessian of the staged entries; the gathered state stays
// in registers for the update.
template <int MODEL, int N>
__device__ __forceinline__ void staged_gh(const IndepParams& P, bool ind, const Staged<N>& s,
                                          double2 (&A)[N], double (&Dn)[N], double& g, double& h) {
    double Wt[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (s.k[i] >= 0) {
            A[i] = __ldcg(P.row + 2 * (int64_t)s.k[i]);
            const double2 b = __ldcg(P.row + 2 * (int64_t)s.k[i] + 1);
            Dn[i] = b.x;
            Wt[i] = b.y;
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (s.k[i] < 0) continue;
        const double x = s.x[i];
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
}

template <int N>
__device__ __forceinline__ void staged_update(const IndepParams& P, const Staged<N>& s,
                                              const double2 (&A)[N], const double (&Dn)[N],
                                              double delta) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (s.k[i] < 0) continue;
        const double xb = A[i].x + delta * s.x[i];
        const double en = exp(xb);
        const double dn = Dn[i] + (en - A[i].y);
        __stcg(P.row + 2 * (int64_t)s.k[i], make_double2(xb, en));
        __stcg(reinterpret_cast<double*>(P.row + 2 * (int64_t)s.k[i] + 1), dn);
    }
}

// The same gather, gradient/Hessian and update with the gathered row state
// held in shared memory instead of registers: each thread copies its entries'
// two 16-byte state words with cp.async (L2, like the register path's loads)
// into its own slots, waits for its own copies, and computes from there; the
// update reads the same slots.  Slot (i, tid) is g[2 * (i * kThreads + tid)].
__device__ __forceinline__ void cp_async16_cg(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

template <int MODEL, int N>
__device__ __forceinline__ void staged_gh_smem(const IndepParams& P, bool ind, const Staged<N>& s,
                                               double2* gbuf, int tid, double& g, double& h) {
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (s.k[i] >= 0) {
            double2* slot = gbuf + 2 * (i * kThreads + tid);
            cp_async16_cg(slot, P.row + 2 * (int64_t)s.k[i]);
            cp_async16_cg(slot + 1, P.row + 2 * (int64_t)s.k[i] + 1);
        }
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;" ::: "memory");
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (s.k[i] < 0) continue;
        const double2 a = gbuf[2 * (i * kThreads + tid)];
        const double2 b = gbuf[2 * (i * kThreads + tid) + 1];
        const double x = s.x[i];
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

template <int N>
__device__ __forceinline__ void staged_update_smem(const IndepParams& P, const Staged<N>& s,
                                                   const double2* gbuf, int tid, double delta) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (s.k[i] < 0) continue;
        const double2 a = gbuf[2 * (i * kThreads + tid)];
        const double dn0 = gbuf[2 * (i * kThreads + tid) + 1].x;
        const double xb = a.x + delta * s.x[i];
        const double en = exp(xb);
        const double dn = dn0 + (en - a.y);
        __stcg(P.row + 2 * (int64_t)s.k[i], make_double2(xb, en));
        __stcg(reinterpret_cast<double*>(P.row + 2 * (int64_t)s.k[i] + 1), dn);
    }
}

constexpr size_t kGatherSmem = sizeof(double2) * 2 * kThreads * kE;  // 128 KiB

__device__ __forceinline__ double meta_step(const ColMeta& m, int64_t entries, double gsum,
                                            double hsum, double& hd_out) {
    double g = 0.0, h = 0.0;
    if (entries > 0) {
        g = gsum - m.xjy;
        h = hsum;
    }
    double delta = newton_prior_delta(g, h, m.beta, m.ptype, m.pvar);
    double hd = m.hd;
    delta = apply_bounds(delta, hd);
    hd_out = hd;
    return delta;
}

__device__ __forceinline__ void meta_write(const IndepParams& P, int j, const ColMeta& m, double delta,
                                           double hd) {
    P.hdelta[j] = hd;
    if (delta != 0.0) P.beta[j] = m.beta + delta;
}

template <int MODEL>
__global__ void __launch_bounds__(kThreads, 1) indep_sweep_kernel(IndepParams P) {
    __shared__ double4 s_red4[kWarps];
    __shared__ double2 s_red2[kWarps];
    __shared__ double2 s_stash[kMaxSplit];  // {beta, hDelta} of split columns, read before arrival
    __shared__ double s_delta;
    __shared__ int32_t s_fail;
    __shared__ int32_t s_done;
    // staged before a level opens: column metadata (slot kWarps = the CTA-level task)
    // and each lane's entries of its warp task
    __shared__ ColMeta s_meta[kWarps + 1];
    __shared__ Staged<kEw> s_wstage[kThreads];
    extern __shared__ __align__(16) double2 s_gath[];  // gathered row state, kGatherSmem bytes

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    unsigned epoch = 0;
    const int64_t seg0 = P.cta_seg[blockIdx.x], seg1 = P.cta_seg[blockIdx.x + 1];

    // initial objective (findMode: lastObjFunc before the first cycle)
    objective_partials<MODEL>(P, 0, s_red4);
    if (!grid_barrier(P.grid_bar, epoch, P.wait_limit_ns, P.st, &s_fail)) return;
    double last = 0.0;
    if (tid == 0) {
        double ll;
        last = objective_of(P, objective_total(P, 0), ll);
    }

    int iteration = 0;
    for (int it = 0; it < P.max_iter; ++it) {
        for (int64_t si = seg0; si < seg1; ++si) {
            const Seg sg = P.segs[si];
            const Task* T = P.tasks + sg.t0;
            const int n_cl = sg.n_chunk + sg.n_cta;  // CTA-level tasks
            const int qw0 = n_cl, qw1 = qw0 + sg.n_warp;

            // ---- before the level opens: stage everything that is immutable
            Task tc{}, tw{};
            bool c_staged = false, w_has = false, w_staged = false;
            int qw_first = -1;
            if (n_cl > 0) {
                tc = T[0];
                c_staged = stageable<kE>(tc, blockDim.x);
                if (c_staged) {
                    Staged<kE> st;  // row ids for the L2 prefetch; re-read from L1 after the wait
                    stage_entries(P, tc, tid, blockDim.x, st);
                    prefetch_rows_l2(P, st);
                } else {
                    prefetch_entries(P, tc, tid, blockDim.x);
                }
                if (tid == 0) s_meta[kWarps] = load_meta(P, tc.col);
            }
            if (sg.n_warp > 0) {
                // first warp task of this warp (tasks of one segment are few)
                for (int q0 = qw0; q0 < qw1 && qw_first < 0; q0 += 32) {
                    const int q = q0 + lane;
                    const bool mine = (q < qw1) && (T[q].warp == wid);
                    const unsigned bal = __ballot_sync(0xffffffffu, mine);
                    if (bal) qw_first = q0 + __ffs(bal) - 1;
                }
                if (qw_first >= 0) {
                    w_has = true;
                    tw = T[qw_first];
                    w_staged = stageable<kEw>(tw, 32);
                    if (w_staged) {
                        Staged<kEw> st;
                        stage_entries(P, tw, lane, 32, st);
                        prefetch_rows_l2(P, st);
                        s_wstage[tid] = st;
                    } else {
                        prefetch_entries(P, tw, lane, 32);
                    }
                    if (lane == 0) s_meta[wid] = load_meta(P, tw.col);
                }
            }

            // ---- wait for the previous level
            if (P.trace && it == 0 && tid == 0) P.trace[3 * si] = global_ns();
            if (sg.level > 0 && tid == 0) {
                const unsigned target = (unsigned)(it + 1) * (unsigned)P.level_need[sg.level - 1];
                s_fail = wait_geq(P.level_done + sg.level - 1, target, P.wait_limit_ns, P.st,
                                  E_WAIT_LEVEL, sg.level) ? 0 : 1;
            }
            // every segment, level 0 included: the metadata staged above by thread 0
            // (s_meta) and by each warp's lane 0 is read by all threads below
            __syncthreads();
            if (sg.level > 0 && s_fail) return;

            if (P.trace && it == 0 && tid == 0) P.trace[3 * si + 1] = global_ns();
            // ---- phase 1: CTA-level tasks (split-column partials are published, not awaited)
            for (int q = 0; q < n_cl; ++q) {
                const Task t = (q == 0) ? tc : T[q];
                const uint8_t f = (q == 0) ? (uint8_t)s_meta[kWarps].fmt : P.fmt[t.col];
                const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
                const bool staged = (q == 0) && c_staged;
                double g = 0.0, h = 0.0;
                Staged<kE> sc;
                if (staged) {
                    stage_entries(P, t, tid, blockDim.x, sc);  // L1 hits after the prefetch
                    staged_gh_smem<MODEL>(P, ind, sc, s_gath, tid, g, h);
                } else {
                    gh_dispatch<MODEL>(P, t.col, f, t.p0, t.p1, tid, blockDim.x, g, h);
                }
                const double2 s = block_sum2<kWarps>(make_double2(g, h), s_red2);
                if (t.kind == 2) {
                    if (tid == 0) {
                        const ColMeta m = (q == 0) ? s_meta[kWarps] : load_meta(P, t.col);
                        s_stash[q] = make_double2(m.beta, m.hd);
                        __stcg(P.partials + t.part_base + t.chunk, s);
                        red_release_gpu_add(P.col_arrive + t.col, 1u);
                    }
                } else {
                    if (tid == 0) {
                        const ColMeta m = (q == 0) ? s_meta[kWarps] : load_meta(P, t.col);
                        double hd;
                        const double d = meta_step(m, t.p1, s.x, s.y, hd);
                        meta_write(P, t.col, m, d, hd);
                        s_delta = d;
                    }
                    __syncthreads();
                    const double d = s_delta;
                    if (d != 0.0) {
                        if (staged) staged_update_smem(P, sc, s_gath, tid, d);
                        else update_dispatch(P, t.col, f, t.p0, t.p1, tid, blockDim.x, d);
                    }
                    __syncthreads();
                }
            }

            if (P.trace2 && it == 0 && tid == 0) P.trace2[2 * si] = global_ns();
            // ---- phase 2: warp tasks
            if (sg.n_warp > 0) {
                for (int q = (w_has ? qw_first : qw1); q < qw1; ++q) {
                    const Task t = (q == qw_first) ? tw : T[q];
                    if (t.warp != wid) continue;
                    const uint8_t f = (q == qw_first) ? (uint8_t)s_meta[wid].fmt : P.fmt[t.col];
                    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
                    const bool staged = (q == qw_first) && w_staged;
                    double g = 0.0, h = 0.0;
                    Staged<kEw> sw;
                    if (staged) {
                        sw = s_wstage[tid];
                        staged_gh_smem<MODEL>(P, ind, sw, s_gath, tid, g, h);
                    } else {
                        gh_dispatch<MODEL>(P, t.col, f, t.p0, t.p1, lane, 32, g, h);
                    }
                    const double2 s = warp_sum2(make_double2(g, h));
                    double d = 0.0;
                    if (lane == 0) {
                        const ColMeta m = (q == qw_first) ? s_meta[wid] : load_meta(P, t.col);
                        double hd;
                        d = meta_step(m, t.p1, s.x, s.y, hd);
                        meta_write(P, t.col, m, d, hd);
                    }
                    d = __shfl_sync(0xffffffffu, d, 0);
                    if (d != 0.0) {
                        if (staged) staged_update_smem(P, sw, s_gath, tid, d);
                        else update_dispatch(P, t.col, f, t.p0, t.p1, lane, 32, d);
                    }
                }
            }

            if (P.trace2 && it == 0 && lane == 0) atomicMax(P.trace2 + 2 * si + 1, global_ns());
            // ---- phase 3: split columns -- combine partials, step, scatter own chunk
            for (int q = 0; q < sg.n_chunk; ++q) {
                const Task t = (q == 0) ? tc : T[q];
                if (tid == 0) {
                    const unsigned target = (unsigned)(it + 1) * (unsigned)t.nchunks;
                    if (!wait_geq(P.col_arrive + t.col, target, P.wait_limit_ns, P.st, E_WAIT_COLUMN,
                                  t.col)) {
                        s_fail = 1;
                    } else {
                        s_fail = 0;
                        double2 s = make_double2(0.0, 0.0);
                        for (int c = 0; c < t.nchunks; ++c) {
                            const double2 v = __ldcg(P.partials + t.part_base + c);
                            s.x += v.x;
                            s.y += v.y;
                        }
                        ColMeta m = (q == 0) ? s_meta[kWarps] : load_meta(P, t.col);
                        m.beta = s_stash[q].x;  // values read before this CTA arrived
                        m.hd = s_stash[q].y;
                        double hd;
                        const double d = meta_step(m, 1, s.x, s.y, hd);  // split columns are never empty
                        if (t.chunk == 0) meta_write(P, t.col, m, d, hd);
                        s_delta = d;
                    }
                }
                __syncthreads();
                if (s_fail) return;
                const double d = s_delta;
                if (d != 0.0) {
                    if (q == 0 && c_staged) {
                        // re-stage (cache hits) and re-gather this chunk: keeping phase 1's
                        // registers alive across phase 2 would spill
                        Staged<kE> s2;
                        stage_entries(P, t, tid, blockDim.x, s2);
                        double g = 0.0, h = 0.0;
                        staged_gh_smem<MODEL>(P, true, s2, s_gath, tid, g, h);
                        staged_update_smem(P, s2, s_gath, tid, d);
                    } else {
                        update_dispatch(P, t.col, P.fmt[t.col], t.p0, t.p1, tid, blockDim.x, d);
                    }
                }
                __syncthreads();
            }
            __syncthreads();
            if (tid == 0) red_release_gpu_add(P.level_done + sg.level, 1u);
            if (P.trace && it == 0 && tid == 0) P.trace[3 * si + 2] = global_ns();
        }
        // the objective reads every row: wait until the last level is complete
        if (tid == 0) {
            const unsigned target = (unsigned)(it + 1) * (unsigned)P.level_need[P.n_levels - 1];
            s_fail = wait_geq(P.level_done + P.n_levels - 1, target, P.wait_limit_ns, P.st,
                              E_WAIT_LEVEL, P.n_levels - 1) ? 0 : 1;
        }
        __syncthreads();
        if (s_fail) return;
        const int buf = (it + 1) & 1;
        objective_partials<MODEL>(P, buf, s_red4);
        if (!grid_barrier(P.grid_bar, epoch, P.wait_limit_ns, P.st, &s_fail)) return;
        iteration = it + 1;
        if (tid == 0) {
            double ll;
            const double4 tot = objective_total(P, buf);
            const double cur = objective_of(P, tot, ll);
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
            s_done = done;
            if (blockIdx.x == 0) {
                P.st->iterations = iteration;
                P.st->objective = cur;
                P.st->loglik = ll;
                P.st->log_prior = tot.w;
                if (done) P.st->flag = flag;
            }
        }
        __syncthreads();
        if (s_done) break;
    }
}

// ---------------------------------------------------------------- cluster sweep
// One thread-block cluster of C CTAs (one per SM) runs a whole findMode.  The
// levels of the schedule are separated by hardware cluster barriers
// (barrier.cluster.arrive.release / wait.acquire), so a level costs one
// barrier instead of a release/acquire round trip through global counters
// across the whole GPU; a level holding a split column costs two, with the
// CTAs' partial sums of that column exchanged through distributed shared
// memory in between.  Every CTA runs the same sequence of barriers: the level
// count, the per-level split flags and the convergence decision are the same
// in every CTA, so no barrier can be left waiting.  There is no spin-wait.
//
// Per level, a CTA: (before the barrier that opens the level) loads the
// metadata of its first tasks and prefetches their entries and row state;
// then runs its CTA tasks (gather, CTA reduction, step, update), its warp
// tasks (one column per warp) and the gather of its split-column chunks,
// sending each chunk's partial (g, h) to every CTA of the cluster; after the
// second barrier every chunk's CTA sums the C partials in rank order, so all
// of them take the same step, and updates its own chunk.

__device__ __forceinline__ void cl_arrive() { asm volatile("barrier.cluster.arrive.release;" ::: "memory"); }
__device__ __forceinline__ void cl_wait() { asm volatile("barrier.cluster.wait.acquire;" ::: "memory"); }
__device__ __forceinline__ unsigned cl_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// store v into CTA `rank`'s copy of the shared variable at p
__device__ __forceinline__ void st_peer_d2(const void* p, unsigned rank, double2 v) {
    unsigned a = (unsigned)__cvta_generic_to_shared(p), ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(ra), "d"(v.x), "d"(v.y) : "memory");
}

// Look-ahead staging of the cluster sweep: a segment's task records (at most
// kSegTaskCap of them; longer segments read them from global memory) are copied
// into shared memory with cp.async while the previous level runs, and their
// columns' metadata is prefetched into L1 before the barrier that opens them.
constexpr int kSegTaskCap = 128;
constexpr size_t kClusterSmem = kGatherSmem + 2 * kSegTaskCap * sizeof(Task);

__device__ __forceinline__ int seg_tasks(const Seg& sg) { return sg.n_chunk + sg.n_cta + sg.n_warp; }

__device__ __forceinline__ void copy_tasks(const IndepParams& P, const Seg& sg, Task* dst, int tid) {
    const int n = seg_tasks(sg);
    if (n > kSegTaskCap) return;
    const char* src = reinterpret_cast<const char*>(P.tasks + sg.t0);
    char* d = reinterpret_cast<char*>(dst);
    for (int c = tid; c < 2 * n; c += blockDim.x) {  // 16-byte pieces of 32-byte records
        const unsigned a = (unsigned)__cvta_generic_to_shared(d + 16 * c);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(src + 16 * c) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all_tasks() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void prefetch_meta(const IndepParams& P, const Seg& sg, const Task* T, int tid) {
    const int n = seg_tasks(sg);
    for (int q = tid; q < n; q += blockDim.x) {
        const int j = T[q].col;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(P.col_ptr + j));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(P.val_ptr + j));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(P.fmt + j));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(P.xjy + j));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(P.pvar + j));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(P.ptype + j));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(P.beta + j));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(P.hdelta + j));
    }
}

// CTA-wide sum of (g, h) with a fixed combination order, returned to every
// thread with identical bits: warp butterflies, one barrier, then every warp
// combines the kWarps per-warp sums by the same half-warp butterfly.
// red[2][kWarps] alternates buffers (`buf`), so consecutive calls need one
// barrier each.
__device__ __forceinline__ double2 cta_sum2(double2 v, double2 (*red)[kWarps], int& buf) {
    v = warp_sum2(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[buf][wid] = v;
    __syncthreads();
    double2 t = (lane < kWarps) ? red[buf][lane] : make_double2(0.0, 0.0);
#pragma unroll
    for (int o = kWarps / 2; o > 0; o >>= 1) {
        t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
    }
    t.x = __shfl_sync(0xffffffffu, t.x, 0);
    t.y = __shfl_sync(0xffffffffu, t.y, 0);
    buf ^= 1;
    return t;
}

// This CTA's share of the objective terms (rows [K r / C, K (r+1) / C)),
// valid in every thread.
template <int MODEL>
__device__ double4 objective_share(const IndepParams& P, unsigned r, unsigned C, double4* s_red4) {
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    const int64_t k0 = P.K * r / C, k1 = P.K * (r + 1) / C;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const double2 a = __ldcg(P.row + 2 * k);
        const double2 dw = __ldcg(P.row + 2 * k + 1);
        const double yk = P.y[k];
        acc.x += (double)((int)yk) * a.x * dw.y;
        if (MODEL == M_LOGISTIC) acc.y += dw.y * log(dw.x);
        else acc.y += dw.y * dw.x;
        acc.z += a.x * yk * dw.y;
    }
    const int64_t j0 = (int64_t)P.J * r / C, j1 = (int64_t)P.J * (r + 1) / C;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x)
        acc.w += log_prior_one(__ldcg(P.beta + j), P.ptype[j], P.pvar[j]);
    return block_sum4<kWarps>(acc, s_red4);
}

template <int MODEL>
__global__ void __launch_bounds__(kThreads, 1) cluster_sweep_kernel(IndepParams P) {
    __shared__ double4 s_red4[kWarps];
    __shared__ double2 s_red2[2][kWarps];
    __shared__ double2 s_split[kMaxSplit][kMaxClusterSweep];  // [slot][chunk] chunk partials
    __shared__ double2 s_obj[kMaxClusterSweep][2];             // [rank] objective terms
    __shared__ double2 s_stash[kMaxSplit];  // {beta, hDelta} of this CTA's chunks, read in phase A
    __shared__ ColMeta s_meta[kWarps + 1];
    __shared__ Staged<kEw> s_wstage[kThreads];
    // look-ahead: the task records of this CTA's next segment are copied here
    // (cp.async) while the current level runs, and the metadata they point to is
    // prefetched into L1 before the level's barrier
    extern __shared__ __align__(16) double2 s_gath[];
    Task (*s_tasks)[kSegTaskCap] = reinterpret_cast<Task (*)[kSegTaskCap]>(
        reinterpret_cast<char*>(s_gath) + kGatherSmem);  // after the gather slots, in dynamic memory

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const unsigned C = gridDim.x, rank = cl_rank();
    const int64_t seg0 = P.cta_seg[rank], seg1 = P.cta_seg[rank + 1];
    int rb = 0;
    unsigned long long moved = 0;  // nonzero steps written by this thread

    // the objective of the current state, combined in rank order in every CTA
    auto objective_all = [&](double& ll) -> double4 {
        const double4 o = objective_share<MODEL>(P, rank, C, s_red4);
        if (tid < (int)C) {
            st_peer_d2(&s_obj[rank][0], tid, make_double2(o.x, o.y));
            st_peer_d2(&s_obj[rank][1], tid, make_double2(o.z, o.w));
        }
        cl_arrive();
        cl_wait();
        double4 t = make_double4(0.0, 0.0, 0.0, 0.0);
        for (unsigned c = 0; c < C; ++c) {
            t.x += s_obj[c][0].x;
            t.y += s_obj[c][0].y;
            t.z += s_obj[c][1].x;
            t.w += s_obj[c][1].y;
        }
        ll = (t.x - t.y) + P.ll_fixed;
        return t;
    };
    // every CTA of the cluster is running before any shared memory of a peer is written
    cl_arrive();
    cl_wait();
    double ll0;
    const double4 t0 = objective_all(ll0);
    double last = (P.conv == C_GRADIENT) ? t0.z : (P.conv == C_MITTAL ? ll0 : ll0 + t0.w);
    cl_arrive();  // s_obj is read; the first level's wait completes this barrier

    for (int it = 0; it < P.max_iter; ++it) {
        int64_t si = seg0;
        // optional timestamps of the first sweep: per level and CTA, entry, opened, phase A done, released
        unsigned long long* tr = (P.trace && it == 0 && tid == 0) ? P.trace + 4 * (size_t)rank : nullptr;
        // this CTA's current (cseg) and next segments; cseg's tasks sit in s_tasks[tb]
        Seg cseg{}, nxt{};
        cseg.level = nxt.level = -1;
        int tb = 0;
        if (si < seg1) {
            cseg = P.segs[si];
            copy_tasks(P, cseg, s_tasks[tb], tid);
        }
        if (si + 1 < seg1) nxt = P.segs[si + 1];
        for (int L = 0; L < P.n_levels; ++L) {
            if (tr) tr[(size_t)L * 4 * C] = global_ns();
            const bool mine = (cseg.level == L);
            Seg sg{};
            if (mine) {
                sg = cseg;
                cp_async_wait_all_tasks();
                __syncthreads();  // every thread's part of the task copy has landed
            }
            const Task* T = (mine && seg_tasks(sg) <= kSegTaskCap) ? s_tasks[tb] : P.tasks + sg.t0;
            const int n_cl = sg.n_chunk + sg.n_cta;
            const int qw0 = n_cl, qw1 = qw0 + sg.n_warp;

            // ---- before the level opens: immutable entries, metadata of the first tasks
            Task tc{}, tw{};
            bool c_staged = false, w_has = false, w_staged = false;
            int qw_first = -1;
            if (mine) {
                if (n_cl > 0) {
                    tc = T[sg.n_cta > 0 ? sg.n_chunk : 0];  // the first CTA task, else the first chunk
                    c_staged = stageable<kE>(tc, blockDim.x);
                    if (c_staged) {
                        Staged<kE> st;
                        stage_entries(P, tc, tid, blockDim.x, st);
                        prefetch_rows_l2(P, st);
                    } else {
                        prefetch_entries(P, tc, tid, blockDim.x);
                    }
                    if (tid == 0) s_meta[kWarps] = load_meta(P, tc.col);
                }
                if (sg.n_warp > 0) {
                    for (int q0 = qw0; q0 < qw1 && qw_first < 0; q0 += 32) {
                        const int q = q0 + lane;
                        const bool own = (q < qw1) && (T[q].warp == wid);
                        const unsigned bal = __ballot_sync(0xffffffffu, own);
                        if (bal) qw_first = q0 + __ffs(bal) - 1;
                    }
                    if (qw_first >= 0) {
                        w_has = true;
                        tw = T[qw_first];
                        w_staged = stageable<kEw>(tw, 32);
                        if (w_staged) {
                            Staged<kEw> st;
                            stage_entries(P, tw, lane, 32, st);
                            prefetch_rows_l2(P, st);
                            s_wstage[tid] = st;
                        } else {
                            prefetch_entries(P, tw, lane, 32);
                        }
                        if (lane == 0) s_meta[wid] = load_meta(P, tw.col);
                    }
                }
            }
            cl_wait();  // the previous level (or the objective) is complete in every CTA
            if (tr) tr[(size_t)L * 4 * C + 1] = global_ns();
            if (mine) {
                __syncthreads();  // s_meta, s_wstage of this level
                if (nxt.level >= 0) copy_tasks(P, nxt, s_tasks[tb ^ 1], tid);
                // ---- CTA tasks
                for (int q = sg.n_chunk; q < n_cl; ++q) {
                    const Task t = T[q];
                    const bool first = (q == sg.n_chunk);
                    const ColMeta m = first ? s_meta[kWarps] : load_meta(P, t.col);
                    const uint8_t f = (uint8_t)m.fmt;
                    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
                    const bool staged = first ? c_staged : stageable<kE>(t, blockDim.x);
                    double g = 0.0, h = 0.0;
                    Staged<kE> sc;
                    if (staged) {
                        stage_entries(P, t, tid, blockDim.x, sc);
                        staged_gh_smem<MODEL>(P, ind, sc, s_gath, tid, g, h);
                    } else {
                        gh_dispatch<MODEL>(P, t.col, f, t.p0, t.p1, tid, blockDim.x, g, h);
                    }
                    const double2 s = cta_sum2(make_double2(g, h), s_red2, rb);
                    double hd;
                    const double d = meta_step(m, t.p1, s.x, s.y, hd);
                    if (tid == 0) {
                        meta_write(P, t.col, m, d, hd);
                        if (d != 0.0) ++moved;
                    }
                    if (d != 0.0) {
                        if (staged) staged_update_smem(P, sc, s_gath, tid, d);
                        else update_dispatch(P, t.col, f, t.p0, t.p1, tid, blockDim.x, d);
                    }
                }
                // ---- warp tasks
                if (sg.n_warp > 0) {
                    for (int q = (w_has ? qw_first : qw1); q < qw1; ++q) {
                        const Task t = (q == qw_first) ? tw : T[q];
                        if (t.warp != wid) continue;
                        const ColMeta m = (q == qw_first) ? s_meta[wid] : load_meta(P, t.col);
                        const uint8_t f = (uint8_t)m.fmt;
                        const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
                        const bool staged = (q == qw_first) ? w_staged : stageable<kEw>(t, 32);
                        double g = 0.0, h = 0.0;
                        Staged<kEw> sw;
                        if (staged) {
                            if (q == qw_first) sw = s_wstage[tid];
                            else stage_entries(P, t, lane, 32, sw);
                            staged_gh_smem<MODEL>(P, ind, sw, s_gath, tid, g, h);
                        } else {
                            gh_dispatch<MODEL>(P, t.col, f, t.p0, t.p1, lane, 32, g, h);
                        }
                        // the butterfly leaves the same sums in every lane: every lane
                        // takes the same step
                        const double2 s = warp_sum2(make_double2(g, h));
                        double hd;
                        const double d = meta_step(m, t.p1, s.x, s.y, hd);
                        if (lane == 0) {
                            meta_write(P, t.col, m, d, hd);
                            if (d != 0.0) ++moved;
                        }
                        if (d != 0.0) {
                            if (staged) staged_update_smem(P, sw, s_gath, tid, d);
                            else update_dispatch(P, t.col, f, t.p0, t.p1, lane, 32, d);
                        }
                    }
                }
                // ---- split-column chunks: partial sums to every CTA of the cluster
                for (int q = 0; q < sg.n_chunk; ++q) {
                    const Task t = T[q];
                    const ColMeta m = (q == 0 && sg.n_cta == 0) ? s_meta[kWarps] : load_meta(P, t.col);
                    const uint8_t f = (uint8_t)m.fmt;
                    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
                    double g = 0.0, h = 0.0;
                    if (stageable<kE>(t, blockDim.x)) {
                        Staged<kE> sc;
                        stage_entries(P, t, tid, blockDim.x, sc);
                        staged_gh_smem<MODEL>(P, ind, sc, s_gath, tid, g, h);
                    } else {
                        gh_dispatch<MODEL>(P, t.col, f, t.p0, t.p1, tid, blockDim.x, g, h);
                    }
                    const double2 s = cta_sum2(make_double2(g, h), s_red2, rb);
                    if (tid == 0) s_stash[q] = make_double2(m.beta, m.hd);
                    // slot [column's exchange slot][chunk index]: every chunk's CTA adds the
                    // partials in chunk order, whichever ranks the chunks sit on
                    if (tid < (int)C) st_peer_d2(&s_split[t.slot][t.chunk], tid, s);
                }
            }
            if (mine && nxt.level >= 0) {
                cp_async_wait_all_tasks();
                __syncthreads();
                prefetch_meta(P, nxt, seg_tasks(nxt) <= kSegTaskCap ? s_tasks[tb ^ 1] : P.tasks + nxt.t0, tid);
            }
            if (tr) tr[(size_t)L * 4 * C + 2] = global_ns();
            if (P.level_split[L]) {
                cl_arrive();
                cl_wait();  // every chunk's partial has arrived
                if (mine) {
                    for (int q = 0; q < sg.n_chunk; ++q) {
                        const Task t = T[q];
                        double2 s = make_double2(0.0, 0.0);
                        for (int c = 0; c < t.nchunks; ++c) {
                            s.x += s_split[t.slot][c].x;
                            s.y += s_split[t.slot][c].y;
                        }
                        ColMeta m = load_meta(P, t.col);
                        m.beta = s_stash[q].x;  // read before any chunk's CTA could write them
                        m.hd = s_stash[q].y;
                        double hd;
                        const double d = meta_step(m, 1, s.x, s.y, hd);  // split columns are never empty
                        if (t.chunk == 0 && tid == 0) {
                            meta_write(P, t.col, m, d, hd);
                            if (d != 0.0) ++moved;
                        }
                        if (d != 0.0) {
                            const uint8_t f = (uint8_t)m.fmt;
                            if (q == sg.n_chunk - 1 && stageable<kE>(t, blockDim.x)) {
                                // the last chunk's gathered state is still in this thread's slots
                                Staged<kE> s2;
                                stage_entries(P, t, tid, blockDim.x, s2);
                                staged_update_smem(P, s2, s_gath, tid, d);
                            } else {
                                update_dispatch(P, t.col, f, t.p0, t.p1, tid, blockDim.x, d);
                            }
                        }
                    }
                }
            }
            cl_arrive();  // this CTA's updates of level L are released to the cluster
            if (tr) tr[(size_t)L * 4 * C + 3] = global_ns();
            if (mine) {
                ++si;
                cseg = nxt;
                tb ^= 1;
                nxt.level = -1;
                if (si + 1 < seg1) nxt = P.segs[si + 1];
            }
        }
        cl_wait();  // every level of the sweep is complete
        double ll;
        const double4 tot = objective_all(ll);
        const int iteration = it + 1;
        const double cur = (P.conv == C_GRADIENT) ? tot.z : (P.conv == C_MITTAL ? ll : ll + tot.w);
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
        if (rank == 0 && tid == 0) {
            P.st->iterations = iteration;
            P.st->objective = cur;
            P.st->loglik = ll;
            P.st->log_prior = tot.w;
            if (done) P.st->flag = flag;
        }
        if (done) break;  // the same decision in every CTA: no barrier is left open
        cl_arrive();      // s_obj is read; the next sweep's first wait completes this barrier
    }
    if (moved) atomicAdd(&P.st->nonzero_steps, moved);
}

// ---------------------------------------------------------------- per-coordinate kernels

template <int MODEL>
__global__ void __launch_bounds__(256) gh_column_kernel(IndepParams P, int j, int64_t entries,
                                                        int64_t per_block, double2* out) {
    __shared__ double2 s_red2[8];
    const int64_t p0 = per_block * blockIdx.x;
    const int64_t p1 = min(entries, p0 + per_block);
    double g = 0.0, h = 0.0;
    if (p0 < p1) gh_dispatch<MODEL>(P, j, P.fmt[j], p0, p1, threadIdx.x, blockDim.x, g, h);
    const double2 s = block_sum2<8>(make_double2(g, h), s_red2);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// (g, h) of a list of columns, one CTA per column (speculative batches).
template <int MODEL>
__global__ void __launch_bounds__(512) gh_batch_kernel(IndepParams P, const int32_t* cols, int ncols,
                                                       double2* out) {
    __shared__ double2 s_red2[kWarps];
    for (int c = blockIdx.x; c < ncols; c += gridDim.x) {
        const int j = cols[c];
        const uint8_t f = P.fmt[j];
        const int64_t entries = (f == F_DENSE || f == F_INTERCEPT) ? P.K : P.col_ptr[j + 1] - P.col_ptr[j];
        double g = 0.0, h = 0.0;
        gh_dispatch<MODEL>(P, j, f, 0, entries, threadIdx.x, blockDim.x, g, h);
        const double2 s = block_sum2<kWarps>(make_double2(g, h), s_red2);
        if (threadIdx.x == 0)
            out[c] = (entries > 0) ? make_double2(s.x - P.xjy[j], s.y) : make_double2(0.0, 0.0);
    }
}

__global__ void gh_finish_kernel(const double2* parts, int n, const double* xjy, int j,
                                 int64_t entries, double2* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double2 s = make_double2(0.0, 0.0);
        for (int c = 0; c < n; ++c) {
            s.x += parts[c].x;
            s.y += parts[c].y;
        }
        if (entries == 0) s = make_double2(0.0, 0.0);
        else s.x -= xjy[j];
        *out = s;
    }
}

// Each thread handles entries p = tid, tid + nthr, ... of column j.
template <int FMT>
__global__ void update_column_grid(IndepParams P, int j, int64_t entries, double delta) {
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < entries; p += nthr) {
        const int64_t k = entry_row<FMT>(P.rows, cb, p);
        const double x = entry_val<FMT>(P.vals, vb, p);
        const double2 a = P.row[2 * k];
        const double2 b = P.row[2 * k + 1];
        const double xb = a.x + delta * x;
        const double en = exp(xb);
        const double dn = b.x + (en - a.y);
        P.row[2 * k] = make_double2(xb, en);
        P.row[2 * k + 1] = make_double2(dn, b.y);
    }
}

// computeRemainingStatistics for independent rows (ModelSpecifics.hpp:1604-1613):
// e = exp(xBeta); denom = null value (LR 1, Poisson 0) + e.  w = row weight.
__global__ void remaining_stats_kernel(double2* row, const double* xb, const double* w, int64_t K,
                                       double null_denom) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K;
         k += (int64_t)gridDim.x * blockDim.x) {
        const double x = xb ? xb[k] : row[2 * k].x;
        const double e = exp(x);
        const double wk = w ? w[k] : row[2 * k + 1].y;
        row[2 * k] = make_double2(x, e);
        row[2 * k + 1] = make_double2(null_denom + e, wk);
    }
}

template <int MODEL>
__global__ void __launch_bounds__(512) objective_kernel(IndepParams P) {
    __shared__ double4 s_red4[kWarps];
    objective_partials<MODEL>(P, 0, s_red4);
}

__global__ void xjy_kernel(const int64_t* col_ptr, const int32_t* rows, const int64_t* val_ptr,
                           const double* vals, const uint8_t* fmt, const double* y, const double* w,
                           int64_t K, int32_t J, double* xjy) {
    __shared__ double2 s_red2[8];
    for (int j = blockIdx.x; j < J; j += gridDim.x) {
        const uint8_t f = fmt[j];
        const int64_t cb = col_ptr[j], vb = val_ptr[j];
        const int64_t n = (f == F_DENSE || f == F_INTERCEPT) ? K : col_ptr[j + 1] - cb;
        double s = 0.0;
        for (int64_t p = threadIdx.x; p < n; p += blockDim.x) {
            const int64_t k = (f == F_SPARSE || f == F_INDICATOR) ? rows[cb + p] : p;
            const double x = (f == F_SPARSE || f == F_DENSE) ? vals[vb + p] : 1.0;
            s += w ? x * y[k] * w[k] : x * y[k];
        }
        const double2 t = block_sum2<8>(make_double2(s, 0.0), s_red2);
        if (threadIdx.x == 0) xjy[j] = t.x;
    }
}

// xBeta = X beta, per row in increasing column order over the row-major copy
// (the same sequence of additions as the column axpy loop of
// CyclicCoordinateDescent::computeXBeta, .cpp:1452-1470).  With `unit_values`
// every entry of non-zero value counts as 1: the product over an INDICATOR
// transpose (ModelSpecifics::computeXBeta, ModelSpecifics.hpp:313-361).
__global__ void xbeta_csr_kernel(const int64_t* row_ptr, const int32_t* col_idx, const double* val,
                                 const double* beta, int64_t K, int unit_values, double* xb) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K;
         k += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t p = row_ptr[k]; p < row_ptr[k + 1]; ++p) {
            const double b = beta[col_idx[p]];
            if (b == 0.0) continue;
            if (!unit_values) s += b * val[p];
            else if (val[p] != 0.0) s += b;
        }
        xb[k] = s;
    }
}

// xBeta = 0 + b * x for a single dense-like column (x = 1 for an intercept).
__global__ void xbeta_dense_kernel(const double* vals, double b, int64_t K, double* xb) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K;
         k += (int64_t)gridDim.x * blockDim.x)
        xb[k] = 0.0 + b * (vals ? vals[k] : 1.0);
}

}  // namespace

// ---------------------------------------------------------------- launchers

cudaError_t launch_xbeta_dense(const double* vals, double b, int64_t K, double* xb,
                               cudaStream_t stream) {
    xbeta_dense_kernel<<<1184, 256, 0, stream>>>(vals, b, K, xb);
    return cudaGetLastError();
}

int indep_threads() { return kThreads; }
int indep_max_split() { return kMaxSplit; }

static cudaError_t indep_sweep_smem_attr() {
    cudaError_t e = cudaFuncSetAttribute(indep_sweep_kernel<M_LOGISTIC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGatherSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(indep_sweep_kernel<M_POISSON>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kGatherSmem);
}

cudaError_t indep_sweep_occupancy(int model, int* blocks_per_sm) {
    cudaError_t e = indep_sweep_smem_attr();
    if (e != cudaSuccess) return e;
    if (model == M_LOGISTIC)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm,
                                                             indep_sweep_kernel<M_LOGISTIC>,
                                                             kThreads, kGatherSmem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm,
                                                         indep_sweep_kernel<M_POISSON>, kThreads, kGatherSmem);
}

cudaError_t launch_indep_sweep(const IndepParams& P, int n_cta, cudaStream_t stream) {
    void* args[] = {(void*)&P};
    const void* fn = (P.model == M_LOGISTIC) ? (const void*)indep_sweep_kernel<M_LOGISTIC>
                                             : (const void*)indep_sweep_kernel<M_POISSON>;
    cudaError_t e = indep_sweep_smem_attr();
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(n_cta), dim3(kThreads), args, kGatherSmem, stream);
}

template <int MODEL>
static cudaError_t cluster_attrs() {
    static std::atomic<uint64_t> done{0};
    return once_per_device(done, [] {
        cudaError_t e = cudaFuncSetAttribute(cluster_sweep_kernel<MODEL>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmem);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(cluster_sweep_kernel<MODEL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
}

template <int MODEL>
static cudaError_t cluster_config(int C, cudaStream_t stream, cudaLaunchConfig_t& cfg, cudaLaunchAttribute* at) {
    cfg = cudaLaunchConfig_t{};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kClusterSmem;
    cfg.stream = stream;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cluster_attrs<MODEL>();
}

cudaError_t cluster_sweep_max_size(int model, int* cluster) {
    *cluster = 0;
    for (int C = kMaxClusterSweep; C >= 1; C /= 2) {
        cudaLaunchConfig_t cfg;
        cudaLaunchAttribute at[1];
        int n = 0;
        cudaError_t e;
        if (model == M_LOGISTIC) {
            e = cluster_config<M_LOGISTIC>(C, 0, cfg, at);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&n, cluster_sweep_kernel<M_LOGISTIC>, &cfg);
        } else {
            e = cluster_config<M_POISSON>(C, 0, cfg, at);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&n, cluster_sweep_kernel<M_POISSON>, &cfg);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();  // an unsupported size is not an error here: try the next
            continue;
        }
        if (n >= 1) {
            *cluster = C;
            return cudaSuccess;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_cluster_sweep(const IndepParams& P, int C, cudaStream_t stream) {
    if (C < 1 || C > kMaxClusterSweep) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    cudaError_t e;
    if (P.model == M_LOGISTIC) {
        e = cluster_config<M_LOGISTIC>(C, stream, cfg, at);
        if (e != cudaSuccess) return e;
        return cudaLaunchKernelEx(&cfg, cluster_sweep_kernel<M_LOGISTIC>, P);
    }
    e = cluster_config<M_POISSON>(C, stream, cfg, at);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, cluster_sweep_kernel<M_POISSON>, P);
}

cudaError_t launch_indep_gh(const IndepParams& P, int j, int64_t entries, double2* parts,
                            int max_parts, double2* out, cudaStream_t stream) {
    int64_t per_block = 8192;
    int nb = (int)((entries + per_block - 1) / per_block);
    if (nb < 1) nb = 1;
    if (nb > max_parts) {
        nb = max_parts;
        per_block = (entries + nb - 1) / nb;
    }
    if (P.model == M_LOGISTIC)
        gh_column_kernel<M_LOGISTIC><<<nb, 256, 0, stream>>>(P, j, entries, per_block, parts);
    else
        gh_column_kernel<M_POISSON><<<nb, 256, 0, stream>>>(P, j, entries, per_block, parts);
    gh_finish_kernel<<<1, 32, 0, stream>>>(parts, nb, P.xjy, j, entries, out);
    return cudaGetLastError();
}

cudaError_t launch_indep_gh_batch(const IndepParams& P, const int32_t* cols, int ncols, double2* out,
                                  cudaStream_t stream) {
    if (ncols <= 0) return cudaSuccess;
    if (P.model == M_LOGISTIC) gh_batch_kernel<M_LOGISTIC><<<ncols, 512, 0, stream>>>(P, cols, ncols, out);
    else gh_batch_kernel<M_POISSON><<<ncols, 512, 0, stream>>>(P, cols, ncols, out);
    return cudaGetLastError();
}

cudaError_t launch_indep_update(const IndepParams& P, int j, uint8_t fmt, int64_t entries,
                                double delta, cudaStream_t stream) {
    if (entries <= 0) return cudaSuccess;
    int nb = (int)((entries + 255) / 256);
    if (nb > 4096) nb = 4096;
    switch (fmt) {
    case F_INDICATOR: update_column_grid<F_INDICATOR><<<nb, 256, 0, stream>>>(P, j, entries, delta); break;
    case F_SPARSE: update_column_grid<F_SPARSE><<<nb, 256, 0, stream>>>(P, j, entries, delta); break;
    case F_DENSE: update_column_grid<F_DENSE><<<nb, 256, 0, stream>>>(P, j, entries, delta); break;
    default: update_column_grid<F_INTERCEPT><<<nb, 256, 0, stream>>>(P, j, entries, delta); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_remaining_stats(double2* row, const double* xb, const double* w, int64_t K,
                                   double null_denom, cudaStream_t stream) {
    remaining_stats_kernel<<<1184, 256, 0, stream>>>(row, xb, w, K, null_denom);
    return cudaGetLastError();
}

cudaError_t launch_indep_objective(const IndepParams& P, int n_blocks, cudaStream_t stream) {
    if (P.model == M_LOGISTIC) objective_kernel<M_LOGISTIC><<<n_blocks, kThreads, 0, stream>>>(P);
    else objective_kernel<M_POISSON><<<n_blocks, kThreads, 0, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_xjy(const int64_t* col_ptr, const int32_t* rows, const int64_t* val_ptr,
                       const double* vals, const uint8_t* fmt, const double* y, const double* w,
                       int64_t K, int32_t J, double* xjy, cudaStream_t stream) {
    int nb = J < 65535 ? J : 65535;
    if (nb < 1) nb = 1;
    xjy_kernel<<<nb, 256, 0, stream>>>(col_ptr, rows, val_ptr, vals, fmt, y, w, K, J, xjy);
    return cudaGetLastError();
}

cudaError_t launch_xbeta_csr(const int64_t* row_ptr, const int32_t* col_idx, const double* val,
                             const double* beta, int64_t K, double* xb, cudaStream_t stream,
                             int unit_values) {
    xbeta_csr_kernel<<<1184, 256, 0, stream>>>(row_ptr, col_idx, val, beta, K, unit_values, xb);
    return cudaGetLastError();
}

}  // namespace ccdb
