// cox.cu -- Breslow-tied Cox proportional hazards (BreslowTiedCoxProportionalHazards,
// src/cyclops/engine/ModelSpecifics.h:1162-1257) on the device.
//
// Rows are sorted by (stratum, -time, y) and grouped into risk-set tie groups
// exactly as ModelSpecifics::setPidForAccumulation (ModelSpecifics.hpp:1809-1868)
// does; the grouping is integer work done on the host.  Device state:
//   per row   : {xBeta, offsExpXBeta}, weight, group id, stratum
//   per group : denominator (sum of w*exp(xBeta) over the group), accumulated
//               denominator D (segmented prefix sum within the stratum, as
//               computeAccumlatedDenominator, ModelSpecifics.hpp:1670-1715),
//               events nEv (hNWeight), and the segmented suffix sums
//               S1(i) = sum_{i' >= i in stratum} nEv/D, S2(i) = sum nEv/D^2.
//
// Gradient of column j.  The reference walks every group from the column's
// first touched group to the end (ModelSpecifics.hpp:904-964):
//     g = sum_i nEv_i A_i / D_i,   h = sum_i nEv_i (A2_i / D_i - A_i^2 / D_i^2)
// where A_i (A2_i) accumulate the column's numerators within the stratum.
// A_i only changes at the column's touched groups, so with n1(t) the sum of
// w*e*x over the column's rows in group t (n2 with x^2):
//     sum_i nEv_i A_i / D_i   = sum_t n1(t) S1(t)
//     sum_i nEv_i A_i^2/D_i^2 = sum_t S2(t) (A(t)^2 - A(t-)^2)
// (summation by parts; A(t-) is A just before t).  The gradient costs O(nnz_j)
// instead of O(#groups); only a nonzero step pays O(#groups) to refresh D,
// S1 and S2.  Equal in exact arithmetic; rounding differs from the serial loop.
//
// Scans are single-pass decoupled look-back scans that combine only the
// predecessors' local aggregates, in an order fixed by the tile indices, so
// results are bit-identical from run to run.
#include <cstdint>

#include "common.cuh"
#include "cox.h"
#include "group_common.cuh"

namespace ccdb {

namespace {

using namespace grp;

// ------------------------------------------------------------------ gradient
// One CTA per column (cox_column_gh, group_common.cuh).
__global__ void __launch_bounds__(kT) cox_gh_kernel(CoxParams P, const int32_t* cols, int ncols,
                                                     double2* out) {
    __shared__ GhShared S;
    for (int c = blockIdx.x; c < ncols; c += gridDim.x) {
        const double2 r = cox_column_gh(P, cols[c], S);
        if (threadIdx.x == 0) out[c] = r;
    }
}

// ------------------------------------------------------------------ update
// updateXBetaImpl, Cox branch (ModelSpecifics.hpp:1548-1559): per entry
// xBeta += delta*x, e = exp(xBeta), denom[group] += w*e_new - w*e_old, the
// additions applied to each group's denominator in row order.
__global__ void __launch_bounds__(kT) cox_update_kernel(CoxParams P, int j, double delta) {
    __shared__ double s_d[kT];
    __shared__ int32_t s_g[kT];
    const uint8_t f = P.fmt[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
    for (int64_t base = 0; base < n; base += kT) {
        const int64_t p = base + threadIdx.x;
        int32_t grp = -1;
        double dd = 0.0;
        if (p < n) {
            const int64_t k = has_rows ? (int64_t)__ldg(P.rows + cb + p) : p;
            const double x = has_vals ? __ldg(P.vals + vb + p) : 1.0;
            const double2 xe = P.xbe[k];
            const double xb = xe.x + delta * x;
            const double en = row_exp(xb, P.mixed);
            P.xbe[k] = make_double2(xb, en);
            grp = P.grp[k];
            if (P.weighted) {
                const double w = P.w[k];
                dd = w * en - w * xe.y;
            } else {
                dd = en - xe.y;
            }
        }
        s_d[threadIdx.x] = dd;
        s_g[threadIdx.x] = grp;
        __syncthreads();
        // the first entry of each group in this tile applies the group's additions in
        // order; rows dropped by a zero weight (group N) may sit between a group's rows
        bool head = (p < n) && (grp != P.N);
        if (head) {
            for (int q = (int)threadIdx.x - 1; q >= 0; --q) {
                if (s_g[q] == P.N) continue;
                head = (s_g[q] != grp);
                break;
            }
        }
        if (head) {
            double d = P.denom[grp];
            for (int q = threadIdx.x; q < kT && base + q < n; ++q) {
                if (s_g[q] == P.N) continue;
                if (s_g[q] != grp) break;
                d = d + s_d[q];
            }
            P.denom[grp] = d;
        }
        __syncthreads();
    }
}

// computeRemainingStatisticsImpl, Cox branch (ModelSpecifics.hpp:1594-1603):
// e = exp(xBeta) per row; denom[g] = 0 + sum of w*e over the group's rows in row order.
__global__ void cox_exp_kernel(CoxParams P) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P.K;
         k += (int64_t)gridDim.x * blockDim.x) {
        const double xb = P.xbe[k].x;
        P.xbe[k] = make_double2(xb, row_exp(xb, P.mixed));
    }
}

__global__ void cox_denom_kernel(CoxParams P) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < P.N;
         g += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int64_t k = P.grow[g]; k < P.grow[g + 1]; ++k) {
            if (P.grp[k] != g) continue;  // dropped rows inside the range
            const double e = P.xbe[k].y;
            d += P.weighted ? P.w[k] * e : e;
        }
        P.denom[g] = d;
    }
}

// ------------------------------------------------------------------ scans
// Decoupled look-back, aggregates only.  Tile t of the (possibly reversed)
// index space publishes (has_start, tail sum) without waiting; a tile whose
// first element continues a segment sums the tails of its predecessors back to
// the nearest tile holding a segment start, in an order fixed by the indices.
struct ScanStatus {
    double v0, v1;  // tail sums (one or two channels)
};

__device__ __forceinline__ int ld_acquire_i32(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// NCH channels scanned together; REV: suffix scan (index i maps to N-1-i).
template <int NCH, bool REV>
__global__ void __launch_bounds__(kT) cox_scan_kernel(CoxParams P, unsigned* ticket, int* status,
                                                       ScanStatus* tails, int epoch) {
    __shared__ Seg2 s_w0[kW], s_w1[kW];
    __shared__ Seg2 s_agg0, s_agg1;
    __shared__ int s_tile;
    __shared__ double s_e0, s_e1;
    __shared__ int s_need;
    const int64_t N = P.N;
    const int n_tiles = (int)((N + kTile - 1) / kTile);
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int t = s_tile;
    if (t >= n_tiles) return;

    // load kPer consecutive elements per thread
    double v0[kPer], v1[kPer];
    int fl[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int64_t ii = (int64_t)t * kTile + (int64_t)threadIdx.x * kPer + i;
        v0[i] = 0.0;
        v1[i] = 0.0;
        fl[i] = 0;
        if (ii < N) {
            const int64_t g = REV ? (N - 1 - ii) : ii;
            if (!REV) {
                v0[i] = P.denom[g];
                fl[i] = P.gfirst[g];
            } else {
                const double D = P.D[g];
                const double ne = P.nEv[g];
                v0[i] = ne / D;
                v1[i] = ne / (D * D);
                fl[i] = P.glast[g];
            }
        }
    }
    // thread-local segmented scan, then block scan of thread aggregates
    Seg2 a0{fl[0], v0[0]}, a1{fl[0], v1[0]};
#pragma unroll
    for (int i = 1; i < kPer; ++i) {
        a0 = seg_combine(a0, Seg2{fl[i], v0[i]});
        if (NCH == 2) a1 = seg_combine(a1, Seg2{fl[i], v1[i]});
    }
    const Seg2 x0 = a0, x1 = a1;
    Seg2 inc0 = block_seg_scan(x0, s_w0, &s_agg0);
    Seg2 inc1 = x1;
    if (NCH == 2) inc1 = block_seg_scan(x1, s_w1, &s_agg1);
    // exclusive prefix of this thread within the tile
    Seg2 ex0{0, 0.0}, ex1{0, 0.0};
    {
        // recover the exclusive value: inclusive of the previous thread
        __shared__ Seg2 s_inc0[kT], s_inc1[kT];
        s_inc0[threadIdx.x] = inc0;
        if (NCH == 2) s_inc1[threadIdx.x] = inc1;
        __syncthreads();
        if (threadIdx.x > 0) {
            ex0 = s_inc0[threadIdx.x - 1];
            if (NCH == 2) ex1 = s_inc1[threadIdx.x - 1];
        }
        __syncthreads();
    }
    // publish this tile's aggregate
    if (threadIdx.x == 0) {
        tails[t].v0 = s_agg0.v;
        tails[t].v1 = (NCH == 2) ? s_agg1.v : 0.0;
        __threadfence();
        asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(status + t),
                     "r"((epoch << 2) | (s_agg0.f << 1) | 1)
                     : "memory");
        s_need = 0;
        s_e0 = 0.0;
        s_e1 = 0.0;
    }
    __syncthreads();
    // does the tile's first element continue a segment from the left?
    __shared__ int s_first_flag;
    if (threadIdx.x == 0) s_first_flag = fl[0];
    __syncthreads();
    double e0 = 0.0, e1 = 0.0;
    if (t > 0 && !s_first_flag) {
        // warp 0 finds the nearest predecessor holding a segment start
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int start = -1;  // nearest tile index u < t with a start (its tail counts)
            bool failed = false;
            for (int hi = t - 1; hi >= 0 && start < 0 && !failed; hi -= 32) {
                const int u = hi - lane;
                int st = 0;
                if (u >= 0) {
                    const unsigned long long t0 = global_ns();
                    for (;;) {
                        st = ld_acquire_i32(status + u);
                        if ((st & 1) && (st >> 2) == epoch) break;
                        if ((long long)(global_ns() - t0) > P.wait_limit_ns) {
                            failed = true;
                            break;
                        }
                        __nanosleep(20);
                    }
                }
                const bool has = (u >= 0) && !failed && ((st >> 1) & 1);
                const unsigned any_fail = __ballot_sync(0xffffffffu, failed);
                if (any_fail) {
                    failed = true;
                    break;
                }
                const unsigned b = __ballot_sync(0xffffffffu, has);
                if (b) start = hi - (__ffs(b) - 1);
                else if (hi - 31 <= 0) start = 0;  // reached the first tile: sum from there
            }
            if (failed) {
                if (lane == 0) {
                    if (atomicCAS(&P.st->error, 0, E_WAIT_COLUMN) == 0) P.st->error_where = t;
                    atomicExch(&P.st->abort, 1);
                }
            } else {
                // sum tails[start .. t-1]: lane l takes u = start + l, start + l + 32, ...
                double s0 = 0.0, s1 = 0.0;
                for (int u = start + lane; u < t; u += 32) {
                    s0 += __ldcg(&tails[u].v0);
                    if (NCH == 2) s1 += __ldcg(&tails[u].v1);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                }
                if (lane == 0) {
                    s_e0 = s0;
                    s_e1 = s1;
                }
            }
        }
        __syncthreads();
        e0 = s_e0;
        e1 = s_e1;
    }
    // final values: elements before the tile's first start add the carry-in
    Seg2 run0 = ex0, run1 = ex1;
    const bool before_start = !ex0.f;  // no start yet at this thread's first element
    (void)before_start;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int64_t ii = (int64_t)t * kTile + (int64_t)threadIdx.x * kPer + i;
        const Seg2 c0{fl[i], v0[i]}, c1{fl[i], v1[i]};
        run0 = (threadIdx.x == 0 && i == 0) ? c0 : seg_combine(run0, c0);
        if (NCH == 2) run1 = (threadIdx.x == 0 && i == 0) ? c1 : seg_combine(run1, c1);
        double o0 = run0.v, o1 = run1.v;
        if (!run0.f) {  // still in the segment that entered from the left
            o0 += e0;
            o1 += e1;
        }
        if (ii < N) {
            const int64_t g = REV ? (N - 1 - ii) : ii;
            if (!REV) {
                P.D[g] = o0;
            } else {
                P.S1[g] = o0;
                P.S2[g] = o1;
            }
        }
    }
}

// ------------------------------------------------------------------ objective
// {sum w*[y==1]*xBeta, sum nEv*log(D), sum w*y*xBeta, 0} partials per block
// (ModelSpecifics.hpp:103-120, 605-650; SurvivalProjection, ModelSpecifics.h:454-483).
__global__ void __launch_bounds__(kT) cox_objective_kernel(CoxParams P, double2* red) {
    __shared__ double4 s_red4[kW];
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    const int64_t G = gridDim.x, b = blockIdx.x;
    const int64_t k0 = P.K * b / G, k1 = P.K * (b + 1) / G;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const double xb = __ldcg(P.xbe + k).x;
        const double yk = P.y[k];
        const double w = P.weighted ? P.w[k] : 1.0;
        const int yi = (int)yk;
        const double c = (yi != 1) ? 0.0 : xb;
        acc.x += P.weighted ? c * w : c;
        acc.z += P.weighted ? xb * yk * w : xb * yk;
    }
    const int64_t g0 = P.N * b / G, g1 = P.N * (b + 1) / G;
    for (int64_t g = g0 + threadIdx.x; g < g1; g += blockDim.x) acc.y += P.nEv[g] * log(__ldcg(P.D + g));
    acc = block_sum4<kW>(acc, s_red4);
    if (threadIdx.x == 0) {
        red[2 * b] = make_double2(acc.x, acc.y);
        red[2 * b + 1] = make_double2(acc.z, 0.0);
    }
}

// ================================================================== grouped models
// ConditionalLogisticRegression / ConditionalPoissonRegression (GroupedData,
// ModelSpecifics.h:329-342, :712-880): one denominator per stratum, no
// accumulation.  The column's entries are walked in row order; numerators
// accumulate per stratum and each stratum run contributes
// t = numer / denom, g += nEv t, h += nEv t (1 - t) (indicator) or
// nEv (numer2 / denom - t^2) (ModelSpecifics.hpp:1101-1179).  Numerators are
// not weighted; CV weights act through nEv and XjY only.

__global__ void __launch_bounds__(kT) grouped_gh_kernel(CoxParams P, const int32_t* cols, int ncols,
                                                         double2* out) {
    __shared__ GhShared S;
    for (int c = blockIdx.x; c < ncols; c += gridDim.x) {
        const double2 r = grouped_column_gh(P, cols[c], S);
        if (threadIdx.x == 0) out[c] = r;
    }
}

// updateXBetaImpl, non-Cox branch (ModelSpecifics.hpp:1561-1571): the
// stratum denominator takes e_new - e_old per row, in row order.
__global__ void __launch_bounds__(kT) grouped_update_kernel(CoxParams P, int j, double delta) {
    __shared__ double s_d[kT];
    __shared__ int32_t s_g[kT];
    const uint8_t f = P.fmt[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
    for (int64_t base = 0; base < n; base += kT) {
        const int64_t p = base + threadIdx.x;
        int32_t grp = -1;
        double dd = 0.0;
        if (p < n) {
            const int64_t k = has_rows ? (int64_t)__ldg(P.rows + cb + p) : p;
            const double x = has_vals ? __ldg(P.vals + vb + p) : 1.0;
            const double2 xe = P.xbe[k];
            const double xb = xe.x + delta * x;
            const double en = exp(xb);
            P.xbe[k] = make_double2(xb, en);
            grp = P.grp[k];
            dd = en - xe.y;
        }
        s_d[threadIdx.x] = dd;
        s_g[threadIdx.x] = grp;
        __syncthreads();
        if (p < n && (threadIdx.x == 0 || s_g[threadIdx.x - 1] != grp)) {
            double d = P.denom[grp];
            for (int q = threadIdx.x; q < kT && base + q < n && s_g[q] == grp; ++q) d = d + s_d[q];
            P.denom[grp] = d;
        }
        __syncthreads();
    }
}

// computeRemainingStatisticsImpl, non-Cox branch: denom[s] = 0 + sum of e over
// the stratum's rows in row order.  grow holds each stratum's first row.
__global__ void grouped_denom_kernel(CoxParams P) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int64_t k = P.grow[s]; k < P.grow[s + 1]; ++k) d += P.xbe[k].y;
        P.denom[s] = d;
    }
}

// {sum w*y*xBeta, sum nEv*log(denom), sum w*y*xBeta, 0}
__global__ void __launch_bounds__(kT) grouped_objective_kernel(CoxParams P, double2* red) {
    __shared__ double4 s_red4[kW];
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    const int64_t G = gridDim.x, b = blockIdx.x;
    const int64_t k0 = P.K * b / G, k1 = P.K * (b + 1) / G;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        const double xb = __ldcg(P.xbe + k).x;
        const double yk = P.y[k];
        const int yi = (int)yk;
        acc.x += P.weighted ? (yi * xb) * P.w[k] : yi * xb;
        acc.z += P.weighted ? xb * yk * P.w[k] : xb * yk;
    }
    const int64_t g0 = P.N * b / G, g1 = P.N * (b + 1) / G;
    for (int64_t g = g0 + threadIdx.x; g < g1; g += blockDim.x)
        acc.y += P.nEv[g] * log(__ldcg(P.denom + g));
    acc = block_sum4<kW>(acc, s_red4);
    if (threadIdx.x == 0) {
        red[2 * b] = make_double2(acc.x, acc.y);
        red[2 * b + 1] = make_double2(acc.z, 0.0);
    }
}

}  // namespace

// ---------------------------------------------------------------- launchers
int cox_scan_tiles(int64_t N) { return (int)((N + kTile - 1) / kTile); }

cudaError_t launch_cox_gh(const CoxParams& P, const int32_t* cols, int ncols, double2* out,
                          cudaStream_t s) {
    if (ncols <= 0) return cudaSuccess;
    cox_gh_kernel<<<ncols, kT, 0, s>>>(P, cols, ncols, out);
    return cudaGetLastError();
}

cudaError_t launch_cox_update(const CoxParams& P, int j, double delta, cudaStream_t s) {
    cox_update_kernel<<<1, kT, 0, s>>>(P, j, delta);
    return cudaGetLastError();
}

cudaError_t launch_cox_remaining(const CoxParams& P, cudaStream_t s) {
    cox_exp_kernel<<<1184, 256, 0, s>>>(P);
    cox_denom_kernel<<<1184, 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_cox_scans(const CoxParams& P, unsigned* tickets, int* status, void* tails,
                             int epoch, cudaStream_t s) {
    const int nt = cox_scan_tiles(P.N);
    if (nt == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(tickets, 0, 2 * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cox_scan_kernel<1, false><<<nt, kT, 0, s>>>(P, tickets, status, (ScanStatus*)tails, 2 * epoch);
    cox_scan_kernel<2, true><<<nt, kT, 0, s>>>(P, tickets + 1, status + nt, (ScanStatus*)tails + nt,
                                               2 * epoch + 1);
    return cudaGetLastError();
}

size_t cox_tail_bytes() { return sizeof(ScanStatus); }

cudaError_t launch_grouped_gh(const CoxParams& P, const int32_t* cols, int ncols, double2* out,
                              cudaStream_t s) {
    if (ncols <= 0) return cudaSuccess;
    grouped_gh_kernel<<<ncols, kT, 0, s>>>(P, cols, ncols, out);
    return cudaGetLastError();
}

cudaError_t launch_grouped_update(const CoxParams& P, int j, double delta, cudaStream_t s) {
    grouped_update_kernel<<<1, kT, 0, s>>>(P, j, delta);
    return cudaGetLastError();
}

cudaError_t launch_grouped_remaining(const CoxParams& P, cudaStream_t s) {
    cox_exp_kernel<<<1184, 256, 0, s>>>(P);
    grouped_denom_kernel<<<1184, 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_grouped_objective(const CoxParams& P, double2* red, int nblocks, cudaStream_t s) {
    grouped_objective_kernel<<<nblocks, kT, 0, s>>>(P, red);
    return cudaGetLastError();
}

cudaError_t launch_cox_objective(const CoxParams& P, double2* red, int nblocks, cudaStream_t s) {
    cox_objective_kernel<<<nblocks, kT, 0, s>>>(P, red);
    return cudaGetLastError();
}

}  // namespace ccdb
