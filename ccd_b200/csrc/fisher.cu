// fisher.cu -- Fisher information of the current state over a set of columns
// (ModelSpecifics::computeFisherInformation / computeFisherInformationImpl,
// ModelSpecifics.hpp:1203-1337; per-model increments ModelSpecifics.h:485-535,
// 1497-1506).
//
// Entry (a, b) is  sum_k v_k x_ak x_bk  -  [grouped] sum_g c_a(g) c_b(g) / d_g^2
// with v_k the model's per-row factor (LR p/d - (p/d)^2, Poisson p, CLR / CPR /
// Cox p/d_g) and c_a(g) = sum of p x_a over column a's rows in group g.  The
// reference walks every pair of columns with a merge of their row lists; here
// one pass takes up to kFisherSlots columns a: a scatter writes their values
// into a row-major table U[k][slot] (and their per-group sums into C[g][slot]),
// then one CTA per column b gathers U at b's rows, so each column b is read
// once per pass for all slots.  Sums over rows use a fixed order (thread
// stride, then warps in index order), so results repeat bit for bit.
#include <algorithm>

#include "common.cuh"
#include "postfit.h"

namespace ccdb {
namespace {

constexpr int kFT = 256;
constexpr int kFW = kFT / 32;
constexpr int kS = kFisherSlots;

struct ColView {
    int64_t cb, vb, n;
    bool has_rows, has_vals;
};

__device__ __forceinline__ ColView col_view(const FisherParams& P, int j) {
    ColView c;
    const uint8_t f = P.fmt[j];
    c.has_rows = (f == F_SPARSE || f == F_INDICATOR);
    c.has_vals = (f == F_SPARSE || f == F_DENSE);
    c.cb = P.col_ptr[j];
    c.vb = P.val_ptr[j];
    c.n = c.has_rows ? (P.col_ptr[j + 1] - c.cb) : P.K;
    return c;
}

__device__ __forceinline__ int64_t col_row(const FisherParams& P, const ColView& c, int64_t p) {
    return c.has_rows ? (int64_t)__ldg(P.rows + c.cb + p) : p;
}

__device__ __forceinline__ double col_val(const FisherParams& P, const ColView& c, int64_t p) {
    return c.has_vals ? __ldg(P.vals + c.vb + p) : 1.0;
}

__device__ __forceinline__ double warp_sum1(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Slot t = blockIdx.y takes column idx[p0 + t]: U[k][t] = x for its rows and,
// for the grouped models, C[g][t] = sum of offsExpXBeta * x over each run of
// its rows sharing a group (getSubjectSpecificHessianIterator,
// ModelSpecifics.hpp:1245-1266), summed in row order by the run's first entry.
__global__ void __launch_bounds__(kFT) fisher_scatter_kernel(FisherParams P, int p0) {
    const int t = blockIdx.y;
    const ColView c = col_view(P, P.idx[p0 + t]);
    for (int64_t p = (int64_t)blockIdx.x * kFT + threadIdx.x; p < c.n; p += (int64_t)gridDim.x * kFT) {
        const int64_t k = col_row(P, c, p);
        P.U[k * kS + t] = col_val(P, c, p);
        if (!P.grouped) continue;
        const int32_t g = P.grp[k];
        if (g >= P.N) continue;  // a row dropped by a zero weight
        if (p > 0 && P.grp[col_row(P, c, p - 1)] == g) continue;  // not the run's first entry
        double s = 0.0;
        for (int64_t q = p; q < c.n; ++q) {
            const int64_t kq = col_row(P, c, q);
            if (P.grp[kq] != g) break;
            s += P.xbe[kq].y * col_val(P, c, q);
        }
        P.C[(int64_t)g * kS + t] = s;
    }
}

// One CTA per column b = idx[q], q = p0 + blockIdx.x: for every slot t, the
// direct sum over b's rows of v_k * (x_ak * x_bk) and the cross sum of
// (p_k x_bk) * c_a(g_k) / d_g^2, combined as direct - cross the way the
// reference subtracts its cross terms.
__global__ void __launch_bounds__(kFT) fisher_gather_kernel(FisherParams P, int p0, int n_slots) {
    __shared__ double s_red[kFW][2 * kS];
    const int q = p0 + blockIdx.x;
    const ColView c = col_view(P, P.idx[q]);
    double dir[kS], crs[kS];
#pragma unroll
    for (int t = 0; t < kS; ++t) dir[t] = crs[t] = 0.0;
    for (int64_t p = threadIdx.x; p < c.n; p += kFT) {
        const int64_t k = col_row(P, c, p);
        const double x = col_val(P, c, p);
        double u[kS];
        const double2* u2 = reinterpret_cast<const double2*>(P.U + k * kS);
#pragma unroll
        for (int i = 0; i < kS / 2; ++i) {
            const double2 v2 = u2[i];
            u[2 * i] = v2.x;
            u[2 * i + 1] = v2.y;
        }
        if (!P.grouped) {
            const double2 xe = P.row[2 * k];
            double v;
            if (P.model == M_LOGISTIC) {
                const double d = P.row[2 * k + 1].x;
                const double g = xe.y / d;
                v = xe.y / d - g * g;
            } else {
                v = xe.y;
            }
#pragma unroll
            for (int t = 0; t < kS; ++t) dir[t] += v * (u[t] * x);
        } else {
            const int32_t g = P.grp[k];
            if (g >= P.N) continue;
            const double e = P.xbe[k].y;
            const double d = P.gden[g];
            const double v = e / d;
            const double ex = e * x;
            const double dd = d * d;
            const double2* c2 = reinterpret_cast<const double2*>(P.C + (int64_t)g * kS);
#pragma unroll
            for (int i = 0; i < kS / 2; ++i) {
                const double2 cv = c2[i];
                dir[2 * i] += v * (u[2 * i] * x);
                dir[2 * i + 1] += v * (u[2 * i + 1] * x);
                crs[2 * i] += ex * cv.x / dd;
                crs[2 * i + 1] += ex * cv.y / dd;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < kS; ++t) {
        const double a = warp_sum1(dir[t]);
        const double b = warp_sum1(crs[t]);
        if (lane == 0) {
            s_red[wid][t] = a;
            s_red[wid][kS + t] = b;
        }
    }
    __syncthreads();
    if (threadIdx.x < n_slots) {
        const int t = threadIdx.x;
        double direct = 0.0, cross = 0.0;
#pragma unroll
        for (int w = 0; w < kFW; ++w) {
            direct += s_red[w][t];
            cross += s_red[w][kS + t];
        }
        const int a = p0 + t;
        if (q >= a) {
            const double info = direct - cross;
            P.out[(int64_t)a * P.n + q] = info;
            P.out[(int64_t)q * P.n + a] = info;
        }
    }
}

}  // namespace

cudaError_t launch_fisher_scatter(const FisherParams& P, int p0, int n_slots, int64_t max_entries,
                                  cudaStream_t s) {
    if (n_slots <= 0 || n_slots > kS || p0 < 0 || p0 + n_slots > P.n) return cudaErrorInvalidValue;
    const int64_t want = (max_entries + kFT - 1) / kFT;
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 2048));
    fisher_scatter_kernel<<<dim3(gx, n_slots), kFT, 0, s>>>(P, p0);
    return cudaGetLastError();
}

cudaError_t launch_fisher_gather(const FisherParams& P, int p0, int n_slots, cudaStream_t s) {
    if (n_slots <= 0 || n_slots > kS || p0 < 0 || p0 + n_slots > P.n) return cudaErrorInvalidValue;
    fisher_gather_kernel<<<P.n - p0, kFT, 0, s>>>(P, p0, n_slots);
    return cudaGetLastError();
}

}  // namespace ccdb
