// mm.cu -- the MM algorithm's step over every coordinate at once
// (CyclicCoordinateDescent::mmUpdateAllBeta, CyclicCoordinateDescent.cpp:1354-1391,
// over ModelSpecifics::computeMMGradientAndHessian(Impl), ModelSpecifics.hpp:776-889).
//
// Every free column's (g, h) comes from the same state, so the J columns are
// independent: one CTA per column reduces over the column's entries in a
// fixed order, and its thread 0 applies the clamp h < 0 -> (0, 0) and the
// prior's closed-form step (JointPrior::getDelta), with no trust-region bound
// (the reference's MM cycle leaves applyBounds out, .cpp:984-987).  xBeta is
// then recomputed from beta by the row-major product (launch_xbeta_csr).
#include "common.cuh"
#include "mm.h"

namespace ccdb {
namespace {

constexpr int kMT = 256;

// incrementMMGradientAndHessian of the Survival models (ModelSpecifics.h:499-516,
// the conditional and Cox models): weight = hNWeight and denominator =
// denomPid of the row's group; indicator columns drop x.
__global__ void __launch_bounds__(kMT) mm_gh_kernel(MMParams P) {
    __shared__ double2 s_red[kMT / 32];
    const int j = blockIdx.x;
    if (P.fixed && P.fixed[j]) {
        if (threadIdx.x == 0) P.gh[j] = make_double2(0.0, 0.0);
        return;
    }
    const uint8_t f = P.fmt[j];
    const bool has_rows = (f == F_SPARSE || f == F_INDICATOR);
    const bool has_vals = (f == F_SPARSE || f == F_DENSE);
    const bool ind = (f == F_INDICATOR || f == F_INTERCEPT);
    const int64_t cb = P.col_ptr[j], vb = P.val_ptr[j];
    const int64_t n = has_rows ? (P.col_ptr[j + 1] - cb) : P.K;
    double g = 0.0, h = 0.0;
    for (int64_t p = threadIdx.x; p < n; p += kMT) {
        const int64_t k = has_rows ? (int64_t)__ldg(P.rows + cb + p) : p;
        const int32_t grp = P.grp[k];
        const double weight = P.nEv[grp], e = P.xbe[k].y, d = P.denom[grp];
        if (ind) {
            g += weight * e / d;
            h += weight * e / d;
        } else {
            const double x = has_vals ? __ldg(P.vals + vb + p) : 1.0;
            g += weight * e * x / d;
            h += weight * e * x * x / d;
        }
    }
    const double2 t = block_sum2<kMT / 32>(make_double2(g, h), s_red);
    if (threadIdx.x == 0) {
        const double gj = t.x - P.xjy[j];  // precomputeGradient
        P.gh[j] = make_double2(gj, t.y);
        if (P.step) {
            const double b = P.beta[j];
            const double delta = newton_prior_delta(gj, t.y, b, P.ptype[j], P.pvar[j]);
            if (delta != 0.0) P.beta[j] = b + delta;
        }
    }
}

}  // namespace

cudaError_t launch_mm_gradient_hessian(const MMParams& P, cudaStream_t s) {
    if (P.J <= 0) return cudaSuccess;
    mm_gh_kernel<<<P.J, kMT, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace ccdb
