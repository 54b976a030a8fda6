// predict.cu -- predictive log-likelihood on held-out weights and the per-row
// predictions of the current state (ModelSpecifics::getPredictiveLogLikelihood /
// getPredictiveEstimates, ModelSpecifics.hpp:652-705).
#include <algorithm>

#include "common.cuh"
#include "postfit.h"

namespace ccdb {
namespace {

constexpr int kPT = 256;

__device__ __forceinline__ double row_xbeta(const PredictParams& P, int64_t k) {
    return P.grouped ? P.xbe[k].x : P.row[2 * k].x;
}

// logPredLikeContrib of each model (ModelSpecifics.h:784-795 CPR, 867-873 CLR,
// 1002-1009 LR, 1243-1251 Breslow Cox, 1583-1590 Poisson):
//   LR           y w (xb - log denom_k)
//   Poisson      (y xb - exp(xb)) w
//   CLR, CPR     y w (xb - log denom_stratum)
//   Cox          w == 0 ? 0 : y w (xb - log accDenom_group)
__global__ void __launch_bounds__(kPT) predictive_ll_kernel(PredictParams P, double* part) {
    __shared__ double2 s_red[kPT / 32];
    double acc = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * kPT + threadIdx.x; k < P.K; k += (int64_t)gridDim.x * kPT) {
        const double y = P.y[k], w = P.w[k];
        switch (P.model) {
            case M_LOGISTIC:
                acc += y * w * (P.row[2 * k].x - log(P.row[2 * k + 1].x));
                break;
            case M_POISSON: {
                const double xb = P.row[2 * k].x;
                acc += (y * xb - exp(xb)) * w;
                break;
            }
            case M_COX:
                if (w != 0.0) acc += y * w * (P.xbe[k].x - log(P.gden[P.grp[k]]));
                break;
            default:  // CLR, CPR
                acc += y * w * (P.xbe[k].x - log(P.gden[P.grp[k]]));
        }
    }
    const double2 t = block_sum2<kPT / 32>(make_double2(acc, 0.0), s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = t.x;
}

// predictEstimate (ModelSpecifics.h:1011-1014 LR, 1592-1594 Poisson; the
// conditional and Cox models return xBeta).
__global__ void __launch_bounds__(kPT) predictive_estimates_kernel(PredictParams P, double* out) {
    for (int64_t k = (int64_t)blockIdx.x * kPT + threadIdx.x; k < P.K; k += (int64_t)gridDim.x * kPT) {
        const double xb = row_xbeta(P, k);
        double r = xb;
        if (P.model == M_LOGISTIC) {
            const double e = exp(xb);
            r = e / (e + 1.0);
        } else if (P.model == M_POISSON) {
            r = exp(xb);
        }
        out[k] = r;
    }
}

}  // namespace

cudaError_t launch_predictive_loglik(const PredictParams& P, double* part, int n_blocks, cudaStream_t s) {
    if (n_blocks <= 0) return cudaErrorInvalidValue;
    predictive_ll_kernel<<<n_blocks, kPT, 0, s>>>(P, part);
    return cudaGetLastError();
}

cudaError_t launch_predictive_estimates(const PredictParams& P, double* out, cudaStream_t s) {
    const int64_t want = (P.K + kPT - 1) / kPT;
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 4096));
    predictive_estimates_kernel<<<g, kPT, 0, s>>>(P, out);
    return cudaGetLastError();
}

}  // namespace ccdb
