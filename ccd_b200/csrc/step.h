// step.h -- the coordinate step shared by host and device code: the Newton
// step with the prior's closed form and the trust-region bound.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define CCDB_HD __host__ __device__ __forceinline__
#else
#define CCDB_HD inline
#endif

namespace ccdb {

CCDB_HD int sgn_d(double x) { return x == 0 ? 0 : (x < 0 ? -1 : 1); }

// ccdUpdateBeta's clamp + JointPrior::getDelta (CyclicCoordinateDescent.cpp:1394-1413;
// priors/CovariatePrior.h:186-188 NoPrior, :240-273 Laplace, :410-415 Normal).
// `lambda` is sqrt(2 / var) of a Laplace prior (CovariatePrior.h:282-292),
// passed in by callers that take many steps under one variance.
CCDB_HD double newton_prior_delta_l(double g, double h, double beta, int ptype, double var,
                                    double lambda) {
    if (h < 0.0) {
        g = 0.0;
        h = 0.0;
    }
    if (ptype == 1) {
        const double neg = -(g - lambda) / h;
        const double pos = -(g + lambda) / h;
        const int s = sgn_d(beta);
        double delta;
        if (s == 0) {
            if (neg < 0) delta = neg;
            else if (pos > 0) delta = pos;
            else delta = 0.0;
        } else {
            delta = (s < 0) ? neg : pos;
            if (sgn_d(beta + delta) != s) delta = -beta;
        }
        return delta;
    } else if (ptype == 2) {
        return -(g + (beta / var)) / (h + (1.0 / var));
    }
    return -(g / h);
}

CCDB_HD double newton_prior_delta(double g, double h, double beta, int ptype, double var) {
    return newton_prior_delta_l(g, h, beta, ptype, var, ptype == 1 ? sqrt(2.0 / var) : 0.0);
}

// applyBounds (CyclicCoordinateDescent.cpp:1503-1520), std::max semantics.
CCDB_HD double apply_bounds(double delta, double& hd) {
    if (delta < -hd) delta = -hd;
    else if (delta > hd) delta = hd;
    double inter = fabs(delta) * 2;
    const double half = hd / 2;
    inter = (inter < half) ? half : inter;
    inter = (inter < 1E-3) ? 1E-3 : inter;
    hd = inter;
    return delta;
}

// log-density of one coefficient (priors/CovariatePrior.h:220-224, :404-408).
CCDB_HD double log_prior_one(double x, int ptype, double var) {
    if (ptype == 1) {
        const double lambda = sqrt(2.0 / var);
        return log(0.5 * lambda) - lambda * fabs(x);
    } else if (ptype == 2) {
        return -0.5 * log(2.0 * 3.14159265358979323846 * var) - 0.5 * x * x / var;
    }
    return 0.0;
}

// host alias used by the host-side objective
inline double log_prior_host(double x, int ptype, double var) { return log_prior_one(x, ptype, var); }

}  // namespace ccdb
