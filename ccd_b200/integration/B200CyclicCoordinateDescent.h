// B200CyclicCoordinateDescent.h -- the reference-side fused path: a
// bsccs::CyclicCoordinateDescent whose update() runs every findMode of
// CyclicCoordinateDescent::update (src/cyclops/CyclicCoordinateDescent.cpp:586-615)
// as one ccdb_find_mode call on the device, instead of one C-ABI round trip
// per coordinate through B200ModelSpecifics.
//
// The reference's findMode is not virtual, so a Cyclops maintainer makes
// CyclicCoordinateDescent::update virtual (one keyword in
// CyclicCoordinateDescent.h:106) and constructs this class where
// CcdInterface::initializeModel builds the solver; without that keyword a
// caller holding this type calls this update() directly, which is what the
// tests here do.  The per-coordinate calls of the base class (ccdUpdateBeta,
// getLogLikelihood, the predictive calls, Fisher information) keep working
// through the adapter on the same device state.
//
// What update() does, in the reference's order:
//   * findMode's lazy preamble (.cpp:917-938): the weights, fixed terms, xBeta
//     and remaining statistics are pushed through the adapter exactly as the
//     base class would push them;
//   * one ccdb_find_mode with the solver's arguments (convergence type,
//     tolerance, iteration cap, initial bound, bound-retry count, CCD or MM,
//     the KKT swindle when the joint prior supports it), the fixed set
//     (fixBeta) and the per-column priors; the device continues from the
//     current state and runs the ILLCONDITIONED retry of update() itself;
//   * the mode, return flag and cycle count land in hBeta, lastReturnFlag and
//     lastIterationCount, as the base class leaves them.
// Convergence types beyond GRADIENT, LANGE and MITTAL (ZHANG_OLES, ONE_STEP)
// are not run on the device: update() hands them to the base class.
//
// The per-column priors are passed in (type 0 none, 1 Laplace, 2 normal, and
// the variance), because the reference's JointPrior keeps its per-column
// list protected; they must describe the same priors as `prior`.
#pragma once

#include <cstdint>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "B200ModelSpecifics.h"
#include "CyclicCoordinateDescent.h"

namespace bsccs {

class B200CyclicCoordinateDescent : public CyclicCoordinateDescent {
public:
    B200CyclicCoordinateDescent(const AbstractModelData& data, B200ModelSpecifics& specifics,
                                priors::JointPriorPtr prior, loggers::ProgressLoggerPtr logger,
                                loggers::ErrorHandlerPtr error, std::vector<int32_t> prior_type,
                                std::vector<double> prior_var)
        : CyclicCoordinateDescent(data, specifics, prior, logger, error), b200_(specifics),
          prior_type_(std::move(prior_type)), prior_var_(std::move(prior_var)) {}

    // the number of ccdb_find_mode calls made so far (one per update())
    int64_t deviceCalls() const { return device_calls_; }

    void update(const ModeFindingArguments& a) {
        if (a.convergenceType < GRADIENT || a.convergenceType > MITTAL) {
            CyclicCoordinateDescent::update(a);
            return;
        }
        initialBound = a.initialBound;
        // findMode's preamble (CyclicCoordinateDescent.cpp:917-938)
        if (!validWeights || hXI.getTouchedY()) {
            computeNEvents();
            computeFixedTermsInLogLikelihood();
            computeFixedTermsInGradientAndHessian();
            validWeights = true;
            hXI.clean();
        }
        if (!xBetaKnown) {
            computeXBeta();
            xBetaKnown = true;
            sufficientStatisticsKnown = false;
        }
        if (!sufficientStatisticsKnown) {
            computeRemainingStatistics(true, 0);
            sufficientStatisticsKnown = true;
        }
        std::vector<uint8_t> fixed(J);
        for (int j = 0; j < J; ++j) fixed[j] = fixBeta[j] ? 1 : 0;
        ccdb_mode_args m{};
        m.prior_type = prior_type_.data();
        m.prior_var = prior_var_.data();
        m.convergence_type = a.convergenceType;
        m.tolerance = a.tolerance;
        m.max_iterations = a.maxIterations;
        m.initial_bound = a.initialBound;
        m.max_bound_count = a.maxBoundCount;
        m.per_coordinate = 0;
        m.strategy = CCDB_SWEEP_AUTO;
        m.algorithm = (a.algorithmType == AlgorithmType::MM) ? CCDB_ALGORITHM_MM : CCDB_ALGORITHM_CCD;
        m.use_kkt_swindle = (a.useKktSwindle && jointPrior->getSupportsKktSwindle()) ? 1 : 0;
        m.fixed = fixed.data();
        ccdb_fit* f = b200_.handle();
        ccdb_fit_result r{};
        check(ccdb_find_mode(f, &m, nullptr, &r), "findMode");
        ++device_calls_;
        std::vector<double> beta(J);
        check(ccdb_get_beta(f, beta.data()), "getBeta");
        for (int j = 0; j < J; ++j) hBeta[j] = beta[j];
        b200_.adopt_device_beta(beta);
        lastReturnFlag = static_cast<UpdateReturnFlags>(r.return_flag);
        lastIterationCount = r.iterations;
        xBetaKnown = true;
        sufficientStatisticsKnown = true;
        fisherInformationKnown = false;
        varianceKnown = false;
    }

private:
    static void check(int rc, const char* what) {
        if (rc != CCDB_OK) {
            std::ostringstream s;
            s << "B200 engine: " << what << " failed (" << rc << "): " << ccdb_last_error();
            throw std::runtime_error(s.str());
        }
    }
    B200ModelSpecifics& b200_;
    std::vector<int32_t> prior_type_;
    std::vector<double> prior_var_;
    int64_t device_calls_ = 0;
};

}  // namespace bsccs
