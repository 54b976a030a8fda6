// B200ModelSpecifics.h -- the reference-side binding: an
// bsccs::AbstractModelSpecifics (src/cyclops/engine/AbstractModelSpecifics.h:36-229)
// whose every operator call goes through the C ABI of libccdb.so
// (include/ccdb.h).  Dropped into the Cyclops source tree, it lets the
// unchanged CyclicCoordinateDescent drive the B200 engine: the GPU slot of
// AbstractModelSpecifics::deviceFactory (AbstractModelSpecifics.cpp:21-41)
// returns it instead of a ModelSpecifics<Model, Real>.
//
// Compiles against the reference headers only; it is built here by
// oracle/Makefile (target ref_b200) to run the reference's own solver on the
// GPU engine in the tests.
#pragma once

#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine/AbstractModelSpecifics.h"
#include "ModelData.h"
#include "ccdb.h"

namespace bsccs {

class B200ModelSpecifics : public AbstractModelSpecifics {
public:
    // modelType: the reference's ModelType; device: CUDA ordinal.
    B200ModelSpecifics(const ModelData<double>& data, ModelType modelType, int device = 0)
        : AbstractModelSpecifics(data), data_(data), modelType_(modelType), device_(device) {
        check(ccdb_context_create(device_, 0, &ctx_), "context");
        const auto& X = data.getX();
        const int64_t K = (int64_t)data.getNumberOfRows();
        const int32_t J = (int32_t)data.getNumberOfCovariates();
        std::vector<int64_t> cs(J + 1, 0), vs(J + 1, 0);
        std::vector<int32_t> rows;
        std::vector<double> vals;
        std::vector<uint8_t> fmt(J);
        for (int j = 0; j < J; ++j) {
            const FormatType f = X.getFormatType(j);
            fmt[j] = static_cast<uint8_t>(f);
            if (f == SPARSE || f == INDICATOR) {
                const auto& r = X.getCompressedColumnVectorSTL(j);
                rows.insert(rows.end(), r.begin(), r.end());
            }
            if (f == SPARSE || f == DENSE) {
                const auto& v = X.getDataVectorSTL(j);
                vals.insert(vals.end(), v.begin(), v.end());
            }
            cs[j + 1] = (int64_t)rows.size();
            vs[j + 1] = (int64_t)vals.size();
        }
        check(ccdb_matrix_create(ctx_, K, J, cs.data(), rows.data(), vs.data(), vals.data(),
                                 fmt.data(), &matrix_), "matrix");
        const auto& y = data.getYVectorRef();
        const auto& time = data.getTimeVectorRef();
        const auto& pid = data.getPidVectorRef();
        y_.assign(y.begin(), y.end());
        if (!time.empty()) time_.assign(time.begin(), time.end());
        strata_.assign(pid.begin(), pid.end());
        ccdb_fit_desc d{};
        d.model_type = static_cast<int32_t>(modelType_);
        d.precision = CCDB_PRECISION_FP64;
        d.y = y_.data();
        d.time = time_.empty() ? nullptr : time_.data();
        d.stratum = strata_.empty() ? nullptr : strata_.data();
        d.offset_col0 = data.getHasOffsetCovariate() ? 1 : 0;
        check(ccdb_fit_create(ctx_, matrix_, &d, &fit_), "fit");
        beta_.assign(J, 0.0);
        if (d.offset_col0) beta_[0] = 1.0;
        J_ = J;
        K_ = K;
    }

    ~B200ModelSpecifics() override {
        if (fit_) ccdb_fit_destroy(fit_);
        if (matrix_) ccdb_matrix_destroy(matrix_);
        if (ctx_) ccdb_context_destroy(ctx_);
    }

    // data are uploaded at construction; the reference's sizes are implied
    void initialize(int, int, int, const void*, double*, double*, double*, double*,
                    std::vector<std::vector<int>*>*, const int*, double*, double*, double*, double*,
                    const double*) override {}

    void setWeights(double* w, double*, bool useCrossValidation) override {
        check(ccdb_set_weights(fit_, useCrossValidation ? w : nullptr), "setWeights");
    }

    void computeGradientAndHessian(int index, double* g, double* h, bool) override {
        sync_beta();
        check(ccdb_compute_gradient_hessian(fit_, index, g, h), "computeGradientAndHessian");
    }

    // the engine fuses the numerator pass into computeGradientAndHessian
    void computeNumeratorForGradient(int, bool) override {}

    void updateXBeta(double delta, int index, bool) override {
        sync_beta();
        beta_[index] += delta;
        check(ccdb_update_xbeta(fit_, index, delta), "updateXBeta");
    }

    // CyclicCoordinateDescent::computeXBeta is zeroXBeta + axpyXBeta per column
    // (CyclicCoordinateDescent.cpp:1452-1470): mirrored on beta, applied lazily.
    void zeroXBeta() override {
        std::fill(beta_.begin(), beta_.end(), 0.0);
        dirty_ = true;
    }
    void axpyXBeta(const double b, const int j) override {
        beta_[j] += b;
        dirty_ = true;
    }
    // ModelSpecifics::computeXBeta(double*, bool) (ModelSpecifics.hpp:313-361),
    // called by the MM cycle: the product over the one-format transpose.
    void computeXBeta(double* beta, bool) override {
        beta_.assign(beta, beta + J_);
        check(ccdb_compute_xbeta(fit_, beta_.data()), "computeXBeta");
        dirty_ = false;
    }

    void computeRemainingStatistics(bool) override {
        sync_beta();
        check(ccdb_compute_remaining_statistics(fit_), "computeRemainingStatistics");
    }

    void computeFixedTermsInLogLikelihood(bool) override {}      // folded into setWeights
    void computeFixedTermsInGradientAndHessian(bool) override {} // folded into setWeights

    double getLogLikelihood(bool) override {
        sync_beta();
        double ll = 0.0;
        check(ccdb_get_log_likelihood(fit_, &ll), "getLogLikelihood");
        return ll;
    }

    double getGradientObjective(bool) override {
        sync_beta();
        double v = 0.0;
        check(ccdb_get_gradient_objective(fit_, &v), "getGradientObjective");
        return v;
    }

    const std::vector<double> getXBeta() override {
        sync_beta();
        std::vector<double> out(K_);
        check(ccdb_get_xbeta(fit_, out.data()), "getXBeta");
        return out;
    }
    const std::vector<double> getXBetaSave() override { return xbetaSave_; }
    void saveXBeta() override { xbetaSave_ = getXBeta(); }

    // outside the coordinate-descent hot path
    // ModelSpecifics::computeMMGradientAndHessian (ModelSpecifics.hpp:776-889).
    void computeMMGradientAndHessian(std::vector<GradientHessian>& gh, const std::vector<bool>& fixBeta,
                                     bool) override {
        sync_beta();
        std::vector<uint8_t> fixed(fixBeta.begin(), fixBeta.end());
        std::vector<double> g(gh.size()), h(gh.size());
        check(ccdb_compute_mm_gradient_hessian(fit_, fixed.data(), g.data(), h.data()),
              "computeMMGradientAndHessian");
        for (size_t j = 0; j < gh.size(); ++j) gh[j] = GradientHessian(g[j], h[j]);
    }
    // ModelSpecifics::computeFisherInformation (ModelSpecifics.hpp:1203-1225): the
    // reference refuses weighted fits with a logic_error; so does this engine.
    void computeFisherInformation(int indexOne, int indexTwo, double* oinfo, bool useWeights) override {
        if (useWeights) throw std::logic_error("Weights are not yet implemented in Fisher Information calculations");
        sync_beta();
        const int32_t idx[2] = {indexOne, indexTwo};
        double out[4];
        check(ccdb_fisher_information(fit_, idx, 2, out), "computeFisherInformation");
        *oinfo = out[1];
    }
    double getPredictiveLogLikelihood(double* weights) override {
        sync_beta();
        double ll = 0.0;
        check(ccdb_get_predictive_log_likelihood(fit_, weights, &ll), "getPredictiveLogLikelihood");
        return ll;
    }
    void getPredictiveEstimates(double* y, double* weights) override {
        sync_beta();
        check(ccdb_get_predictive_estimates(fit_, weights, y), "getPredictiveEstimates");
    }
    void printTiming() override {}

    AbstractModelSpecifics* clone() const override {
        return new B200ModelSpecifics(data_, modelType_, device_);
    }

    // For B200CyclicCoordinateDescent, which runs a whole findMode in one
    // ccdb_find_mode call on this fit: the handle, and the mode the device now
    // holds (its xBeta and remaining statistics already match these
    // coefficients, so no ccdb_set_beta follows).
    ccdb_fit* handle() {
        sync_beta();
        return fit_;
    }
    void adopt_device_beta(const std::vector<double>& beta) {
        beta_ = beta;
        dirty_ = false;
    }

protected:
    void deviceInitialization() override {}
    bool allocateXjY() override { return true; }
    bool allocateXjX() override { return false; }
    bool initializeAccumulationVectors() override { return modelType_ == ModelType::COX; }
    bool hasResetableAccumulators() override { return false; }

private:
    void sync_beta() {
        if (!dirty_) return;
        check(ccdb_set_beta(fit_, beta_.data()), "computeXBeta");
        dirty_ = false;
    }
    static void check(int rc, const char* what) {
        if (rc != CCDB_OK) {
            std::ostringstream s;
            s << "B200 engine: " << what << " failed (" << rc << "): " << ccdb_last_error();
            throw std::runtime_error(s.str());
        }
    }
    const ModelData<double>& data_;
    ModelType modelType_;
    int device_;
    ccdb_context* ctx_ = nullptr;
    ccdb_matrix* matrix_ = nullptr;
    ccdb_fit* fit_ = nullptr;
    std::vector<double> y_, time_;
    std::vector<int64_t> strata_;
    std::vector<double> beta_, xbetaSave_;
    int32_t J_ = 0;
    int64_t K_ = 0;
    bool dirty_ = true;
};

}  // namespace bsccs
