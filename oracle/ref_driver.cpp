// ref_driver.cpp -- ORACLE / TEST INFRASTRUCTURE ONLY.
//
// A flat extern "C" driver around the reference Cyclops engine (namespace
// bsccs), compiled from the reference's own sources by oracle/Makefile into
// oracle/_ref/libccd_ref.so.  It is the checker the CUDA path is compared
// against and the timed CPU baseline; nothing in the product links it.
//
// Data enters exactly the way the reference's R binding feeds it:
//   ModelData::loadY   (src/cyclops/ModelData.cpp:69-140)
//   ModelData::loadX   (src/cyclops/ModelData.cpp:246-370), intercept first
//   ModelData::setOffsetCovariate (src/cyclops/ModelData.cpp:640-651)
//   AbstractModelSpecifics::factory (src/cyclops/engine/AbstractModelSpecifics.cpp:128-154)
//   CyclicCoordinateDescent::update (src/cyclops/CyclicCoordinateDescent.cpp:586-615)
// so the resulting column order is [offset?, intercept?, covariates...].

#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <map>

#include "ModelData.h"
#include "CyclicCoordinateDescent.h"
#include "CcdInterface.h"
#include "drivers/AutoSearchCrossValidationDriver.h"
#include "drivers/CrossValidationSelector.h"
#include "drivers/GridSearchCrossValidationDriver.h"
#include "priors/JointPrior.h"
#include "priors/CovariatePrior.h"
#include "utils/HParSearch.h"
#ifdef CCDB_B200_ADAPTER
#include "B200CyclicCoordinateDescent.h"
#include "B200ModelSpecifics.h"
#endif

using namespace bsccs;

namespace {

struct QuietLogger : loggers::ProgressLogger {
    void writeLine(const std::ostringstream&) override {}
    void yield() override {}
};
struct ThrowingErrors : loggers::ErrorHandler {
    void throwError(const std::ostringstream& s) override { throw std::runtime_error(s.str()); }
};

// Keeps every line the cross-validation drivers log (their per-step summaries).
// Worker threads of a multi-threaded cross-validation write lines concurrently
// (AbstractCrossValidationDriver.cpp:196-235), so appends are serialised.
struct RecordingLogger : loggers::ProgressLogger {
    std::string text;
    std::mutex lock;
    void writeLine(const std::ostringstream& s) override {
        std::lock_guard<std::mutex> g(lock);
        text += s.str() + "\n";
    }
    void yield() override {}
};

// The grid driver's evaluated points and values (protected members).
struct GridDriver : GridSearchCrossValidationDriver {
    using GridSearchCrossValidationDriver::GridSearchCrossValidationDriver;
    const std::vector<double>& points() const { return gridPoint; }
    const std::vector<double>& values() const { return gridValue; }
};

// A CcdInterface used only for profileModel (CcdInterface.cpp:262-525); the
// model-building hooks of the R and command-line front ends are not needed.
struct ProfileInterface : CcdInterface {
    ProfileInterface(loggers::ProgressLoggerPtr l, loggers::ErrorHandlerPtr e, const ModeFindingArguments& mf) {
        logger = l;
        error = e;
        arguments.modeFinding = mf;
        arguments.noiseLevel = SILENT;
    }

protected:
    void initializeModelImpl(AbstractModelData**, CyclicCoordinateDescent**, AbstractModelSpecifics**) override {}
    void predictModelImpl(CyclicCoordinateDescent*, AbstractModelData*) override {}
    void logModelImpl(CyclicCoordinateDescent*, AbstractModelData*, ProfileInformationMap&, bool) override {}
    void diagnoseModelImpl(CyclicCoordinateDescent*, AbstractModelData*, double, double) override {}
};

// Column format codes: the reference's FormatType (CompressedDataMatrix.h:36-38).
enum { F_DENSE = 0, F_SPARSE = 1, F_INDICATOR = 2, F_INTERCEPT = 3 };

struct RefHandle {
    std::shared_ptr<QuietLogger> log;
    std::shared_ptr<ThrowingErrors> err;
    std::unique_ptr<AbstractModelData> data;
    std::unique_ptr<AbstractModelSpecifics> ms;
    priors::JointPriorPtr prior;
    std::unique_ptr<CyclicCoordinateDescent> ccd;
#ifdef CCDB_B200_ADAPTER
    B200CyclicCoordinateDescent* fused = nullptr;  // ccd, when it is the fused solver
#endif
    int J = 0;
    int64_t K = 0;
    bool weighted = false;
};

void set_err(char* err, int errlen, const char* msg) {
    if (err && errlen > 0) {
        std::strncpy(err, msg, errlen - 1);
        err[errlen - 1] = 0;
    }
}

template <typename Real>
AbstractModelData* build_data(ModelType mt, int64_t K, int J, const double* y, const double* time,
                              const int64_t* stratum, const int64_t* col_start, const int32_t* rows,
                              const int64_t* val_start, const double* vals, const uint8_t* fmt,
                              int offset_col0, loggers::ProgressLoggerPtr lg,
                              loggers::ErrorHandlerPtr er) {
    auto* md = new ModelData<Real>(mt, lg, er);
    std::vector<IdType> rid(K);
    for (int64_t i = 0; i < K; ++i) rid[i] = i;
    std::vector<IdType> sid;
    if (stratum) sid.assign(stratum, stratum + K);
    std::vector<double> yv(y, y + K);
    std::vector<double> tv;
    if (time) tv.assign(time, time + K);
    md->loadY(sid, rid, yv, tv);

    // The reference moves an INTERCEPT to the front on load and the offset to
    // the front on setOffsetCovariate; loading the intercept first and the
    // offset last reproduces the caller's [offset?, intercept?, rest] order.
    const int first = offset_col0 ? 1 : 0;
    std::vector<int> order;
    for (int j = first; j < J; ++j)
        if (fmt[j] == F_INTERCEPT) order.push_back(j);
    for (int j = first; j < J; ++j)
        if (fmt[j] != F_INTERCEPT) order.push_back(j);
    if (offset_col0) order.push_back(0);

    for (int j : order) {
        std::vector<IdType> r;
        std::vector<double> v;
        bool forceSparse = false;
        switch (fmt[j]) {
        case F_INTERCEPT:
            break;
        case F_DENSE:
            v.assign(vals + val_start[j], vals + val_start[j + 1]);
            break;
        case F_INDICATOR:
            r.assign(rows + col_start[j], rows + col_start[j + 1]);
            break;
        case F_SPARSE:
            r.assign(rows + col_start[j], rows + col_start[j + 1]);
            v.assign(vals + val_start[j], vals + val_start[j + 1]);
            forceSparse = true;
            break;
        default:
            throw std::runtime_error("unknown column format");
        }
        const IdType label = (offset_col0 && j == 0) ? IdType(1000000000) : IdType(j + 1);
        if ((fmt[j] == F_INDICATOR || fmt[j] == F_SPARSE) && r.empty()) {
            // An empty column: loadX would read "no rows, no values" as an
            // intercept (ModelData.cpp:257-263) and move it to the front, so the
            // empty column goes into the matrix directly, as the reference's other
            // constructors build columns (CompressedDataMatrix::push_back).
            md->getX().push_back(fmt[j] == F_INDICATOR ? INDICATOR : SPARSE);
            md->getX().getColumn(md->getX().getNumberOfColumns() - 1).add_label(label);
        } else {
            md->loadX(label, r, v, false, false, forceSparse);
        }
    }
    if (offset_col0) md->setOffsetCovariate(IdType(1000000000));
    return md;
}

}  // namespace

extern "C" {

// Build ModelData + ModelSpecifics + MixtureJointPrior + CyclicCoordinateDescent.
// model_type uses the reference's ModelType numbering (Types.h:134-147).
// prior_type per column: 0 none, 1 Laplace, 2 Normal (priors::PriorType, Types.h:100-105).
static void* create_impl(bool on_b200, bool fused, int model_type, int fp32, int64_t K, int J, const double* y,
                         const double* time, const int64_t* stratum, const int64_t* col_start,
                         const int32_t* rows, const int64_t* val_start, const double* vals,
                         const uint8_t* fmt, int offset_col0, const int32_t* prior_type,
                         const double* prior_var, char* err, int errlen) {
    try {
        auto h = new RefHandle();
        h->log = std::make_shared<QuietLogger>();
        h->err = std::make_shared<ThrowingErrors>();
        h->J = J;
        h->K = K;
        const ModelType mt = static_cast<ModelType>(model_type);
        if (fp32) {
            h->data.reset(build_data<float>(mt, K, J, y, time, stratum, col_start, rows, val_start,
                                            vals, fmt, offset_col0, h->log, h->err));
        } else {
            h->data.reset(build_data<double>(mt, K, J, y, time, stratum, col_start, rows, val_start,
                                             vals, fmt, offset_col0, h->log, h->err));
        }
        if (on_b200) {
#ifdef CCDB_B200_ADAPTER
            if (fp32) throw std::runtime_error("the B200 adapter is built for ModelData<double>");
            h->ms.reset(new B200ModelSpecifics(static_cast<const ModelData<double>&>(*h->data), mt));
#else
            throw std::runtime_error("built without the B200 adapter");
#endif
        } else {
            h->ms.reset(AbstractModelSpecifics::factory(mt, *h->data, DeviceType::CPU, "native"));
        }
        if (!h->ms) throw std::runtime_error("factory returned nullptr (unsupported model)");

        std::map<std::pair<int, double>, priors::PriorPtr> unique;
        auto getPrior = [&](int type, double var) -> priors::PriorPtr {
            auto key = std::make_pair(type, type == 0 ? 0.0 : var);
            auto it = unique.find(key);
            if (it != unique.end()) return it->second;
            priors::PriorPtr p;
            if (type == 1) p = std::make_shared<priors::LaplacePrior>(var);
            else if (type == 2) p = std::make_shared<priors::NormalPrior>(var);
            else p = std::make_shared<priors::NoPrior>();
            unique[key] = p;
            return p;
        };
        auto mix = std::make_shared<priors::MixtureJointPrior>(getPrior(prior_type[0], prior_var[0]), J);
        for (int j = 1; j < J; ++j) mix->changePrior(getPrior(prior_type[j], prior_var[j]), j);
        h->prior = mix;
        if (fused) {
#ifdef CCDB_B200_ADAPTER
            auto* c = new B200CyclicCoordinateDescent(
                *h->data, static_cast<B200ModelSpecifics&>(*h->ms), h->prior, h->log, h->err,
                std::vector<int32_t>(prior_type, prior_type + J), std::vector<double>(prior_var, prior_var + J));
            h->fused = c;
            h->ccd.reset(c);
#else
            throw std::runtime_error("built without the B200 adapter");
#endif
        } else {
            h->ccd.reset(new CyclicCoordinateDescent(*h->data, *h->ms, h->prior, h->log, h->err));
        }
        h->ccd->setNoiseLevel(SILENT);
        return h;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return nullptr;
    }
}

void* ref_create(int model_type, int fp32, int64_t K, int J, const double* y, const double* time,
                 const int64_t* stratum, const int64_t* col_start, const int32_t* rows,
                 const int64_t* val_start, const double* vals, const uint8_t* fmt, int offset_col0,
                 const int32_t* prior_type, const double* prior_var, char* err, int errlen) {
    return create_impl(false, false, model_type, fp32, K, J, y, time, stratum, col_start, rows, val_start,
                       vals, fmt, offset_col0, prior_type, prior_var, err, errlen);
}

// The reference's own CyclicCoordinateDescent driving B200ModelSpecifics
// (ccd_b200/integration/B200ModelSpecifics.h) in place of ModelSpecifics.
void* ref_create_b200(int model_type, int fp32, int64_t K, int J, const double* y, const double* time,
                      const int64_t* stratum, const int64_t* col_start, const int32_t* rows,
                      const int64_t* val_start, const double* vals, const uint8_t* fmt, int offset_col0,
                      const int32_t* prior_type, const double* prior_var, char* err, int errlen) {
    return create_impl(true, false, model_type, fp32, K, J, y, time, stratum, col_start, rows, val_start,
                       vals, fmt, offset_col0, prior_type, prior_var, err, errlen);
}

// The same, with B200CyclicCoordinateDescent (ccd_b200/integration) as the
// solver: every findMode of update() is one ccdb_find_mode on the device.
void* ref_create_b200_fused(int model_type, int fp32, int64_t K, int J, const double* y, const double* time,
                            const int64_t* stratum, const int64_t* col_start, const int32_t* rows,
                            const int64_t* val_start, const double* vals, const uint8_t* fmt, int offset_col0,
                            const int32_t* prior_type, const double* prior_var, char* err, int errlen) {
    return create_impl(true, true, model_type, fp32, K, J, y, time, stratum, col_start, rows, val_start,
                       vals, fmt, offset_col0, prior_type, prior_var, err, errlen);
}

// ccdb_find_mode calls made by a fused solver (-1 for any other handle).
int64_t ref_device_calls(void* hp) {
#ifdef CCDB_B200_ADAPTER
    auto h = static_cast<RefHandle*>(hp);
    return h->fused ? h->fused->deviceCalls() : -1;
#else
    (void)hp;
    return -1;
#endif
}

void ref_destroy(void* hp) {
    auto h = static_cast<RefHandle*>(hp);
    if (!h) return;
    h->ccd.reset();
    h->ms.reset();
    h->data.reset();
    delete h;
}

// Row weights (CV fold weights); NULL clears them (CyclicCoordinateDescent.cpp:496-519).
int ref_set_weights(void* hp, const double* w) {
    auto h = static_cast<RefHandle*>(hp);
    if (w) {
        std::vector<double> buf(w, w + h->K);
        h->ccd->setWeights(buf.data());
        h->weighted = true;
    } else {
        h->ccd->setWeights(nullptr);
        h->weighted = false;
    }
    return 0;
}

int ref_set_beta(void* hp, const double* beta) {
    auto h = static_cast<RefHandle*>(hp);
    std::vector<double> b(beta, beta + h->J);
    h->ccd->setBeta(b);
    return 0;
}

// Full mode finding through CyclicCoordinateDescent::update.  algorithm:
// AlgorithmType (0 CCD, 1 MM); use_kkt: ModeFindingArguments::useKktSwindle;
// fixed: J flags for setFixedBeta, or NULL (the offset stays fixed either way).
int ref_fit(void* hp, int conv_type, double tol, int max_iter, double initial_bound,
            int max_bound_count, int algorithm, int use_kkt, const uint8_t* fixed, double* beta_out,
            double* ll_out, int* iters_out, int* flag_out, char* err, int errlen) {
    auto h = static_cast<RefHandle*>(hp);
    try {
        ModeFindingArguments a;
        a.tolerance = tol;
        a.maxIterations = max_iter;
        a.convergenceType = conv_type;
        a.initialBound = initial_bound;
        a.maxBoundCount = max_bound_count;
        a.algorithmType = algorithm == 1 ? AlgorithmType::MM : AlgorithmType::CCD;
        a.useKktSwindle = use_kkt != 0;
        if (fixed) {
            const bool offset = h->data->getHasOffsetCovariate();
            for (int j = 0; j < h->J; ++j) h->ccd->setFixedBeta(j, fixed[j] != 0 || (offset && j == 0));
        }
#ifdef CCDB_B200_ADAPTER
        if (h->fused) h->fused->update(a);  // update() is not virtual in the reference
        else h->ccd->update(a);
#else
        h->ccd->update(a);
#endif
        for (int j = 0; j < h->J; ++j) beta_out[j] = h->ccd->getBeta(j);
        *ll_out = h->ccd->getLogLikelihood();
        *iters_out = h->ccd->getIterationCount();
        *flag_out = static_cast<int>(h->ccd->getUpdateReturnFlag());
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return -1;
    } catch (std::logic_error* e) {  // the reference throws some errors by pointer
        set_err(err, errlen, e->what());
        delete e;
        return -1;
    }
}

// Per-coordinate gradient/Hessian exactly as ccdUpdateBeta obtains them
// (CyclicCoordinateDescent.cpp:1394-1405), before the h<0 clamp.
int ref_grad_hess(void* hp, int j, double* g, double* hs) {
    auto h = static_cast<RefHandle*>(hp);
    h->ccd->getLogLikelihood();  // brings the lazy state up to date (checkAllLazyFlags)
    h->ms->computeNumeratorForGradient(j, h->weighted);
    h->ms->computeGradientAndHessian(j, g, hs, h->weighted);
    return 0;
}

// beta[j] += delta followed by ModelSpecifics::updateXBeta (setBeta(int,double),
// CyclicCoordinateDescent.cpp:719-733).
int ref_update_beta(void* hp, int j, double delta) {
    auto h = static_cast<RefHandle*>(hp);
    h->ccd->getLogLikelihood();
    h->ccd->setBeta(j, h->ccd->getBeta(j) + delta);
    return 0;
}

int ref_loglik(void* hp, double* ll) {
    auto h = static_cast<RefHandle*>(hp);
    *ll = h->ccd->getLogLikelihood();
    return 0;
}

int ref_log_prior(void* hp, double* lp) {
    auto h = static_cast<RefHandle*>(hp);
    *lp = h->ccd->getLogPrior();
    return 0;
}

int ref_get_beta(void* hp, double* out) {
    auto h = static_cast<RefHandle*>(hp);
    for (int j = 0; j < h->J; ++j) out[j] = h->ccd->getBeta(j);
    return 0;
}

int ref_get_xbeta(void* hp, double* out) {
    auto h = static_cast<RefHandle*>(hp);
    h->ccd->getLogLikelihood();
    auto xb = h->ms->getXBeta();
    std::memcpy(out, xb.data(), sizeof(double) * xb.size());
    return static_cast<int>(xb.size());
}

// Predictive log-likelihood on held-out weights (CyclicCoordinateDescent.cpp:319-355).
int ref_predictive_loglik(void* hp, const double* w, double* out) {
    auto h = static_cast<RefHandle*>(hp);
    std::vector<double> buf(w, w + h->K);
    *out = h->ccd->getNewPredictiveLogLikelihood(buf.data());
    return 0;
}

int ref_num_patients(void* hp) {
    auto h = static_cast<RefHandle*>(hp);
    return static_cast<int>(h->data->getNumberOfPatients());
}

// CyclicCoordinateDescent::computeFisherInformation(indices) (.cpp:1288-1299),
// the call behind the R binding's getFisherInformation, after the lazy state is
// brought current (that call itself does not check it).  out: n x n, row-major.
// Returns -2 when the engine refuses (weighted fits: ModelSpecifics.hpp:1207-1208
// throws a std::logic_error*, the B200 adapter a std::logic_error), -1 on any
// other error.
int ref_fisher_information(void* hp, const int32_t* idx, int n, double* out, char* err, int errlen) {
    auto h = static_cast<RefHandle*>(hp);
    try {
        h->ccd->getLogLikelihood();
        std::vector<IdType> indices(idx, idx + n);
        const auto m = h->ccd->computeFisherInformation(indices);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) out[(size_t)i * n + j] = m(i, j);
        return 0;
    } catch (std::logic_error* e) {
        set_err(err, errlen, e->what());
        delete e;
        return -2;
    } catch (const std::logic_error& e) {
        set_err(err, errlen, e.what());
        return -2;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return -1;
    }
}

// CyclicCoordinateDescent::getAsymptoticVariance(i, j) (.cpp:1249-1269): the
// inverse of the Fisher information over the free, non-zero-Laplace columns
// (computeAsymptoticPrecisionMatrix, .cpp:1301-1347); NaN for other columns.
int ref_asymptotic_variance(void* hp, int i, int j, double* out, char* err, int errlen) {
    auto h = static_cast<RefHandle*>(hp);
    try {
        *out = h->ccd->getAsymptoticVariance(i, j);
        return 0;
    } catch (std::logic_error* e) {
        set_err(err, errlen, e->what());
        delete e;
        return -2;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return -1;
    }
}

// Cross-validation as CcdInterface::runCrossValidation (CcdInterface.cpp:731-790)
// runs it: a CrossValidationSelector over the data's ids (by row for Cox, by
// id otherwise, getDefaultSelectorTypeOrOverride :675-690), the auto-search or
// grid driver, then resetForOptimal and the fit at the selected variance.
// Cold starts (resetCoefficients); with threads = 1 the run is deterministic
// (more threads run the (fold, variance) tasks on clones of the engine).
// fold_to_compute: the folds of the split actually fitted (0: all).
// row_fold_out[K]: the held-out fold of each row under the selector's first
// permutation (the one every step reuses after reseed()).  Grid: points_out /
// values_out receive the grid (n_points).  log_out receives the drivers' log.
// hyper_out: every variance parameter of the joint prior after the refit
// (n_hyper of them; the auto search tunes each in turn when there are several).
int ref_cross_validate(void* hp, int auto_search, int fold, int grid_steps, double lower, double upper,
                       double starting_variance, long seed, int conv_type, double tol, int max_iter,
                       int32_t* row_fold_out, double* points_out, double* values_out, int max_points,
                       int* n_points, double* variance_out, double* beta_out, double* ll_out, char* log_out,
                       int log_len, double* hyper_out, int max_hyper, int* n_hyper, int threads,
                       int fold_to_compute, char* err, int errlen) {
    auto h = static_cast<RefHandle*>(hp);
    try {
        CCDArguments args = CCDArguments();
        args.threads = threads > 0 ? threads : 1;
        args.resetCoefficients = true;
        args.seed = seed;
        args.useHierarchy = false;
        args.noiseLevel = SILENT;
        args.useNormalPrior = false;
        args.crossValidation.doCrossValidation = true;
        args.crossValidation.useAutoSearchCV = auto_search != 0;
        args.crossValidation.fold = fold;
        args.crossValidation.foldToCompute = fold_to_compute > 0 ? fold_to_compute : fold;
        args.crossValidation.gridSteps = grid_steps;
        args.crossValidation.lowerLimit = lower;
        args.crossValidation.upperLimit = upper;
        args.crossValidation.startingVariance = starting_variance;
        args.modeFinding.tolerance = tol;
        args.modeFinding.convergenceType = conv_type;
        args.modeFinding.maxIterations = max_iter;
        const SelectorType type = (h->data->getModelType() == ModelType::COX) ? SelectorType::BY_ROW
                                                                               : SelectorType::BY_PID;
        auto log = std::make_shared<RecordingLogger>();
        CrossValidationSelector selector(fold, h->data->getPidVectorSTL(), type, seed, log, h->err, nullptr,
                                         nullptr);
        selector.reseed();
        selector.permute();
        std::vector<double> w;
        for (int f = 0; f < fold; ++f) {
            selector.getWeights(f, w);
            for (int64_t k = 0; k < h->K; ++k)
                if (w[k] == 0.0) row_fold_out[k] = f;
        }
        std::unique_ptr<AbstractCrossValidationDriver> driver;
        GridDriver* grid = nullptr;
        if (auto_search) {
            driver.reset(new AutoSearchCrossValidationDriver(*h->data, args, log, h->err));
        } else {
            grid = new GridDriver(args, log, h->err);
            driver.reset(grid);
        }
        driver->drive(*h->ccd, selector, args);
        driver->resetForOptimal(*h->ccd, selector, args);
        h->ccd->update(args.modeFinding);
        const std::vector<double> hyper = h->ccd->getHyperprior();
        *variance_out = hyper[0];
        *n_hyper = (int)hyper.size();
        for (int i = 0; i < std::min<int>(max_hyper, (int)hyper.size()); ++i) hyper_out[i] = hyper[i];
        for (int j = 0; j < h->J; ++j) beta_out[j] = h->ccd->getBeta(j);
        *ll_out = h->ccd->getLogLikelihood();
        *n_points = 0;
        if (grid) {
            const int n = std::min<int>(max_points, (int)grid->points().size());
            for (int i = 0; i < n; ++i) {
                points_out[i] = grid->points()[i];
                values_out[i] = grid->values()[i];
            }
            *n_points = n;
        }
        set_err(log_out, log_len, log->text.c_str());
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return -1;
    }
}

// Profile-likelihood bounds of columns cols[0..n) around the current mode,
// one thread (CcdInterface::profileModel, CcdInterface.cpp:262-525): per
// column the upper then the lower bound, each a sign-change bracket and a
// zeroin root of LL(beta_j fixed) + threshold - LL(mode).  NaN where no sign
// change was found.  The engine must hold a fitted mode.
int ref_profile(void* hp, const int32_t* cols, int n, double threshold, int include_penalty,
                int override_no_regularization, int conv_type, double tol, int max_iter, double* lower_out,
                double* upper_out, int32_t* evals_out, char* err, int errlen) {
    auto h = static_cast<RefHandle*>(hp);
    try {
        ModeFindingArguments mf;
        mf.tolerance = tol;
        mf.maxIterations = max_iter;
        mf.convergenceType = conv_type;
        ProfileInterface iface(h->log, h->err, mf);
        ProfileVector labels;
        const bool offset = h->data->getHasOffsetCovariate();
        for (int i = 0; i < n; ++i)  // the labels build_data gave the columns
            labels.push_back((offset && cols[i] == 0) ? IdType(1000000000) : IdType(cols[i] + 1));
        ProfileInformationMap out;
        iface.profileModel(h->ccd.get(), h->data.get(), labels, out, 1, threshold,
                           override_no_regularization != 0, include_penalty != 0);
        for (int i = 0; i < n; ++i) {
            const ProfileInformation& p = out.at(labels[i]);
            lower_out[i] = p.lower95Bound;
            upper_out[i] = p.upper95Bound;
            evals_out[i] = p.evaluations;
        }
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return -1;
    }
}

// CyclicCoordinateDescent::getPredictiveEstimates (.cpp:357-359); w may be NULL.
int ref_predictive_estimates(void* hp, const double* w, double* y) {
    auto h = static_cast<RefHandle*>(hp);
    h->ccd->getLogLikelihood();
    std::vector<double> wb;
    if (w) wb.assign(w, w + h->K);
    h->ccd->getPredictiveEstimates(y, w ? wb.data() : nullptr);
    return 0;
}

// The auto search's quadratic fit (utils/HParSearch.cpp:22-64) on a history of
// n points (x, mean, stdev); out: c0, c1, c2.
int ref_quadr_log_fit(int n, const double* x, const double* m, const double* sd, double* out) {
    std::map<double, UniModalSearch::MS> h;
    for (int i = 0; i < n; ++i) h[x[i]] = UniModalSearch::MS(m[i], sd[i]);
    const QuadrCoefs c = QuadrLogFit(h);
    out[0] = c.c0;
    out[1] = c.c1;
    out[2] = c.c2;
    return 0;
}

}  // extern "C"
