/* ccdb.h -- C ABI of the B200 coordinate-descent engine (libccdb.so).
 *
 * The engine replaces the CPU implementation behind the reference Cyclops
 * operator API: bsccs::AbstractModelSpecifics (engine/AbstractModelSpecifics.h:36-229)
 * and the mode-finding loop of bsccs::CyclicCoordinateDescent
 * (CyclicCoordinateDescent.cpp:586-615, 909-1216).  Every call takes plain
 * pointers and sizes; no C++ or framework types cross this boundary, no
 * exception escapes it.  All functions return CCDB_OK (0) or a negative status
 * code; ccdb_last_error() gives the message of the last failure on the
 * calling thread.
 *
 * Conventions shared with the reference:
 *   - model_type uses the reference's ModelType numbering (Types.h:134-147):
 *     POISSON=2, LOGISTIC=3, CONDITIONAL_LOGISTIC=4, CONDITIONAL_POISSON=6, COX=8.
 *   - column formats use FormatType (CompressedDataMatrix.h:36-38):
 *     DENSE=0, SPARSE=1, INDICATOR=2, INTERCEPT=3.
 *   - prior types use priors::PriorType (Types.h:100-105): NONE=0, LAPLACE=1, NORMAL=2.
 *   - convergence types use ConvergenceType (Types.h:108-114): GRADIENT=0, LANGE=1, MITTAL=2.
 *   - return flags of a fit use UpdateReturnFlags (Types.h:124-130).
 *   - column order is the reference's after ModelData::loadX/setOffsetCovariate
 *     (ModelData.cpp:246-370, 640-651): [offset?, intercept?, covariates...];
 *     with an offset, column 0's coefficient is fixed at 1.
 *   - survival rows are sorted by (stratum, -time, y) (R/DataManagement.R:166).
 */
#ifndef CCDB_H
#define CCDB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCDB_OK 0
#define CCDB_ERR_INVALID (-1)     /* bad argument or inconsistent data */
#define CCDB_ERR_CUDA (-2)        /* CUDA runtime failure */
#define CCDB_ERR_UNSUPPORTED (-3) /* model/format/option not implemented */
#define CCDB_ERR_BUDGET (-4)      /* request exceeds the context's HBM budget */
#define CCDB_ERR_TIMEOUT (-5)     /* a bounded device-side wait ran out */

#define CCDB_PRECISION_FP64 0  /* all arithmetic in double, as the reference's RealType=double */
#define CCDB_PRECISION_MIXED 1 /* FP64 xBeta and step; exp, ratios and per-entry
                                  gradient/Hessian terms in FP32 with compensated sums; FP64
                                  cross-thread reductions, Cox risk-set sums and
                                  log-likelihoods.  Logistic/Poisson: batched fits only
                                  (ccdb_batch_find_mode); Cox: every call */

typedef struct ccdb_context ccdb_context;
typedef struct ccdb_matrix ccdb_matrix;
typedef struct ccdb_fit ccdb_fit;

/* Thread-local text of the last failure. */
const char* ccdb_last_error(void);

/* One context per GPU.  hbm_budget_bytes = 0 means "no limit". */
int ccdb_context_create(int device, size_t hbm_budget_bytes, ccdb_context** out);
int ccdb_context_destroy(ccdb_context* ctx);
/* Bytes of device memory currently held by matrices and fits of ctx. */
int ccdb_context_memory(const ccdb_context* ctx, size_t* bytes_in_use);

/* Streaming multiprocessors of the context's GPU.  No reference counterpart. */
int ccdb_context_sm_count(const ccdb_context* ctx, int32_t* n_sm);

/* Host waits of this context's calls sleep until the device signals instead
 * of spinning (cudaEventBlockingSync).  Off by default: a spinning wait
 * returns sooner, but a process that runs many contexts' calls at once (one
 * per serving slot) starves its own host threads when every waiting thread
 * spins.  Call it between calls of the context's fits (it remakes the
 * context's timing events).  No reference counterpart. */
int ccdb_context_set_blocking_wait(ccdb_context* ctx, int32_t on);

/* Persistent sweep kernels launched by this context's fits use at most
 * max_ctas CTAs (0: one per SM, the default).  Contexts that run fits at the
 * same time on one GPU (the serving loop's slots) split the SMs between them
 * so that every persistent grid can be resident at once.  No reference
 * counterpart (the reference runs one fit per thread on the CPU). */
int ccdb_context_set_max_ctas(ccdb_context* ctx, int32_t max_ctas);

/* Upload a column-major CompressedDataMatrix (CompressedDataMatrix.h:40-452).
 * col_start[J+1] offsets into rows[] (SPARSE/INDICATOR entries, row ids ascending);
 * val_start[J+1] offsets into vals[] (SPARSE: one per entry; DENSE: K values);
 * fmt[J] per-column FormatType.  The matrix is immutable and may be shared by
 * any number of fits of the same context.  Replaces ModelData::loadX. */
int ccdb_matrix_create(ccdb_context* ctx, int64_t K, int32_t J, const int64_t* col_start,
                       const int32_t* rows, const int64_t* val_start, const double* vals,
                       const uint8_t* fmt, ccdb_matrix** out);
int ccdb_matrix_destroy(ccdb_matrix* m);
/* The matrix's row-major copy, the one computeXBeta's row sums and the MM
 * cycle read (the transpose ModelSpecifics.hpp:313-361 walks), copied to host
 * buffers: row_ptr (K + 1 offsets), col and val (one entry per matrix entry,
 * DENSE and INTERCEPT columns at every row): per row the columns in increasing
 * order.  Built on the device on first use and kept with the matrix. */
int ccdb_matrix_row_major(ccdb_matrix* m, int64_t* row_ptr, int32_t* col, double* val);

typedef struct {
    int32_t model_type;    /* ModelType */
    int32_t precision;     /* CCDB_PRECISION_* */
    const double* y;       /* K outcomes (Cox: event indicator) */
    const double* time;    /* K survival times (Cox) or NULL */
    const int64_t* stratum; /* K stratum ids (CLR, Cox) or NULL */
    int32_t offset_col0;   /* column 0 is an offset with beta fixed at 1 */
} ccdb_fit_desc;

/* Per-fit state on the device (xBeta, offsExpXBeta, denominators, beta ...):
 * the device counterpart of ModelSpecifics<Model,Real> constructed by
 * AbstractModelSpecifics::factory (AbstractModelSpecifics.cpp:128-154) and
 * ModelSpecifics::initialize (ModelSpecifics.hpp:1899-1952). */
int ccdb_fit_create(ccdb_context* ctx, const ccdb_matrix* m, const ccdb_fit_desc* desc,
                    ccdb_fit** out);
int ccdb_fit_destroy(ccdb_fit* f);

/* --- per-coordinate operator API (AbstractModelSpecifics) ------------------ */

/* CV row weights, NULL = unweighted (ModelSpecifics::setWeights, ModelSpecifics.hpp:427-484,
 * followed by computeFixedTermsInLogLikelihood/GradientAndHessian :570-587, :589-603). */
int ccdb_set_weights(ccdb_fit* f, const double* weights);
/* beta[J] -> xBeta, offsExpXBeta, denominators (computeXBeta + computeRemainingStatistics,
 * CyclicCoordinateDescent.cpp:1452-1470, ModelSpecifics.hpp:1588-1633). */
int ccdb_set_beta(ccdb_fit* f, const double* beta);
/* beta[J] -> xBeta by ModelSpecifics::computeXBeta(double* beta, bool)
 * (ModelSpecifics.hpp:313-361), the MM cycle's product over hX.transpose():
 * that transpose gives every row one format (CompressedDataMatrix.cpp:151-209),
 * and when the matrix has an INDICATOR column and no DENSE column it keeps no
 * values, so every non-zero entry counts as 1.  Other matrices get X beta.
 * The remaining statistics are left to ccdb_compute_remaining_statistics. */
int ccdb_compute_xbeta(ccdb_fit* f, const double* beta);
/* computeNumeratorForGradient + computeGradientAndHessian for column j
 * (ModelSpecifics.hpp:1353-1464, 711-766). */
int ccdb_compute_gradient_hessian(ccdb_fit* f, int32_t j, double* gradient, double* hessian);
/* beta[j] += delta and updateXBeta (ModelSpecifics.hpp:1466-1586). */
int ccdb_update_xbeta(ccdb_fit* f, int32_t j, double delta);
/* computeRemainingStatistics (ModelSpecifics.hpp:1588-1633). */
int ccdb_compute_remaining_statistics(ccdb_fit* f);
/* getLogLikelihood (ModelSpecifics.hpp:605-650). */
int ccdb_get_log_likelihood(ccdb_fit* f, double* loglik);
/* getXBeta (ModelSpecifics.hpp:286-289): K values. */
int ccdb_get_xbeta(ccdb_fit* f, double* out);
int ccdb_get_beta(ccdb_fit* f, double* out);
/* getGradientObjective (ModelSpecifics.hpp:103-120): sum of y * xBeta (* weight). */
int ccdb_get_gradient_objective(ccdb_fit* f, double* out);
/* CyclicCoordinateDescent::setFixedBeta for every column (.cpp:384-386):
 * fixed[j] != 0 holds column j at its current beta in later mode finding; the
 * offset column stays fixed.  Host state only. */
int ccdb_set_fixed(ccdb_fit* f, const uint8_t* fixed);

/* --- calls on a fitted state ------------------------------------------------ */

/* Fisher information over the columns indices[0..n) on the current state:
 * out[i * n + j] for the pair (indices[i], indices[j]), symmetric, n x n.
 * Replaces CyclicCoordinateDescent::computeFisherInformation(indices)
 * (CyclicCoordinateDescent.cpp:1288-1299) and, with n = 2, the per-pair
 * ModelSpecifics::computeFisherInformation (ModelSpecifics.hpp:1203-1337,
 * AbstractModelSpecifics.h:68).  A weighted fit (ccdb_set_weights with
 * weights) is refused with CCDB_ERR_UNSUPPORTED, as the reference throws for
 * it (ModelSpecifics.hpp:1207-1208).  The strata cross terms of the grouped
 * and Cox models come from the current state on every call. */
int ccdb_fisher_information(ccdb_fit* f, const int32_t* indices, int32_t n, double* out);
/* Predictive log-likelihood of the current beta on held-out row weights
 * weights[K] (CyclicCoordinateDescent::getNewPredictiveLogLikelihood,
 * CyclicCoordinateDescent.cpp:319-355, over ModelSpecifics::
 * getPredictiveLogLikelihood, ModelSpecifics.hpp:652-690,
 * AbstractModelSpecifics.h:106).  The Cox model takes its risk sets under the
 * held-out weights and then returns to the fit's own weights. */
int ccdb_get_predictive_log_likelihood(ccdb_fit* f, const double* weights, double* out);
/* The MM algorithm's all-coordinate gradient and Hessian bound on the current
 * state (ModelSpecifics::computeMMGradientAndHessian, ModelSpecifics.hpp:776-889,
 * AbstractModelSpecifics.h:66): gradient[J], hessian[J]; columns with
 * fixed[j] != 0 give (0, 0) (fixed may be NULL).  Conditional logistic,
 * conditional Poisson and Cox fits; others return CCDB_ERR_UNSUPPORTED (the
 * reference's Poisson increment throws, and its MM set-up reads stratum ids that
 * unstratified data does not have). */
int ccdb_compute_mm_gradient_hessian(ccdb_fit* f, const uint8_t* fixed, double* gradient,
                                     double* hessian);
/* predictEstimate of each row's xBeta into y[K]: LR exp(xb)/(exp(xb)+1),
 * Poisson exp(xb), conditional and Cox models xb (getPredictiveEstimates,
 * ModelSpecifics.hpp:692-705, AbstractModelSpecifics.h:108).  With weights
 * non-NULL only rows whose weight is nonzero are written. */
int ccdb_get_predictive_estimates(ccdb_fit* f, const double* weights, double* y);

/* --- mode finding (CyclicCoordinateDescent::update) ------------------------ */

typedef struct {
    const int32_t* prior_type; /* J, PriorType per column */
    const double* prior_var;   /* J, prior variance per column */
    int32_t convergence_type;  /* ConvergenceType */
    double tolerance;          /* default 1e-6 (CcdInterface.h:83-93) */
    int32_t max_iterations;    /* default 1000 */
    double initial_bound;      /* default 2.0 */
    int32_t max_bound_count;   /* default 5 */
    int32_t per_coordinate;    /* 0: on-device mode finding (default); 1: host loop over
                                  the per-coordinate calls above (the reference's call pattern) */
    int32_t strategy;          /* sweep strategy.  Logistic/Poisson: CCDB_SWEEP_AUTO runs
                                  the resident sweep (one CTA, the row state in shared
                                  memory) when the fit's rows fit it, else the cluster
                                  sweep; _RESIDENT asks for the resident sweep (beyond
                                  shared memory its global form, the row state in device
                                  memory); _LEVELS runs the cluster sweep (one
                                  launch per findMode over dependency levels),
                                  _GRID_LEVELS the grid-wide level sweep,
                                  _SPECULATIVE host-driven batches of gradients that restart
                                  after each nonzero step.  Cox and conditional models: one
                                  persistent launch per findMode of device-driven speculative
                                  batches -- one thread-block cluster with hardware barriers
                                  for fits a few SMs cover (forced by _LEVELS), else a
                                  cooperative grid (forced by _GRID_LEVELS) -- or with
                                  _SPECULATIVE the host-driven batches */
    int32_t algorithm;         /* AlgorithmType (Types.h:149-153): CCDB_ALGORITHM_CCD (0,
                                  default) or CCDB_ALGORITHM_MM (findMode's MM cycle,
                                  CyclicCoordinateDescent.cpp:974-1001; conditional logistic,
                                  conditional Poisson and Cox fits only) */
    int32_t use_kkt_swindle;   /* ModeFindingArguments::useKktSwindle: 1 runs
                                  CyclicCoordinateDescent::kktSwindle (.cpp:636-826) when
                                  some column has a Laplace prior */
    const uint8_t* fixed;      /* J flags or NULL: setFixedBeta for every column (the
                                  offset column stays fixed); NULL keeps the fit's set */
} ccdb_mode_args;

#define CCDB_ALGORITHM_CCD 0
#define CCDB_ALGORITHM_MM 1

#define CCDB_SWEEP_AUTO 0
#define CCDB_SWEEP_LEVELS 1        /* one thread-block cluster, levels ordered by cluster barriers */
#define CCDB_SWEEP_SPECULATIVE 2
#define CCDB_SWEEP_GRID_LEVELS 3   /* one CTA per SM, levels ordered by global counters */
#define CCDB_SWEEP_RESIDENT 4      /* one CTA, the row state in shared memory (or device memory) */

typedef struct {
    int32_t return_flag;        /* UpdateReturnFlags */
    int32_t iterations;         /* sweeps of the last findMode */
    double log_likelihood;
    double objective;           /* last convergence objective */
    int64_t coordinate_updates; /* ccdUpdateBeta calls over all sweeps */
    double device_seconds;      /* device-timeline span of the call (CUDA events on the
                                   engine's stream): ccdb_find_mode from its first to its last
                                   device operation; ccdb_fit_model from the first upload to
                                   the copy of beta back to the host */
    double kernel_seconds;      /* span of the fused sweep launches alone */
    int64_t kernel_launches;    /* engine kernels launched by the call */
    int32_t attempts;           /* findMode runs: 1, plus one per ILLCONDITIONED retry */
    int32_t sweeps_total;       /* cycles over every attempt (iterations counts the last) */
    int64_t nonzero_steps;      /* coordinate steps that moved a coefficient, every attempt;
                                   -1 where the sweep used does not count them */
} ccdb_fit_result;

/* Run CyclicCoordinateDescent::update (.cpp:586-615): findMode, with the
 * ILLCONDITIONED retry shrinking the bound.  beta_inout[J]: starting values in,
 * the mode out (NULL: start from 0 / offset 1, discard). */
int ccdb_find_mode(ccdb_fit* f, const ccdb_mode_args* args, double* beta_inout,
                   ccdb_fit_result* result);

/* One-call fit from host buffers: upload, find the mode, copy beta back.  The
 * reference-facing convenience used by fitCyclopsModel-style callers. */
int ccdb_fit_model(ccdb_context* ctx, int64_t K, int32_t J, const int64_t* col_start,
                   const int32_t* rows, const int64_t* val_start, const double* vals,
                   const uint8_t* fmt, const ccdb_fit_desc* desc, const double* weights,
                   const ccdb_mode_args* args, double* beta_out, ccdb_fit_result* result);

/* --- batched fits: the cross-validation grid ------------------------------- */

typedef struct {
    int32_t n_instances;
    const int32_t* row_fold; /* K fold id per row, or NULL (no row held out) */
    const int32_t* holdout;  /* n_instances: fold held out by each instance (-1: none) */
    const double* variance;  /* n_instances: prior variance of the regularised columns */
    int32_t group;           /* CCDB_PRECISION_MIXED fits: instances stepped in lockstep per CTA
                                (1, 2 or 4); 0 lets the engine choose.  Ignored for FP64 fits. */
    int32_t cluster;         /* CCDB_PRECISION_MIXED fits: CTAs per group, each owning a range of
                                rows (1..16); 0 lets the engine choose.  Ignored for FP64 fits. */
} ccdb_batch_desc;

typedef struct {
    int32_t return_flag;
    int32_t iterations;
    double log_likelihood;     /* on the instance's training rows */
    double objective;
    double predictive_loglik;  /* on its held-out rows (getPredictiveLogLikelihood,
                                  ModelSpecifics.hpp:652-690) */
    int64_t steps;             /* coordinate steps over all sweeps */
    int64_t updates;           /* nonzero steps */
    int64_t update_entries;    /* column entries touched by the nonzero steps */
    int64_t gradient_entries;  /* column entries gathered for gradients */
} ccdb_batch_result;

/* Fit n_instances models over the fit's matrix and outcomes in one launch:
 * instance i weights rows 0 on fold holdout[i] and 1 elsewhere (the weights
 * CrossValidationSelector::getWeights gives, drivers/CrossValidationSelector.cpp:72-130),
 * uses args->prior_type per column with variance[i], and starts from beta = 0.
 * Each instance runs the sequential sweep of a standalone fit; instances do not
 * interact.  Logistic and Poisson models.  beta_out: n_instances x J.
 * A CCDB_PRECISION_MIXED fit runs the mixed-precision engine, whose instances
 * step through the columns in lockstep groups of batch->group (at most
 * 16,777,215 rows; held-out fold ids below 127). */
int ccdb_batch_find_mode(ccdb_fit* f, const ccdb_batch_desc* batch, const ccdb_mode_args* args,
                         double* beta_out, ccdb_batch_result* results, double* device_seconds);

/* --- allocation-free gradient (no reference counterpart) -------------------- */

/* For callers that cannot allocate device memory -- code running while a
 * stream is captured into a CUDA graph, hosts whose device memory belongs to
 * a pool they must not grow, embedders given a fixed device arena: the
 * gradient and Hessian of one column of a logistic or Poisson model, computed
 * from device buffers the caller owns.  This entry point has no counterpart
 * in the reference; it allocates nothing.
 *   rows[n_entries] (SPARSE/INDICATOR) and vals[n_entries] (SPARSE/DENSE):
 *     the column, device memory; fmt is its FormatType; DENSE/INTERCEPT
 *     columns cover rows 0..n_entries-1.
 *   row_state: device array of 4 doubles per row {xBeta, offsExpXBeta,
 *     denominator, weight} (weight 1 when unweighted).
 *   xjy: the column's sum of x*y*weight.  out: device array of 2 doubles,
 *     receives (gradient, Hessian) as computeGradientAndHessian defines them.
 *   stream: a cudaStream_t (NULL: the default stream); the call only enqueues
 *     work and returns, so synchronise before reading out.
 * Partial sums go to a fixed scratch array compiled into the library (2,048
 * slots; columns of at most 16,777,216 entries -- longer ones are rejected with
 * CCDB_ERR_INVALID before anything is launched).  Every GPU that loads the
 * library holds that array until the process exits.  All calls share it and
 * it keeps the last call's contents (each call overwrites the slots it
 * reads); calls whose kernels overlap on the GPU race on it.  The first call
 * on each device looks up the array's device address and loads this entry
 * point's kernels there (no allocation): make one call on a device before any
 * stream capture, and do not reset the device (cudaDeviceReset) afterwards,
 * since the address is kept for the life of the process. */
int ccdb_column_gradient_hessian_noalloc(int32_t model_type, int32_t fmt, int64_t n_entries,
                                         const int32_t* rows, const double* vals,
                                         const double* row_state, double xjy, double* out,
                                         void* stream);

/* --- inspection (no reference counterpart) ---------------------------------- */

/* The checks ccdb_matrix_create applies before any device work: offsets start
 * at 0 and never decrease; DENSE columns hold K values and no rows, INTERCEPT
 * nothing, INDICATOR rows only, SPARSE one value per row; row ids strictly
 * ascending within a column and < K.  CCDB_ERR_INVALID with the first
 * violation in ccdb_last_error.  Host-only: needs no GPU. */
int ccdb_matrix_validate(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                         const int64_t* val_start, const double* vals, const uint8_t* fmt);

/* Bound, in nanoseconds, on every single device-side wait of this fit's later
 * launches: the grid-wide level sweep's waits for a level, a split column and
 * the grid barrier (default 20 s), and the mixed batch engine's wait for the
 * per-column sums of the other CTAs of its cluster (default 2 s).  0 restores
 * the defaults.  A wait that runs out ends the call with CCDB_ERR_TIMEOUT and
 * leaves the context usable; the fit's state is then undefined until the next
 * ccdb_set_beta or ccdb_find_mode with starting values.  The cluster sweep
 * (CCDB_SWEEP_LEVELS) has no such wait.  No reference counterpart. */
int ccdb_fit_set_wait_limit(ccdb_fit* f, int64_t nanoseconds);

/* Device time (CUDA events on the fit's stream) of the kernels of the fit's last
 * ccdb_fisher_information call, in seconds; copies to and from the host are
 * outside it.  0 before any such call. */
int ccdb_get_last_call_seconds(const ccdb_fit* f, double* seconds);

/* Dependency level of every column in one fused sweep over this matrix
 * (independent-row models: columns conflict when they share a row).  Columns
 * on one level touch disjoint rows; running levels in order reproduces the
 * reference's visiting order j = 0..J-1 (CyclicCoordinateDescent.cpp:1008-1021).
 * fixed[j] != 0 marks columns the sweep skips (level -1).  Host-only: needs no
 * GPU. */
int ccdb_sweep_levels(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                      const uint8_t* fmt, const uint8_t* fixed, int32_t* level_out,
                      int32_t* n_levels);

#ifdef __cplusplus
}
#endif
#endif /* CCDB_H */
