/* ccd_oracle.h -- ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference Cyclops coordinate-descent path
 * (ModelSpecifics + CyclicCoordinateDescent + Laplace/Normal/None priors) in
 * FP64.  Used only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the checker; the product never links it.  Every function
 * cites the reference file:line it restates (paths relative to the reference
 * project root).  The argument lists mirror oracle/ref_driver.cpp so the two
 * checkers are interchangeable.
 */
#ifndef CCD_ORACLE_H
#define CCD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void* orc_create(int model_type, int fp32_unused, int64_t K, int J, const double* y,
                 const double* time, const int64_t* stratum, const int64_t* col_start,
                 const int32_t* rows, const int64_t* val_start, const double* vals,
                 const uint8_t* fmt, int offset_col0, const int32_t* prior_type,
                 const double* prior_var, char* err, int errlen);
void orc_destroy(void* h);
int orc_set_weights(void* h, const double* w);
int orc_set_beta(void* h, const double* beta);
/* algorithm: 0 CCD, 1 MM (AlgorithmType, Types.h:149-153); use_kkt: the KKT
 * swindle (ModeFindingArguments::useKktSwindle); fixed: J flags or NULL. */
int orc_fit(void* h, int conv_type, double tol, int max_iter, double initial_bound,
            int max_bound_count, int algorithm, int use_kkt, const uint8_t* fixed, double* beta_out,
            double* ll_out, int* iters_out, int* flag_out, char* err, int errlen);
/* Cycles of each findMode attempt of the last orc_fit (the ILLCONDITIONED
 * retry runs several); returns the number of attempts, writes at most max_n. */
int orc_fit_attempts(void* h, int* sweeps, int max_n);
int orc_grad_hess(void* h, int j, double* g, double* hs);
int orc_update_beta(void* h, int j, double delta);
int orc_loglik(void* h, double* ll);
int orc_log_prior(void* h, double* lp);
int orc_get_beta(void* h, double* out);
int orc_get_xbeta(void* h, double* out);
int orc_predictive_loglik(void* h, const double* w, double* out);
int orc_num_patients(void* h);
/* Fisher information of the current state over columns idx[0..n) (n x n,
 * row-major); -2 for a weighted fit, which the reference refuses. */
int orc_fisher_information(void* h, const int32_t* idx, int n, double* out);
/* predictEstimate per row; rows whose weight is zero keep y (w may be NULL). */
int orc_predictive_estimates(void* h, const double* w, double* y);
/* Test hook: exp moved by one ulp on 2 in one_in arguments (0: off); see ccd_oracle.c. */
void orc_set_exp_perturbation(unsigned one_in, unsigned salt);
/* Cox grouping as setPidForAccumulation computes it: group id per row (N for
 * dropped rows), the stratum-start list accReset, returns N. */
int orc_cox_groups(void* h, int32_t* group_out, int32_t* acc_reset_out, int* n_reset_out);

#ifdef __cplusplus
}
#endif
#endif
