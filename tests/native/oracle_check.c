/* oracle_check.c -- host run of the oracle restatement (oracle/ccd_oracle.c)
 * under AddressSanitizer and UndefinedBehaviorSanitizer, built by
 * tests/test_host_sanitizers.py.  Random small problems of every model and
 * column format, with and without weights (zero weights included) and fixed
 * columns, through every call: the CCD, KKT-swindle and MM fits, per-coordinate
 * gradients and updates, log-likelihood and prior, Fisher information,
 * predictive log-likelihood and estimates, Cox grouping.  The checks here are
 * the sanitizers' (no out-of-bounds access, leak or undefined behaviour) plus
 * finite results; the oracle's values are pinned by the Python tests.
 * Exit status 0 when every case runs clean. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccd_oracle.h"

enum { MT_POISSON = 2, MT_LOGISTIC = 3, MT_CLR = 4, MT_CPR = 6, MT_COX = 8 };
enum { F_DENSE = 0, F_SPARSE = 1, F_INDICATOR = 2, F_INTERCEPT = 3 };

static uint64_t state = 0x9E3779B97F4A7C15ull;
static double unif(void) { /* xorshift64* */
    state ^= state >> 12;
    state ^= state << 25;
    state ^= state >> 27;
    return (double)((state * 2685821657736338717ull) >> 11) * (1.0 / 9007199254740992.0);
}
static int irand(int n) { return (int)(unif() * n); }

static int failures = 0;

static void run_case(int id) {
    static const int models[5] = {MT_LOGISTIC, MT_POISSON, MT_CLR, MT_CPR, MT_COX};
    const int model = models[id % 5];
    const int64_t K = 20 + irand(120);
    const int P = 1 + irand(10);
    const int grouped = (model == MT_CLR || model == MT_CPR || model == MT_COX);
    const int intercept = !grouped && irand(2);
    const int J = P + intercept;
    int64_t* col_start = calloc(J + 1, sizeof(int64_t));
    int64_t* val_start = calloc(J + 1, sizeof(int64_t));
    int32_t* rows = malloc(sizeof(int32_t) * (size_t)(K * J + 1));
    double* vals = malloc(sizeof(double) * (size_t)(K * J + 1));
    uint8_t* fmt = calloc(J, 1);
    int32_t* ptype = calloc(J, sizeof(int32_t));
    double* pvar = calloc(J, sizeof(double));
    int64_t nr = 0, nv = 0;
    for (int j = 0; j < J; ++j) {
        fmt[j] = (intercept && j == 0) ? F_INTERCEPT : (uint8_t)irand(3);
        ptype[j] = (intercept && j == 0) ? 0 : irand(3);
        pvar[j] = 0.1 + unif() * 2.0;
        if (fmt[j] == F_DENSE) {
            for (int64_t k = 0; k < K; ++k) vals[nv++] = unif() * 2.0 - 1.0;
        } else if (fmt[j] != F_INTERCEPT) {
            for (int64_t k = 0; k < K; ++k)
                if (unif() < 0.3) {
                    rows[nr++] = (int32_t)k;
                    if (fmt[j] == F_SPARSE) vals[nv++] = 0.2 + unif();
                }
        }
        col_start[j + 1] = nr;
        val_start[j + 1] = nv;
    }
    double* y = malloc(sizeof(double) * K);
    double* time = NULL;
    int64_t* stratum = NULL;
    if (grouped) {
        stratum = malloc(sizeof(int64_t) * K);
        const int n_strata = 1 + irand(12);
        for (int64_t k = 0; k < K; ++k) stratum[k] = (k * n_strata) / K;
    }
    for (int64_t k = 0; k < K; ++k) {
        if (model == MT_POISSON || model == MT_CPR) y[k] = (double)irand(4);
        else y[k] = unif() < 0.35 ? 1.0 : 0.0;
    }
    if (model == MT_CLR) /* one case per stratum, as a matched design */
        for (int64_t k = 0; k < K; ++k) y[k] = (k == 0 || stratum[k] != stratum[k - 1]) ? 1.0 : 0.0;
    if (model == MT_COX) { /* rows in (stratum, -time, y) order, ties on a coarse grid */
        time = malloc(sizeof(double) * K);
        double t = 100.0;
        for (int64_t k = 0; k < K; ++k) {
            if (k > 0 && stratum[k] != stratum[k - 1]) t = 100.0;
            if (unif() < 0.6) t -= 1.0;
            time[k] = t;
        }
        for (int64_t k = 1; k < K; ++k) /* within a tie, censored before events */
            if (stratum[k] == stratum[k - 1] && time[k] == time[k - 1] && y[k] < y[k - 1]) {
                double tmp = y[k];
                y[k] = y[k - 1];
                y[k - 1] = tmp;
            }
    }
    char err[256];
    void* h = orc_create(model, 0, K, J, y, time, stratum, col_start, rows, val_start, vals, fmt, 0, ptype,
                         pvar, err, sizeof err);
    if (!h) {
        fprintf(stderr, "case %d: create failed: %s\n", id, err);
        ++failures;
        goto done;
    }
    double* w = NULL;
    if (irand(3) == 0) {
        w = malloc(sizeof(double) * K);
        for (int64_t k = 0; k < K; ++k) w[k] = irand(4) == 0 ? 0.0 : 0.5 + unif();
        orc_set_weights(h, w);
    }
    uint8_t* fixed = calloc(J, 1);
    if (J > 1 && irand(2)) fixed[1 + irand(J - 1)] = 1;
    double* beta = malloc(sizeof(double) * J);
    double ll, lp;
    int iters, flag;
    const int algorithm = grouped && irand(2);
    const int kkt = irand(2);
    int rc = orc_fit(h, irand(3), 1e-6, 200, 2.0, 5, algorithm, kkt, fixed, beta, &ll, &iters, &flag, err,
                     sizeof err);
    if (rc == 0 && !isfinite(ll) && flag == 0) {
        fprintf(stderr, "case %d: non-finite log-likelihood with a successful flag\n", id);
        ++failures;
    }
    /* an MM fit may stop with the reference's "Non-increasing!" error: that is a result, not a fault */
    for (int j = 0; j < J; ++j) {
        double g, hs;
        orc_grad_hess(h, j, &g, &hs);
        orc_update_beta(h, j, 0.01);
    }
    orc_loglik(h, &ll);
    orc_log_prior(h, &lp);
    int32_t* idx = malloc(sizeof(int32_t) * (J + 1));
    for (int j = 0; j < J; ++j) idx[j] = j;
    idx[J] = 0; /* a repeat */
    double* info = malloc(sizeof(double) * (size_t)(J + 1) * (J + 1));
    orc_fisher_information(h, idx, J + 1, info);
    double* held = malloc(sizeof(double) * K);
    for (int64_t k = 0; k < K; ++k) held[k] = (k % 3 == 0) ? 1.0 : 0.0;
    double pll;
    orc_predictive_loglik(h, held, &pll);
    double* est = calloc(K, sizeof(double));
    orc_predictive_estimates(h, w, est);
    double* xb = malloc(sizeof(double) * K);
    orc_get_xbeta(h, xb);
    if (model == MT_COX) {
        int32_t* grp = malloc(sizeof(int32_t) * K);
        int32_t* reset = malloc(sizeof(int32_t) * (K + 2));
        int nreset = 0;
        orc_cox_groups(h, grp, reset, &nreset);
        free(grp);
        free(reset);
    }
    orc_destroy(h);
    free(w);
    free(fixed);
    free(beta);
    free(idx);
    free(info);
    free(held);
    free(est);
    free(xb);
done:
    free(col_start);
    free(val_start);
    free(rows);
    free(vals);
    free(fmt);
    free(ptype);
    free(pvar);
    free(y);
    free(time);
    free(stratum);
}

int main(int argc, char** argv) {
    const int cases = argc > 1 ? atoi(argv[1]) : 300;
    for (int i = 0; i < cases; ++i) run_case(i);
    if (failures) {
        fprintf(stderr, "%d case(s) failed\n", failures);
        return 1;
    }
    printf("%d oracle cases ran clean\n", cases);
    return 0;
}
