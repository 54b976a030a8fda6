/* ccd_oracle.c -- ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C, FP64 restatement of the reference Cyclops cyclic-coordinate-descent
 * path.  It is the checker for the CUDA implementation (tests, smoke, the CPU
 * baseline leg of bench.py); the product never links or calls it.  It is
 * itself pinned against the reference engine compiled from source
 * (oracle/_ref/libccd_ref.so) and the committed golden fixtures.
 *
 * Citations are "file:line" relative to the reference project root; MS.hpp
 * abbreviates src/cyclops/engine/ModelSpecifics.hpp, MS.h its .h, CCD.cpp
 * src/cyclops/CyclicCoordinateDescent.cpp, CP.h src/cyclops/priors/CovariatePrior.h.
 *
 * Models: LOGISTIC, POISSON (IndependentData), CONDITIONAL_LOGISTIC,
 * CONDITIONAL_POISSON (GroupedData), COX = Breslow-tied Cox (OrderedWithTiesData).
 */
#include "ccd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* reference ModelType numbering (src/cyclops/Types.h:134-147) */
enum { MT_POISSON = 2, MT_LOGISTIC = 3, MT_CLR = 4, MT_CPR = 6, MT_COX = 8 };
/* FormatType (src/cyclops/CompressedDataMatrix.h:36-38) */
enum { F_DENSE = 0, F_SPARSE = 1, F_INDICATOR = 2, F_INTERCEPT = 3 };
/* ConvergenceType (Types.h:108-114) and UpdateReturnFlags (Types.h:124-130) */
enum { C_GRADIENT = 0, C_LANGE = 1, C_MITTAL = 2 };
enum { R_SUCCESS = 0, R_MAX_ITERATIONS = 2, R_ILLCONDITIONED = 3 };

#define ORC_MAX_ATTEMPTS 16
#define ORC_PI 3.14159265358979323851280895940618620443274267017841339111328125

/* Test hook: a copy of the arithmetic with exp moved by one unit in the last
 * place on a deterministic pseudo-random share of its arguments (2 in
 * `one_in`, chosen by a hash of the argument's bits and `salt`; 0 turns it
 * off).  Parity tests use it to see whether a problem's result is decided by
 * rounding: glibc's exp itself is not correctly rounded on every argument,
 * and the CUDA engine's exp is a different implementation, so a result that
 * moves when exp moves by one ulp cannot be held to a tolerance tighter than
 * that movement.  Off by default; nothing in the product calls it. */
static unsigned g_exp_one_in = 0, g_exp_salt = 0;
void orc_set_exp_perturbation(unsigned one_in, unsigned salt) {
    g_exp_one_in = one_in;
    g_exp_salt = salt;
}
static double orc_exp(double x) {
    double r = exp(x);
    if (g_exp_one_in == 0) return r;
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    b ^= (uint64_t)g_exp_salt * 0x9e3779b97f4a7c15ULL;
    b ^= b >> 33;
    b *= 0xff51afd7ed558ccdULL;
    b ^= b >> 33;
    b *= 0xc4ceb9fe1a85ec53ULL;
    b ^= b >> 33;
    const unsigned m = (unsigned)(b % g_exp_one_in);
    if (m == 0) return nextafter(r, INFINITY);
    if (m == 1) return nextafter(r, -INFINITY);
    return r;
}

typedef struct {
    int model;
    int64_t K;
    int J, N, Npatients;
    double *y, *offs;
    int32_t* pid0; /* stratum index per row as ModelData::loadY assigns it, or NULL */
    int64_t *col_start, *val_start;
    int32_t* rows;
    double* vals;
    uint8_t* fmt;
    int offset_col0;
    int32_t* prior_type;
    double* prior_var;

    double *kw, *nw, *xb, *e, *denom, *numer, *numer2, *acc;
    int32_t* hpid; /* group per row (COX after regrouping, CLR = pid0) */
    int32_t* acc_reset;
    int n_reset;
    int32_t** sidx;
    int* sidx_n;
    double *xjy, llfixed;
    double *beta, *hdelta, bound;
    uint8_t* fix;
    double* w; /* CV weights or NULL */
    int valid_weights, xb_known, suff_known, touched_y;
    int last_flag, last_iter;
    /* cycles of each findMode attempt of the last orc_fit (the ILLCONDITIONED
     * retry of CyclicCoordinateDescent::update, CCD.cpp:598-614) */
    int n_attempts, attempt_sweeps[ORC_MAX_ATTEMPTS];
} Orc;

static int is_indep(const Orc* o) { return o->model == MT_LOGISTIC || o->model == MT_POISSON; }
static int is_cox(const Orc* o) { return o->model == MT_COX; }
static int is_grouped(const Orc* o) { return o->model == MT_CLR || o->model == MT_CPR; }
static int group_of(const Orc* o, int64_t k) { return is_indep(o) ? (int)k : o->hpid[k]; }
static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max semantics */
static int sgn(double x) { return x == 0 ? 0 : (x < 0 ? -1 : 1); } /* CP.h:310-318 */

/* Column iteration helpers: INTERCEPT/DENSE cover all K rows (Iterators.h). */
static int64_t col_len(const Orc* o, int j) {
    switch (o->fmt[j]) {
    case F_INTERCEPT:
        return o->K;
    case F_DENSE:
        return o->val_start[j + 1] - o->val_start[j];
    default:
        return o->col_start[j + 1] - o->col_start[j];
    }
}
static int64_t col_row(const Orc* o, int j, int64_t p) {
    return (o->fmt[j] == F_INTERCEPT || o->fmt[j] == F_DENSE) ? p : o->rows[o->col_start[j] + p];
}
static double col_val(const Orc* o, int j, int64_t p) {
    switch (o->fmt[j]) {
    case F_DENSE:
    case F_SPARSE:
        return o->vals[o->val_start[j] + p];
    default:
        return 1.0;
    }
}
static int col_is_indicator(const Orc* o, int j) { /* IteratorType::isIndicator */
    return o->fmt[j] == F_INDICATOR || o->fmt[j] == F_INTERCEPT;
}
/* getNumberOfNonZeroEntries, CompressedDataMatrix.cpp:92-100 */
static int64_t col_nnz(const Orc* o, int j) {
    return (o->fmt[j] == F_INTERCEPT || o->fmt[j] == F_DENSE) ? o->K : col_len(o, j);
}

static double obs_count(const Orc* o, double y) { /* observationCount, MS.h:986,1492,816,1178 */
    return is_indep(o) ? 1.0 : y;
}
static double null_denom(const Orc* o) { return o->model == MT_LOGISTIC ? 1.0 : 0.0; } /* MS.h:980 */

/* setPidForAccumulation, MS.hpp:1809-1868 (+ setupSparseIndices :1870-1892) */
static void set_pid_for_accumulation(Orc* o, const double* weights) {
    const int ignore = -1;
    int64_t K = o->K;
    for (int64_t k = 0; k < K; ++k) o->hpid[k] = o->pid0 ? o->pid0[k] : 0;
    o->n_reset = 0;
    int64_t index = 0;
    while (weights != NULL && weights[index] == 0.0 && index < K) {
        o->hpid[index] = ignore;
        index++;
    }
    int lastPid = o->hpid[index];
    double lastTime = o->offs[index];
    double lastEvent = o->y[index];
    int pid = o->hpid[index] = 0;
    for (int64_t k = index + 1; k < K; ++k) {
        if (weights == NULL || weights[k] != 0.0) {
            int nextPid = o->hpid[k];
            if (nextPid != lastPid) {
                pid++;
                o->acc_reset[o->n_reset++] = pid;
                lastPid = nextPid;
            } else {
                if (lastEvent == 1.0 && lastTime == o->offs[k] && lastEvent == o->y[k]) {
                    /* tie: same risk-set group */
                } else {
                    pid++;
                }
            }
            lastTime = o->offs[k];
            lastEvent = o->y[k];
            o->hpid[k] = pid;
        } else {
            o->hpid[k] = ignore;
        }
    }
    pid++;
    o->acc_reset[o->n_reset++] = pid;
    o->N = pid;
    if (weights != NULL)
        for (int64_t i = 0; i < K; ++i)
            if (o->hpid[i] == ignore) o->hpid[i] = o->N;

    /* setupSparseIndices: sorted unique group ids < N per non-dense column */
    for (int j = 0; j < o->J; ++j) {
        free(o->sidx[j]);
        o->sidx[j] = NULL;
        o->sidx_n[j] = 0;
        if (o->fmt[j] == F_DENSE || o->fmt[j] == F_INTERCEPT) continue;
        int64_t n = col_len(o, j);
        o->sidx[j] = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
        int cnt = 0;
        int last = -1;
        for (int64_t p = 0; p < n; ++p) { /* rows ascending => groups non-decreasing */
            int i = o->hpid[col_row(o, j, p)];
            if (i < o->N && i != last) {
                o->sidx[j][cnt++] = i;
                last = i;
            }
        }
        o->sidx_n[j] = cnt;
    }
}

/* setWeights, MS.hpp:427-484 */
static void set_weights_ms(Orc* o) {
    for (int64_t k = 0; k < o->K; ++k) o->kw[k] = o->w ? o->w[k] : 1.0;
    if (is_cox(o)) set_pid_for_accumulation(o, o->w);
    for (int i = 0; i <= o->N; ++i) o->nw[i] = 0.0;
    for (int64_t k = 0; k < o->K; ++k) o->nw[group_of(o, k)] += obs_count(o, o->y[k]) * o->kw[k];
}

/* computeFixedTermsInLogLikelihood, MS.hpp:570-587; Poisson term MS.h:1596-1601 */
static void fixed_ll(Orc* o) {
    o->llfixed = 0.0;
    if (o->model != MT_POISSON && o->model != MT_CPR) return;
    for (int64_t i = 0; i < o->K; ++i) {
        double t = 0.0;
        for (int c = 2; c <= (int)o->y[i]; c++) {
            if (o->model == MT_POISSON) t += -log((double)c);
            else t -= log((double)c);
        }
        o->llfixed += o->w ? t * o->kw[i] : t;
    }
}

/* computeXjY, MS.hpp:486-524 */
static void compute_xjy(Orc* o) {
    for (int j = 0; j < o->J; ++j) {
        double s = 0.0;
        int64_t n = col_len(o, j);
        for (int64_t p = 0; p < n; ++p) {
            int64_t k = col_row(o, j, p);
            double x = col_val(o, j, p);
            double yy = is_cox(o) ? obs_count(o, o->y[k]) : o->y[k];
            if (o->w) s += x * yy * o->kw[k];
            else s += x * yy;
        }
        o->xjy[j] = s;
    }
}

/* CyclicCoordinateDescent::computeXBeta, CCD.cpp:1452-1470 (zeroXBeta + axpyXBeta) */
static void compute_xbeta(Orc* o) {
    memset(o->xb, 0, sizeof(double) * o->K);
    for (int j = 0; j < o->J; ++j) {
        double b = o->beta[j];
        if (b == 0.0) continue;
        int64_t n = col_len(o, j);
        for (int64_t p = 0; p < n; ++p) o->xb[col_row(o, j, p)] += b * col_val(o, j, p);
    }
}

/* The MM cycle's xBeta: ModelSpecifics::computeXBeta (MS.hpp:313-361) over
 * hX.transpose() (CompressedDataMatrix.cpp:151-209).  The transpose gives all
 * rows one format: INDICATOR when some column is INDICATOR and none is DENSE,
 * DENSE when some column is DENSE and none is INDICATOR, else SPARSE.  Only
 * the INDICATOR transpose changes the product: it keeps no values, so every
 * entry of non-zero value counts as 1 (a SPARSE column's values are lost).
 * The row sums run in increasing column order, as compute_xbeta's do. */
static void compute_xbeta_mm(Orc* o) {
    int any_indicator = 0, any_dense = 0;
    for (int j = 0; j < o->J; ++j) {
        any_indicator |= o->fmt[j] == F_INDICATOR;
        any_dense |= o->fmt[j] == F_DENSE;
    }
    if (!any_indicator || any_dense) {
        compute_xbeta(o);
        return;
    }
    memset(o->xb, 0, sizeof(double) * o->K);
    for (int j = 0; j < o->J; ++j) {
        double b = o->beta[j];
        if (b == 0.0) continue;
        int64_t n = col_len(o, j);
        for (int64_t p = 0; p < n; ++p)
            if (col_val(o, j, p) != 0.0) o->xb[col_row(o, j, p)] += b;
    }
}

/* computeAccumlatedDenominator, MS.hpp:1670-1715 (Breslow: one-way scan) */
static void acc_denominator(Orc* o) {
    if (!is_cox(o)) return;
    double total = 0.0;
    int r = 0;
    for (int i = 0; i < o->N; ++i) {
        if (o->acc_reset[r] == i) {
            total = 0.0;
            ++r;
        }
        total += o->denom[i];
        o->acc[i] = total;
    }
}

/* computeRemainingStatisticsImpl, MS.hpp:1588-1617 */
static void remaining_statistics(Orc* o) {
    for (int i = 0; i < o->N; ++i) o->denom[i] = null_denom(o);
    for (int64_t k = 0; k < o->K; ++k) {
        o->e[k] = orc_exp(o->xb[k]);
        if (is_cox(o)) o->denom[group_of(o, k)] += o->w ? o->kw[k] * orc_exp(o->xb[k]) : orc_exp(o->xb[k]);
        else o->denom[group_of(o, k)] += o->e[k];
    }
    acc_denominator(o);
}

/* getLogLikelihood, MS.hpp:605-650 */
static double log_likelihood(Orc* o) {
    double ll = 0.0;
    for (int64_t i = 0; i < o->K; ++i) {
        int yi = (int)o->y[i]; /* logLikeNumeratorContrib takes int yi (MS.h:440, :461) */
        double c = is_cox(o) ? (yi != 1 ? 0.0 : o->xb[i]) : yi * o->xb[i];
        ll += o->w ? c * o->kw[i] : c;
    }
    for (int i = 0; i < o->N; ++i) {
        double d = is_cox(o) ? o->acc[i] : o->denom[i];
        double c = (o->model == MT_POISSON) ? o->nw[i] * d : o->nw[i] * log(d);
        ll -= c;
    }
    if (o->model == MT_POISSON || o->model == MT_CPR) ll += o->llfixed;
    return ll;
}

/* getGradientObjective, MS.hpp:103-120 */
static double gradient_objective(Orc* o) {
    double c = 0.0;
    for (int64_t i = 0; i < o->K; ++i) c += o->w ? o->xb[i] * o->y[i] * o->kw[i] : o->xb[i] * o->y[i];
    return c;
}

/* MixtureJointPrior::logDensity (JointPrior.h:121-128); CP.h:220-224 Laplace, :404-408 Normal */
static double log_prior(Orc* o) {
    double r = 0.0;
    for (int j = 0; j < o->J; ++j) {
        double x = o->beta[j], v = o->prior_var[j];
        if (o->prior_type[j] == 1) {
            double lambda = sqrt(2.0 / v);
            r += log(0.5 * lambda) - lambda * fabs(x);
        } else if (o->prior_type[j] == 2) {
            r += -0.5 * log(2.0 * ORC_PI * v) - 0.5 * x * x / v;
        }
    }
    return r;
}

/* CyclicCoordinateDescent::checkAllLazyFlags, CCD.cpp:388-406 */
static void check_lazy(Orc* o) {
    if (!o->xb_known) {
        compute_xbeta(o);
        o->xb_known = 1;
        o->suff_known = 0;
    }
    if (!o->valid_weights) {
        set_weights_ms(o);
        fixed_ll(o);
        compute_xjy(o);
        o->valid_weights = 1;
    }
    if (!o->suff_known) {
        remaining_statistics(o);
        o->suff_known = 1;
    }
}

/* computeNumeratorForGradient (+ incrementNumeratorForGradientImpl), MS.hpp:1353-1464 */
static void numerator_for_gradient(Orc* o, int j) {
    if (!is_cox(o)) return;
    int ind = col_is_indicator(o, j);
    if (o->fmt[j] == F_DENSE || o->fmt[j] == F_INTERCEPT) {
        for (int i = 0; i < o->N; ++i) {
            o->numer[i] = 0.0;
            o->numer2[i] = 0.0;
        }
    } else {
        for (int q = 0; q < o->sidx_n[j]; ++q) {
            o->numer[o->sidx[j][q]] = 0.0;
            if (!ind) o->numer2[o->sidx[j][q]] = 0.0;
        }
    }
    int64_t n = col_len(o, j);
    for (int64_t p = 0; p < n; ++p) {
        int64_t k = col_row(o, j, p);
        double x = col_val(o, j, p);
        int g = group_of(o, k);
        double c1 = o->e[k] * x;
        o->numer[g] += o->w ? o->kw[k] * c1 : c1;
        if (!ind) {
            double c2 = o->e[k] * x * x;
            o->numer2[g] += o->w ? o->kw[k] * c2 : c2;
        }
    }
}

/* Survival-style increment shared by CLR/CPR/Cox (MS.h:827-837, :1185-1201) */
static void inc_nevents(int indicator, double* g, double* h, double numer, double numer2, double denom,
                        double nEvents) {
    double t = numer / denom;
    double gg = nEvents * t;
    *g += gg;
    if (indicator) *h += gg * (1.0 - t);
    else *h += nEvents * (numer2 / denom - t * t);
}

/* computeGradientAndHessian(+Impl), MS.hpp:711-766 and :891-1201 */
static void gradient_hessian(Orc* o, int j, double* og, double* oh) {
    if (col_nnz(o, j) == 0) {
        *og = 0.0;
        *oh = 0.0;
        return;
    }
    const int ind = col_is_indicator(o, j);
    const int weighted = o->w != NULL;
    double g = 0.0, h = 0.0;
    if (is_cox(o)) { /* cumulative branch, MS.hpp:904-964 */
        const int dense = (o->fmt[j] == F_DENSE || o->fmt[j] == F_INTERCEPT);
        const int n = dense ? o->N : o->sidx_n[j];
        if (dense || n > 0) {
            double a1 = 0.0, a2 = 0.0;
            int r = 0;
            int first = dense ? 0 : o->sidx[j][0];
            while (o->acc_reset[r] < first) ++r;
            for (int q = 0; q < n; ++q) {
                int i = dense ? q : o->sidx[j][q];
                if (o->acc_reset[r] <= i) {
                    a1 = 0.0;
                    a2 = 0.0;
                    ++r;
                }
                a1 += o->numer[i];
                a2 += o->numer2[i];
                inc_nevents(ind, &g, &h, a1, a2, o->acc[i], o->nw[i]);
                if (!dense) { /* IteratorType::isSparse */
                    int next = (q + 1 < n) ? o->sidx[j][q + 1] : o->N;
                    for (++i; i < next; ++i) {
                        if (o->acc_reset[r] <= i) {
                            a1 = 0.0;
                            a2 = 0.0;
                            ++r;
                        }
                        inc_nevents(ind, &g, &h, a1, a2, o->acc[i], o->nw[i]);
                    }
                }
            }
        }
    } else if (is_indep(o)) { /* MS.hpp:1022-1038 */
        int64_t len = col_len(o, j);
        for (int64_t p = 0; p < len; ++p) {
            int64_t i = col_row(o, j, p);
            double x = col_val(o, j, p);
            double n1 = o->e[i] * x;
            double n2 = ind ? 0.0 : o->e[i] * x * x;
            double wt = o->nw[i];
            if (o->model == MT_LOGISTIC) { /* Logistic::incrementGradientAndHessian, MS.h:541-568 */
                double gg = n1 / o->denom[i];
                g += weighted ? wt * gg : gg;
                if (ind) h += weighted ? wt * gg * (1.0 - gg) : gg * (1.0 - gg);
                else h += weighted ? wt * (n2 / o->denom[i] - gg * gg) : (n2 / o->denom[i] - gg * gg);
            } else { /* PoissonRegression, MS.h:1509-1543 */
                if (ind) {
                    if (weighted) {
                        double v = wt * n1;
                        g += v;
                        h += v;
                    } else {
                        g += n1;
                        h += n1;
                    }
                } else {
                    g += weighted ? wt * n1 : n1;
                    h += weighted ? wt * n2 : n2;
                }
            }
        }
    } else { /* grouped, MS.hpp:1101-1179 */
        int64_t len = col_len(o, j);
        double n1 = 0.0, n2 = 0.0;
        int key = o->hpid[col_row(o, j, 0)];
        for (int64_t p = 0; p < len; ++p) {
            int64_t i = col_row(o, j, p);
            double x = col_val(o, j, p);
            n1 += o->e[i] * x;
            n2 += ind ? 0.0 : o->e[i] * x * x;
            if (p + 1 < len) {
                int nextKey = o->hpid[col_row(o, j, p + 1)];
                if (key != nextKey) {
                    inc_nevents(ind, &g, &h, n1, n2, o->denom[key], o->nw[key]);
                    n1 = 0.0;
                    n2 = 0.0;
                    key = nextKey;
                }
            }
        }
        inc_nevents(ind, &g, &h, n1, n2, o->denom[key], o->nw[key]);
    }
    g -= o->xjy[j]; /* precomputeGradient */
    *og = g;
    *oh = h;
}

/* updateXBeta(+Impl), MS.hpp:1466-1586 */
static void update_xbeta_ms(Orc* o, int j, double delta) {
    int64_t n = col_len(o, j);
    for (int64_t p = 0; p < n; ++p) {
        int64_t k = col_row(o, j, p);
        o->xb[k] += delta * col_val(o, j, p);
        int g = group_of(o, k);
        if (is_cox(o)) {
            double oldE = o->w ? o->kw[k] * o->e[k] : o->e[k];
            o->e[k] = orc_exp(o->xb[k]);
            double newE = o->w ? o->kw[k] * o->e[k] : o->e[k];
            o->denom[g] += (newE - oldE);
        } else {
            double oldE = o->e[k];
            double newE = o->e[k] = orc_exp(o->xb[k]);
            o->denom[g] += (newE - oldE);
        }
    }
    acc_denominator(o);
}

/* JointPrior getDelta: NoPrior CP.h:186-188, Laplace CP.h:240-273, Normal CP.h:410-415 */
static double prior_delta(const Orc* o, int j, double g, double h) {
    double beta = o->beta[j];
    if (o->prior_type[j] == 1) {
        double lambda = sqrt(2.0 / o->prior_var[j]);
        double delta = 0.0;
        double neg = -(g - lambda) / h;
        double pos = -(g + lambda) / h;
        int s = sgn(beta);
        if (s == 0) {
            if (neg < 0) delta = neg;
            else if (pos > 0) delta = pos;
            else delta = 0;
        } else {
            delta = (s < 0) ? neg : pos;
            if (sgn(beta + delta) != s) delta = -beta;
        }
        return delta;
    } else if (o->prior_type[j] == 2) {
        double v = o->prior_var[j];
        return -(g + (beta / v)) / (h + (1.0 / v));
    }
    return -(g / h);
}

/* ccdUpdateBeta, CCD.cpp:1394-1413 */
static double ccd_update_beta(Orc* o, int j) {
    double g, h;
    numerator_for_gradient(o, j);
    gradient_hessian(o, j, &g, &h);
    if (h < 0.0) {
        g = 0.0;
        h = 0.0;
    }
    return prior_delta(o, j, g, h);
}

/* applyBounds, CCD.cpp:1503-1520 */
static double apply_bounds(Orc* o, double delta, int j) {
    if (delta < -o->hdelta[j]) delta = -o->hdelta[j];
    else if (delta > o->hdelta[j]) delta = o->hdelta[j];
    double inter = dmax(fabs(delta) * 2, o->hdelta[j] / 2);
    inter = dmax(inter, 1E-3);
    o->hdelta[j] = inter;
    return delta;
}

/* getObjectiveFunction, CCD.cpp:541-558 */
static double objective(Orc* o, int conv) {
    if (conv == C_GRADIENT) return gradient_objective(o);
    if (conv == C_MITTAL) return log_likelihood(o);
    return log_likelihood(o) + log_prior(o);
}

/* findMode, CCD.cpp:909-1024 (CCD algorithm, no QN) + performCheckConvergence :839-906 */
static void find_mode(Orc* o, int max_iter, int conv, double eps) {
    if (!o->valid_weights || o->touched_y) {
        set_weights_ms(o);
        fixed_ll(o);
        compute_xjy(o);
        o->valid_weights = 1;
        o->touched_y = 0;
    }
    if (!o->xb_known) {
        compute_xbeta(o);
        o->xb_known = 1;
        o->suff_known = 0;
    }
    if (!o->suff_known) {
        remaining_statistics(o);
        o->suff_known = 1;
    }
    for (int j = 0; j < o->J; ++j) o->hdelta[j] = o->bound; /* resetBounds */
    int iteration = 0, done = 0;
    double last = objective(o, conv);
    while (!done) {
        for (int j = 0; j < o->J; ++j) {
            if (o->fix[j]) continue;
            double delta = ccd_update_beta(o, j);
            delta = apply_bounds(o, delta, j);
            if (delta != 0.0) {
                o->beta[j] += delta;
                update_xbeta_ms(o, j, delta);
            }
        }
        iteration++;
        double cur = objective(o, conv), c;
        int ill = 0;
        if (cur != cur) {
            c = 0.0;
            ill = 1;
        } else {
            c = fabs(cur - last) / (fabs(cur) + 1.0); /* computeConvergenceCriterion :1498-1501 */
        }
        last = cur;
        if (eps > 0 && c < eps) {
            o->last_flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
            done = 1;
        } else if (iteration == max_iter) {
            o->last_flag = R_MAX_ITERATIONS;
            done = 1;
        }
    }
    o->last_iter = iteration;
}

/* computeMMGradientAndHessianImpl, MS.hpp:848-889, with the model's
 * incrementMMGradientAndHessian: Logistic MS.h:570-583 and Survival MS.h:499-516
 * (the same expressions; weight = hNWeight and denominator = denomPid of the
 * row's group).  PoissonRegression's throws (MS.h:1545-1552): returns -1. */
static int mm_gradient_hessian(Orc* o, int j, double* og, double* oh) {
    if (o->model == MT_POISSON) return -1;
    double gradient = 0.0, hessian = 0.0;
    const int ind = col_is_indicator(o, j);
    const int64_t n = col_len(o, j);
    for (int64_t p = 0; p < n; ++p) {
        const int64_t k = col_row(o, j, p);
        const int g = group_of(o, k);
        const double weight = o->nw[g], e = o->e[k], d = o->denom[g];
        if (ind) {
            gradient += weight * e / d;
            hessian += weight * e / d;
        } else {
            const double x = col_val(o, j, p);
            gradient += weight * e * x / d;
            hessian += weight * e * x * x / d;
        }
    }
    gradient -= o->xjy[j]; /* precomputeGradient */
    *og = gradient;
    *oh = hessian;
    return 0;
}

static void find_mode_prepare(Orc* o) {
    if (!o->valid_weights || o->touched_y) {
        set_weights_ms(o);
        fixed_ll(o);
        compute_xjy(o);
        o->valid_weights = 1;
        o->touched_y = 0;
    }
    if (!o->xb_known) {
        compute_xbeta(o);
        o->xb_known = 1;
        o->suff_known = 0;
    }
    if (!o->suff_known) {
        remaining_statistics(o);
        o->suff_known = 1;
    }
    for (int j = 0; j < o->J; ++j) o->hdelta[j] = o->bound; /* resetBounds */
}

/* findMode with AlgorithmType::MM, CCD.cpp:957-1001 and the MM check
 * :1032-1048: every free coordinate's step from one all-coordinate (g, h)
 * (mmUpdateAllBeta, CCD.cpp:1354-1391; no applyBounds), then xBeta from beta
 * (ModelSpecifics::computeXBeta, MS.hpp:313-361) and the remaining
 * statistics.  A log posterior that decreases raises "Non-increasing!"
 * (returned as -1 with the message). */
static int find_mode_mm(Orc* o, int max_iter, int conv, double eps, const char** msg) {
    if (o->model == MT_POISSON) {
        *msg = "Not model-specific";
        return -1;
    }
    if (is_indep(o)) {
        /* initializeMM (MS.hpp:181-257) reduces each column by stratum through
         * ModelData::binaryReductionByStratum (ModelData.h:606-660), which
         * indexes the stratum ids that unstratified data does not have: the
         * reference reads out of bounds there. */
        *msg = "the MM algorithm needs stratified data";
        return -1;
    }
    find_mode_prepare(o);
    int iteration = 0, done = 0;
    double last = objective(o, conv), last_lp = -10E10;
    double* delta = (double*)malloc(sizeof(double) * o->J);
    while (!done) {
        for (int j = 0; j < o->J; ++j) {
            delta[j] = 0.0;
            if (o->fix[j]) continue;
            double g, h;
            if (mm_gradient_hessian(o, j, &g, &h) != 0) {
                free(delta);
                *msg = "Not model-specific";
                return -1;
            }
            if (h < 0.0) {
                g = 0.0;
                h = 0.0;
            }
            delta[j] = prior_delta(o, j, g, h);
        }
        for (int j = 0; j < o->J; ++j)
            if (!o->fix[j] && delta[j] != 0.0) o->beta[j] += delta[j];
        compute_xbeta_mm(o);
        remaining_statistics(o);
        iteration++;
        const double lp = log_likelihood(o) + log_prior(o);
        if (iteration > 1 && lp - last_lp < 0.0) {
            free(delta);
            *msg = "Non-increasing!";
            return -1;
        }
        last_lp = lp;
        double cur = objective(o, conv), c;
        int ill = 0;
        if (cur != cur) {
            c = 0.0;
            ill = 1;
        } else {
            c = fabs(cur - last) / (fabs(cur) + 1.0);
        }
        last = cur;
        if (eps > 0 && c < eps) {
            o->last_flag = ill ? R_ILLCONDITIONED : R_SUCCESS;
            done = 1;
        } else if (iteration == max_iter) {
            o->last_flag = R_MAX_ITERATIONS;
            done = 1;
        }
    }
    o->last_iter = iteration;
    free(delta);
    return 0;
}

static int find_mode_alg(Orc* o, int max_iter, int conv, double eps, int algorithm, const char** msg) {
    if (algorithm == 1) return find_mode_mm(o, max_iter, conv, eps, msg);
    find_mode(o, max_iter, conv, eps);
    return 0;
}

/* One KKT score: |gradient| of column idx at the current state, and whether
 * the column is forced into the active set (computeKktConditions,
 * CCD.cpp:809-826). */
typedef struct {
    int idx;
    double score;
    int force;
} Score;

/* std::list::sort with computeKktConditions' comparator (CCD.cpp:819-825):
 * forced entries first, then decreasing score; a stable merge, as list::sort. */
static void kkt_sort(Score* a, int n) {
    for (int i = 1; i < n; ++i) { /* insertion sort: stable */
        Score t = a[i];
        int j = i - 1;
        while (j >= 0) {
            const int before = (t.force == a[j].force) ? (a[j].score < t.score) : t.force;
            if (!before) break;
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = t;
    }
}

/* CyclicCoordinateDescent::kktSwindle, CCD.cpp:636-807: Laplace columns start
 * inactive at beta = 0 (the intercept and non-Laplace columns are active);
 * findMode over the active set; the inactive columns whose |gradient| exceeds
 * their Laplace lambda (getKktBoundary, CP.h:235-238) move into the active
 * set, largest first, until every inactive column satisfies the condition. */
static int kkt_swindle(Orc* o, int max_iter, int conv, double eps, int algorithm, const char** msg) {
    check_lazy(o);
    const int J = o->J;
    int has_intercept = 0;
    for (int j = 0; j < J; ++j) has_intercept |= (o->fmt[j] == F_INTERCEPT);
    const int intercept = has_intercept ? (o->offset_col0 ? 1 : 0) : -1;
    const size_t cap = (size_t)(J > 0 ? J : 0) + 1;
    uint8_t* exclude = (uint8_t*)malloc(cap);
    Score* active = (Score*)malloc(sizeof(Score) * cap);
    Score* inactive = (Score*)malloc(sizeof(Score) * cap);
    int na = 0, ni = 0;
    for (int j = 0; j < J; ++j) {
        exclude[j] = o->fix[j];
        if (o->fix[j]) continue;
        Score s = {j, 0.0, 0};
        if (j == intercept || o->prior_type[j] != 1) {
            s.force = 1;
            active[na++] = s;
        } else {
            inactive[ni++] = s;
        }
    }
    int done = 0, count = 1, rc = 0;
    while (!done) {
        for (int q = 0; q < ni; ++q) { /* setBeta(i, 0.0): an incremental step of -beta */
            const int i = inactive[q].idx;
            if (o->beta[i] != 0.0) {
                const double delta = 0.0 - o->beta[i];
                o->beta[i] += delta;
                update_xbeta_ms(o, i, delta);
            }
        }
        o->last_flag = R_SUCCESS;
        if (na > 0) { /* findMode(begin(activeSet), end(activeSet)), CCD.cpp:621-634 */
            for (int j = 0; j < J; ++j) o->fix[j] = 1;
            for (int q = 0; q < na; ++q) o->fix[active[q].idx] = 0;
            rc = find_mode_alg(o, max_iter, conv, eps, algorithm, msg);
            if (rc != 0) break;
        }
        if (ni == 0 || o->last_flag != R_SUCCESS) {
            done = 1;
        } else if (count == max_iter) {
            o->last_flag = R_MAX_ITERATIONS;
            done = 1;
        } else {
            for (int q = 0; q < ni; ++q) {
                double g, h;
                numerator_for_gradient(o, inactive[q].idx);
                gradient_hessian(o, inactive[q].idx, &g, &h);
                inactive[q].score = fabs(g);
            }
            kkt_sort(inactive, ni);
            int satisfied = 1;
            for (int q = 0; q < ni; ++q)
                if (!(inactive[q].score <= sqrt(2.0 / o->prior_var[inactive[q].idx]))) satisfied = 0;
            if (satisfied) {
                done = 1;
            } else {
                int moved = 0;
                while (moved < ni &&
                       !(inactive[moved].score <= sqrt(2.0 / o->prior_var[inactive[moved].idx]))) {
                    active[na++] = inactive[moved];
                    ++moved;
                }
                memmove(inactive, inactive + moved, sizeof(Score) * (ni - moved));
                ni -= moved;
            }
        }
        ++count;
    }
    for (int j = 0; j < J; ++j) o->fix[j] = exclude[j]; /* restore fixBeta */
    free(exclude);
    free(active);
    free(inactive);
    return rc;
}

static void set_err(char* err, int errlen, const char* msg) {
    if (err && errlen > 0) {
        strncpy(err, msg, errlen - 1);
        err[errlen - 1] = 0;
    }
}

void* orc_create(int model_type, int fp32_unused, int64_t K, int J, const double* y,
                 const double* time, const int64_t* stratum, const int64_t* col_start,
                 const int32_t* rows, const int64_t* val_start, const double* vals,
                 const uint8_t* fmt, int offset_col0, const int32_t* prior_type,
                 const double* prior_var, char* err, int errlen) {
    (void)fp32_unused;
    if (model_type != MT_LOGISTIC && model_type != MT_POISSON && model_type != MT_CLR &&
        model_type != MT_CPR && model_type != MT_COX) {
        set_err(err, errlen, "unsupported model type");
        return NULL;
    }
    if ((model_type == MT_CLR || model_type == MT_CPR) && !stratum) {
        set_err(err, errlen, "conditional models require stratum ids");
        return NULL;
    }
    if (model_type == MT_COX && !time) {
        set_err(err, errlen, "Cox requires event times");
        return NULL;
    }
    Orc* o = (Orc*)calloc(1, sizeof(Orc));
    o->model = model_type;
    o->K = K;
    o->J = J;
    o->y = (double*)malloc(sizeof(double) * K);
    memcpy(o->y, y, sizeof(double) * K);
    o->offs = (double*)calloc(K, sizeof(double));
    if (time) memcpy(o->offs, time, sizeof(double) * K);
    /* loadY: contiguous patient index per stratum change (ModelData.cpp:96-125) */
    o->Npatients = (int)K;
    if (stratum) {
        o->pid0 = (int32_t*)malloc(sizeof(int32_t) * K);
        int p = 0;
        for (int64_t k = 0; k < K; ++k) {
            if (k > 0 && stratum[k] != stratum[k - 1]) p++;
            o->pid0[k] = p;
        }
        o->Npatients = K > 0 ? p + 1 : 0;
    }
    o->col_start = (int64_t*)malloc(sizeof(int64_t) * (J + 1));
    o->val_start = (int64_t*)malloc(sizeof(int64_t) * (J + 1));
    memcpy(o->col_start, col_start, sizeof(int64_t) * (J + 1));
    memcpy(o->val_start, val_start, sizeof(int64_t) * (J + 1));
    int64_t nr = col_start[J], nv = val_start[J];
    o->rows = (int32_t*)malloc(sizeof(int32_t) * (nr > 0 ? nr : 1));
    if (nr) memcpy(o->rows, rows, sizeof(int32_t) * nr);
    o->vals = (double*)malloc(sizeof(double) * (nv > 0 ? nv : 1));
    if (nv) memcpy(o->vals, vals, sizeof(double) * nv);
    o->fmt = (uint8_t*)malloc(J);
    memcpy(o->fmt, fmt, J);
    o->offset_col0 = offset_col0;
    o->prior_type = (int32_t*)malloc(sizeof(int32_t) * J);
    o->prior_var = (double*)malloc(sizeof(double) * J);
    memcpy(o->prior_type, prior_type, sizeof(int32_t) * J);
    memcpy(o->prior_var, prior_var, sizeof(double) * J);

    size_t cap = (size_t)(K > o->Npatients ? K : o->Npatients) + 2;
    o->kw = (double*)calloc(K, sizeof(double));
    o->nw = (double*)calloc(cap, sizeof(double));
    o->xb = (double*)calloc(K, sizeof(double));
    o->e = (double*)calloc(K, sizeof(double));
    o->denom = (double*)calloc(cap, sizeof(double));
    o->numer = (double*)calloc(cap, sizeof(double));
    o->numer2 = (double*)calloc(cap, sizeof(double));
    o->acc = (double*)calloc(cap, sizeof(double));
    o->hpid = (int32_t*)calloc(K, sizeof(int32_t));
    o->acc_reset = (int32_t*)calloc(cap, sizeof(int32_t));
    o->sidx = (int32_t**)calloc(J, sizeof(int32_t*));
    o->sidx_n = (int*)calloc(J, sizeof(int));
    o->xjy = (double*)calloc(J, sizeof(double));
    o->beta = (double*)calloc(J, sizeof(double));
    o->hdelta = (double*)calloc(J, sizeof(double));
    o->fix = (uint8_t*)calloc(J, 1);
    o->bound = 2.0;
    /* CyclicCoordinateDescent::init, CCD.cpp:200-239 */
    for (int j = 0; j < J; ++j) o->hdelta[j] = o->bound;
    o->N = o->Npatients;
    if (is_grouped(o))
        for (int64_t k = 0; k < K; ++k) o->hpid[k] = o->pid0[k];
    if (offset_col0) {
        o->beta[0] = 1.0;
        o->fix[0] = 1;
        o->xb_known = 0;
    } else {
        o->xb_known = 1;
    }
    /* ModelSpecifics::initialize, MS.hpp:1899-1952: Cox regroups with no weights */
    if (is_cox(o)) set_pid_for_accumulation(o, NULL);
    o->touched_y = 1;
    return o;
}

void orc_destroy(void* hp) {
    Orc* o = (Orc*)hp;
    if (!o) return;
    for (int j = 0; j < o->J; ++j) free(o->sidx[j]);
    free(o->sidx);
    free(o->sidx_n);
    free(o->y);
    free(o->offs);
    free(o->pid0);
    free(o->col_start);
    free(o->val_start);
    free(o->rows);
    free(o->vals);
    free(o->fmt);
    free(o->prior_type);
    free(o->prior_var);
    free(o->kw);
    free(o->nw);
    free(o->xb);
    free(o->e);
    free(o->denom);
    free(o->numer);
    free(o->numer2);
    free(o->acc);
    free(o->hpid);
    free(o->acc_reset);
    free(o->xjy);
    free(o->beta);
    free(o->hdelta);
    free(o->fix);
    free(o->w);
    free(o);
}

/* CyclicCoordinateDescent::setWeights, CCD.cpp:496-519 */
int orc_set_weights(void* hp, const double* w) {
    Orc* o = (Orc*)hp;
    free(o->w);
    o->w = NULL;
    if (w) {
        o->w = (double*)malloc(sizeof(double) * o->K);
        memcpy(o->w, w, sizeof(double) * o->K);
    }
    o->valid_weights = 0;
    o->suff_known = 0;
    return 0;
}

int orc_set_beta(void* hp, const double* beta) { /* CCD.cpp:700-708 */
    Orc* o = (Orc*)hp;
    memcpy(o->beta, beta, sizeof(double) * o->J);
    o->xb_known = 0;
    o->suff_known = 0;
    return 0;
}

/* CyclicCoordinateDescent::update, CCD.cpp:586-615 (resetBeta :256-264) */
int orc_fit(void* hp, int conv_type, double tol, int max_iter, double initial_bound,
            int max_bound_count, int algorithm, int use_kkt, const uint8_t* fixed, double* beta_out,
            double* ll_out, int* iters_out, int* flag_out, char* err, int errlen) {
    Orc* o = (Orc*)hp;
    if (conv_type < C_GRADIENT || conv_type > C_MITTAL) {
        set_err(err, errlen, "unsupported convergence type");
        return -1;
    }
    if (fixed) /* setFixedBeta per column; the offset stays fixed (CCD.cpp:218-221) */
        for (int j = 0; j < o->J; ++j) o->fix[j] = (fixed[j] != 0) || (o->offset_col0 && j == 0);
    o->bound = initial_bound;
    int count = 0;
    o->n_attempts = 0;
    for (;;) {
        const char* msg = NULL;
        /* update: kktSwindle when asked and a Laplace prior supports it (CCD.cpp:598-603) */
        int any_laplace = 0;
        for (int j = 0; j < o->J; ++j) any_laplace |= (o->prior_type[j] == 1);
        const int rc = (use_kkt && any_laplace) ? kkt_swindle(o, max_iter, conv_type, tol, algorithm, &msg)
                                                : find_mode_alg(o, max_iter, conv_type, tol, algorithm, &msg);
        if (rc != 0) {
            set_err(err, errlen, msg ? msg : "mode finding failed");
            return -1;
        }
        ++count;
        if (o->n_attempts < ORC_MAX_ATTEMPTS) o->attempt_sweeps[o->n_attempts++] = o->last_iter;
        if (o->last_flag == R_ILLCONDITIONED && count < max_bound_count) {
            o->bound /= 10.0;
            for (int j = o->offset_col0 ? 1 : 0; j < o->J; ++j) o->beta[j] = 0.0;
            compute_xbeta(o);
            o->suff_known = 0;
        } else {
            break;
        }
    }
    memcpy(beta_out, o->beta, sizeof(double) * o->J);
    check_lazy(o);
    *ll_out = log_likelihood(o);
    *iters_out = o->last_iter;
    *flag_out = o->last_flag;
    return 0;
}

int orc_fit_attempts(void* hp, int* sweeps, int max_n) {
    const Orc* o = (const Orc*)hp;
    for (int i = 0; i < o->n_attempts && i < max_n; ++i) sweeps[i] = o->attempt_sweeps[i];
    return o->n_attempts;
}

int orc_grad_hess(void* hp, int j, double* g, double* h) {
    Orc* o = (Orc*)hp;
    check_lazy(o);
    numerator_for_gradient(o, j);
    gradient_hessian(o, j, g, h);
    return 0;
}

/* beta[j] += delta through CyclicCoordinateDescent::setBeta(int, double)
 * (CyclicCoordinateDescent.cpp:719-733), which re-derives the step as
 * (beta + delta) - beta before updateXBeta. */
int orc_update_beta(void* hp, int j, double delta) {
    Orc* o = (Orc*)hp;
    check_lazy(o);
    const double target = o->beta[j] + delta;
    const double applied = target - o->beta[j];
    o->beta[j] += applied;
    update_xbeta_ms(o, j, applied);
    return 0;
}

int orc_loglik(void* hp, double* ll) {
    Orc* o = (Orc*)hp;
    check_lazy(o);
    *ll = log_likelihood(o);
    return 0;
}

int orc_log_prior(void* hp, double* lp) {
    *lp = log_prior((Orc*)hp);
    return 0;
}

int orc_get_beta(void* hp, double* out) {
    Orc* o = (Orc*)hp;
    memcpy(out, o->beta, sizeof(double) * o->J);
    return 0;
}

int orc_get_xbeta(void* hp, double* out) {
    Orc* o = (Orc*)hp;
    check_lazy(o);
    memcpy(out, o->xb, sizeof(double) * o->K);
    return (int)o->K;
}

/* getNewPredictiveLogLikelihood, CCD.cpp:319-355 -> getPredictiveLogLikelihood MS.hpp:652-690 */
int orc_predictive_loglik(void* hp, const double* w, double* out) {
    Orc* o = (Orc*)hp;
    check_lazy(o);
    compute_xbeta(o);
    remaining_statistics(o);
    double* save = NULL;
    if (is_cox(o)) {
        save = (double*)malloc(sizeof(double) * o->K);
        memcpy(save, o->kw, sizeof(double) * o->K);
        double* keep = o->w;
        o->w = (double*)w;
        set_weights_ms(o);
        remaining_statistics(o);
        o->w = keep;
    }
    double ll = 0.0;
    for (int64_t k = 0; k < o->K; ++k) {
        double yk = o->y[k], wk = w[k], xbk = o->xb[k];
        switch (o->model) {
        case MT_LOGISTIC:
            ll += yk * wk * (xbk - log(o->denom[k]));
            break;
        case MT_POISSON:
            ll += (yk * xbk - orc_exp(xbk)) * wk;
            break;
        case MT_CLR:
        case MT_CPR:
            ll += yk * wk * (xbk - log(o->denom[o->hpid[k]]));
            break;
        default: /* COX */
            ll += wk == 0.0 ? 0.0 : yk * wk * (xbk - log(o->acc[o->hpid[k]]));
        }
    }
    if (is_cox(o)) {
        double* keep = o->w;
        o->w = save;
        set_weights_ms(o);
        remaining_statistics(o);
        o->w = keep;
        free(save);
    }
    o->suff_known = 1;
    *out = ll;
    return 0;
}

/* incrementFisherInformation of the model (weight = hKWeight = 1: the unweighted
 * fits computeFisherInformation accepts, MS.hpp:434-440):
 *   Logistic MS.h:521-535   weight * (p/d - (p/d)^2) * x1x2
 *   Poisson  MS.h:1497-1506 weight * p * x1x2
 *   Survival MS.h:485-498   weight * p / d * x1x2   (CLR, CPR, Breslow Cox)
 * d is denomPid of the row's group (its own slot for independent rows). */
static double fisher_increment(const Orc* o, int64_t k, double x12) {
    const double weight = 1.0, p = o->e[k];
    switch (o->model) {
    case MT_LOGISTIC: {
        const double d = o->denom[k];
        const double g = p / d;
        return weight * (p / d - g * g) * x12;
    }
    case MT_POISSON:
        return weight * p * x12;
    default:
        return weight * p / o->denom[o->hpid[k]] * x12;
    }
}

/* getSubjectSpecificHessianIterator, MS.hpp:1245-1266: walk the column in row
 * order, one (hPid, sum of e*x) pair per run of rows sharing hPid. */
static int fisher_cross_terms(const Orc* o, int j, int32_t* gid, double* val) {
    const int64_t len = col_len(o, j);
    int n = 0;
    int64_t p = 0;
    while (p < len) {
        double v = 0.0;
        const int g = o->hpid[col_row(o, j, p)];
        do {
            const int64_t k = col_row(o, j, p);
            v += o->e[k] * col_val(o, j, p); /* gradientNumeratorContrib, MS.h:437-441 */
            ++p;
        } while (p < len && o->hpid[col_row(o, j, p)] == g);
        gid[n] = g;
        val[n] = v;
        ++n;
    }
    return n;
}

/* computeFisherInformationImpl, MS.hpp:1268-1337: the pair-product walk over
 * the rows both columns hold (PairProductIterator, Iterators.h:627-680), minus
 * the strata cross terms for GroupedData / OrderedWithTiesData models. */
static double fisher_pair(const Orc* o, int i, int j, int32_t* g1, double* v1, int32_t* g2, double* v2) {
    double information = 0.0;
    const int64_t n1 = col_len(o, i), n2 = col_len(o, j);
    int64_t p = 0, q = 0;
    while (p < n1 && q < n2) {
        const int64_t a = col_row(o, i, p), b = col_row(o, j, q);
        if (a < b) {
            ++p;
        } else if (b < a) {
            ++q;
        } else {
            information += fisher_increment(o, a, col_val(o, i, p) * col_val(o, j, q));
            ++p;
            ++q;
        }
    }
    if (!is_indep(o)) { /* hasStrataCrossTerms */
        const int m1 = fisher_cross_terms(o, i, g1, v1), m2 = fisher_cross_terms(o, j, g2, v2);
        double cross = 0.0;
        int r = 0, s = 0;
        while (r < m1 && s < m2) {
            if (g1[r] < g2[s]) {
                ++r;
            } else if (g2[s] < g1[r]) {
                ++s;
            } else {
                const double d = o->denom[g1[r]];
                cross += v1[r] * v2[s] / (d * d);
                ++r;
                ++s;
            }
        }
        information -= cross;
    }
    return information;
}

/* CyclicCoordinateDescent::computeFisherInformation(indices), CCD.cpp:1288-1299
 * -> ModelSpecifics::computeFisherInformation, MS.hpp:1203-1225.  `out` is
 * n x n, row-major, symmetric.  Weighted (cross-validation) fits are refused
 * as the reference refuses them (MS.hpp:1207-1208): returns -2. */
int orc_fisher_information(void* hp, const int32_t* idx, int n, double* out) {
    Orc* o = (Orc*)hp;
    if (o->w) return -2;
    check_lazy(o);
    const size_t cap = (size_t)o->K + 1;
    int32_t *g1 = (int32_t*)malloc(sizeof(int32_t) * cap), *g2 = (int32_t*)malloc(sizeof(int32_t) * cap);
    double *v1 = (double*)malloc(sizeof(double) * cap), *v2 = (double*)malloc(sizeof(double) * cap);
    for (int ii = 0; ii < n; ++ii)
        for (int jj = ii; jj < n; ++jj) {
            const double e = fisher_pair(o, idx[ii], idx[jj], g1, v1, g2, v2);
            out[(size_t)ii * n + jj] = e;
            out[(size_t)jj * n + ii] = e;
        }
    free(g1);
    free(g2);
    free(v1);
    free(v2);
    return 0;
}

/* getPredictiveEstimates, MS.hpp:692-705, with predictEstimate of the model:
 * LR exp(xb)/(exp(xb)+1) (MS.h:1011-1014), Poisson exp(xb) (MS.h:1592-1594),
 * the conditional and Cox models xb.  Rows with a zero weight keep y. */
int orc_predictive_estimates(void* hp, const double* w, double* y) {
    Orc* o = (Orc*)hp;
    check_lazy(o);
    for (int64_t k = 0; k < o->K; ++k) {
        if (w && !w[k]) continue;
        const double xb = o->xb[k];
        if (o->model == MT_LOGISTIC) {
            const double t = orc_exp(xb);
            y[k] = t / (t + 1.0);
        } else if (o->model == MT_POISSON) {
            y[k] = orc_exp(xb);
        } else {
            y[k] = xb;
        }
    }
    return 0;
}

int orc_num_patients(void* hp) { return ((Orc*)hp)->Npatients; }

int orc_cox_groups(void* hp, int32_t* group_out, int32_t* acc_reset_out, int* n_reset_out) {
    Orc* o = (Orc*)hp;
    if (!is_cox(o)) return -1;
    check_lazy(o);
    memcpy(group_out, o->hpid, sizeof(int32_t) * o->K);
    memcpy(acc_reset_out, o->acc_reset, sizeof(int32_t) * o->n_reset);
    *n_reset_out = o->n_reset;
    return o->N;
}
