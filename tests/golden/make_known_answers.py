"""Known-answer fixtures from the reference's own R tests, read as text.

    make -C oracle ref && python tests/golden/make_known_answers.py

The reference's testthat files compare Cyclops with glm / coxph / clogit on
small inline data sets.  R is not available here, so this script reads those
data sets out of the test sources (and the CLR test's infert data from the
reference's fixture file), builds the same design matrices, and records what
the reference Cyclops engine (compiled from source) returns for them:
coefficients, log-likelihood, the Fisher information at the mode and the
predictions.  The tests check the oracle and the GPU against these fixtures,
and the fixtures against an independent Newton solve of the same likelihood
(the stand-in for the R gold packages).  Run only where the reference sources
are present; the fixtures are committed.

Data sources (paths within the reference project):
  tests/testthat/test-smallBernoulli.R  binomial_bid / binomial_n / binomial_y
  tests/testthat/test-smallPoisson.R    dobson: counts, outcome = gl(3,1,9), treatment = gl(3,3)
  tests/testthat/test-smallCox.R        the inline `read.table(text = ...)` tables
  tests/testthat/test-weighting.R       weighted Bernoulli / Poisson / Cox fits, zero
                                        weights against the subset fit, the Cox
                                        predictive log-likelihood on held-out rows
  inst/extdata/infert_ccd.txt           case ~ spontaneous + induced + strata(stratum)
  inst/extdata/CCD_LOGISTIC_TEST_17var.txt with the SAS fit's 2 x log-likelihood that
                                        tests/testthat/test-largeBernoulli.R quotes
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ccd_b200.data import (DENSE, GRADIENT, INDICATOR, INTERCEPT, MODEL_CONDITIONAL_LOGISTIC,  # noqa: E402
                           MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_NONE, SPARSE, CyclopsData,
                           build_columns, cox_sort_order)
from oracle.checker import ReferenceEngine  # noqa: E402

REF = os.environ.get("CYCLOPS_REFERENCE",
                     os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "..", "reference"))
TESTS = os.path.join(REF, "tests", "testthat")


def r_vector(src: str, name: str) -> np.ndarray:
    """The first `name <- c(...)` or `name = c(...)` numeric vector in R source."""
    m = re.search(name + r"\s*(?:<-|=)\s*c\(([^)]*)\)", src)
    return np.array([float(x) for x in m.group(1).split(",")])


def r_gl(src: str, name: str) -> np.ndarray:
    """`name = gl(n, k[, length])`: levels 1..n, each repeated k times, cycled."""
    m = re.search(name + r"\s*(?:<-|=)\s*gl\((\d+)\s*,\s*(\d+)(?:\s*,\s*(\d+))?\)", src)
    n, k = int(m.group(1)), int(m.group(2))
    length = int(m.group(3)) if m.group(3) else n * k
    base = np.repeat(np.arange(1, n + 1), k)
    return np.resize(base, length)


def r_blocks(src: str):
    """The bodies of the `test_that(...)` blocks, in order."""
    return re.split(r"\ntest_that\(", src)[1:]


def r_tables(src: str):
    """Every inline `read.table(header=T, sep = ",", text = "...")` table."""
    out = []
    for body in re.findall(r'read\.table\(header\s*=\s*T,\s*sep\s*=\s*",",\s*text\s*=\s*"(.*?)"\)', src, re.S):
        lines = [ln.strip() for ln in body.strip().splitlines() if ln.strip()]
        head = [h.strip() for h in lines[0].split(",")]
        rows = np.array([[float(v) for v in ln.split(",")] for ln in lines[1:]])
        out.append({h: rows[:, i] for i, h in enumerate(head)})
    return out


def dense_data(model, y, cols, fmts, stratum=None, time=None) -> CyclopsData:
    """CyclopsData from dense covariate vectors; SPARSE / INDICATOR columns keep
    their nonzero rows."""
    K = len(y)
    built = []
    for x, f in zip(cols, fmts):
        if f == INTERCEPT:
            built.append((None, None))
        elif f == DENSE:
            built.append((None, np.asarray(x, np.float64)))
        else:
            r = np.nonzero(np.asarray(x) != 0)[0].astype(np.int32)
            built.append((r, None if f == INDICATOR else np.asarray(x, np.float64)[r]))
    cs, rows, vs, vals, fmt = build_columns(K, built, fmts)
    J = len(fmts)
    return CyclopsData(model, np.asarray(y, np.float64), cs, rows, vs, vals, fmt,
                       np.full(J, PRIOR_NONE, np.int32), np.ones(J),
                       time=None if time is None else np.asarray(time, np.float64),
                       stratum=None if stratum is None else np.asarray(stratum, np.int64))


def bernoulli_xy():
    src = open(os.path.join(TESTS, "test-smallBernoulli.R")).read()
    bid, n, yy = (r_vector(src, "binomial_bid"), r_vector(src, "binomial_n"), r_vector(src, "binomial_y"))
    # log(c(rep(bid, n - y), rep(bid, y))) and y = c(rep(0, sum(n - y)), rep(1, sum(y)))
    log_bid = np.log(np.concatenate([np.repeat(bid, (n - yy).astype(int)), np.repeat(bid, yy.astype(int))]))
    y = np.concatenate([np.zeros(int(np.sum(n - yy))), np.ones(int(np.sum(yy)))])
    return log_bid, y


def bernoulli(fmt, rows=None):
    log_bid, y = bernoulli_xy()
    if rows is not None:
        log_bid, y = log_bid[rows], y[rows]
    return dense_data(MODEL_LOGISTIC, y, [None, log_bid], [INTERCEPT, fmt])


def gl_weights(n_levels: int, length: int) -> np.ndarray:
    """as.numeric(gl(n, 1, length)): 1..n cycled."""
    return np.resize(np.arange(1, n_levels + 1, dtype=np.float64), length)


def dobson(fmt):
    src = open(os.path.join(TESTS, "test-smallPoisson.R")).read()
    counts = r_vector(src, "counts")
    outcome, treatment = r_gl(src, "outcome"), r_gl(src, "treatment")
    # treatment contrasts: intercept, outcome2, outcome3, treatment2, treatment3
    cols = [None] + [(outcome == lv).astype(float) for lv in (2, 3)] + [(treatment == lv).astype(float) for lv in (2, 3)]
    return dense_data(MODEL_POISSON, counts, cols, [INTERCEPT] + [fmt] * 4)


def cox_tables():
    src = open(os.path.join(TESTS, "test-smallCox.R")).read()
    return r_tables(src)[:4]


def cox(table, strata_x2=False):
    """Surv(length, event) ~ x1 + x2, or ~ x1 + strata(x2); rows in the order the
    R layer gives the engine (stratum, -time, event)."""
    t, ev = table["length"], table["event"]
    stratum = table["x2"].astype(np.int64) if strata_x2 else np.zeros(len(t), np.int64)
    order = cox_sort_order(stratum, t, ev)
    cols = [table["x1"][order]] + ([] if strata_x2 else [table["x2"][order]])
    return dense_data(MODEL_COX, ev[order], cols, [DENSE] * len(cols), stratum=stratum[order], time=t[order])


def weighting_tests():
    """test-weighting.R: its inline tables and weight vectors, by test block."""
    src = open(os.path.join(TESTS, "test-weighting.R")).read()
    blocks = r_blocks(src)
    out = []
    for b in blocks:
        tabs = r_tables(b)
        m = re.search(r"\n\s*weights\s*<-\s*c\(([^)]*)\)", b)
        w = np.array([float(x) for x in m.group(1).split(",")]) if m else None
        out.append((tabs[0] if tabs else None, w))
    return out


def cox_w(table, weights=None, strata_x2=False, fmts=(DENSE, DENSE)):
    """A test-weighting.R Cox table (event column `status` or `event`)."""
    t = table["length"]
    ev = table["status"] if "status" in table else table["event"]
    stratum = table["x2"].astype(np.int64) if strata_x2 else np.zeros(len(t), np.int64)
    order = cox_sort_order(stratum, t, ev)
    cols = [table["x1"][order]] + ([] if strata_x2 else [table["x2"][order]])
    d = dense_data(MODEL_COX, ev[order], cols, list(fmts[:len(cols)]), stratum=stratum[order], time=t[order])
    return d, None if weights is None else np.asarray(weights, np.float64)[order]


def rows_of(table, idx):
    return {k: v[idx] for k, v in table.items()}


def infert():
    """inst/extdata/infert_ccd.txt: `stratum y covariate:value ...` per row."""
    rows = []
    with open(os.path.join(REF, "inst", "extdata", "infert_ccd.txt")) as fh:
        for line in fh:
            if line.startswith("#") or not line.strip():
                continue
            parts = line.split()
            x = {int(k): float(v) for k, v in (p.split(":") for p in parts[2:])}
            rows.append((int(parts[0]), float(parts[1]), x.get(1, 0.0), x.get(2, 0.0)))
    a = np.array(rows)
    order = np.argsort(a[:, 0], kind="stable")
    a = a[order]
    return dense_data(MODEL_CONDITIONAL_LOGISTIC, a[:, 1], [a[:, 2], a[:, 3]], [DENSE, DENSE],
                      stratum=a[:, 0].astype(np.int64))


def large_bernoulli():
    """CCD_LOGISTIC_TEST_17var.txt (`row_label y covariate:value ...`, intercept
    added), and the published 2 x log-likelihood of its SAS fit quoted in
    test-largeBernoulli.R."""
    rows, ids = [], set()
    with open(os.path.join(REF, "inst", "extdata", "CCD_LOGISTIC_TEST_17var.txt")) as fh:
        for line in fh:
            if line.startswith("#") or not line.strip():
                continue
            parts = line.split()
            x = {int(k): float(v) for k, v in (p.split(":") for p in parts[2:])}
            ids |= set(x)
            rows.append((float(parts[1]), x))
    ids = sorted(ids)
    y = np.array([a for a, _ in rows])
    cols = [None] + [np.array([x.get(c, 0.0) for _, x in rows]) for c in ids]
    src = open(os.path.join(TESTS, "test-largeBernoulli.R")).read()
    published = float(re.search(r"log_likelihood\s*\*\s*2\s*,\s*(-?[0-9.]+)", src).group(1))
    return dense_data(MODEL_LOGISTIC, y, cols, [INTERCEPT] + [SPARSE] * len(ids)), published


def problems():
    """name -> (data, fixed flags or None, weights or None, held-out weights or None)."""
    out = {
        "bernoulli_dense": (bernoulli(DENSE), None, None, None),
        "bernoulli_sparse": (bernoulli(SPARSE), None, None, None),
        "dobson_dense": (dobson(DENSE), None, None, None),
        "dobson_indicator": (dobson(INDICATOR), None, None, None),
        "dobson_fixed": (dobson(DENSE), np.array([0, 1, 0, 1, 0], np.uint8), None, None),
        "infert_clr": (infert(), None, None, None),
        "bernoulli_17var": (large_bernoulli()[0], None, None, None),
    }
    for i, name in enumerate(("cox_no_ties", "cox_time_ties", "cox_failure_ties", "cox_failure_ties_after")):
        out[name] = (cox(cox_tables()[i]), None, None, None)
    out["cox_strata"] = (cox(cox_tables()[0], strata_x2=True), None, None, None)
    # test-weighting.R
    src = open(os.path.join(TESTS, "test-weighting.R")).read()
    wsrc = re.search(r"weights\s*<-\s*c\((1,2,1,2,4,3,2,1,1)\)", src)
    K = len(bernoulli_xy()[1])
    out["bernoulli_weighted"] = (bernoulli(DENSE), None, gl_weights(5, K), None)
    zero = gl_weights(2, K) - 1.0
    out["bernoulli_zero_weights"] = (bernoulli(DENSE), None, zero, None)
    out["bernoulli_subset"] = (bernoulli(DENSE, rows=np.nonzero(zero == 1.0)[0]), None, None, None)
    out["dobson_weighted"] = (dobson(DENSE), None, np.array([float(x) for x in wsrc.group(1).split(",")]), None)
    wt = weighting_tests()
    d, w = cox_w(wt[0][0])
    out["coxw_ties"] = (d, None, None, None)
    d, w = cox_w(wt[1][0], wt[1][1])
    out["coxw_no_ties_weighted"] = (d, None, w, None)
    d, w = cox_w(wt[2][0], wt[2][1])
    out["coxw_ties_weighted"] = (d, None, w, None)
    # doubled rows (each row twice, consecutively), the second copy fitted, the
    # first held out: the held-out predictive LL is the stratified fit's LL
    tab = wt[3][0]
    twice = rows_of(tab, np.repeat(np.arange(len(tab["length"])), 2))
    fitw = np.resize(np.array([0.0, 1.0]), 2 * len(tab["length"]))
    d, w = cox_w(twice, fitw, strata_x2=True)
    out["coxw_predictive"] = (d, None, w, cox_w(twice, 1.0 - fitw, strata_x2=True)[1])
    out["coxw_predictive_gold"] = (cox_w(tab, strata_x2=True)[0], None, None, None)
    # duplicated rows re-weighted to the original fit; then sparse x1 / indicator x2
    tab = wt[4][0]
    dup = rows_of(tab, np.concatenate([np.arange(len(tab["length"])), [0, 2, 3]]))
    d, w = cox_w(dup, wt[4][1])
    out["coxw_duplicated"] = (d, None, w, None)
    d, w = cox_w(dup, wt[4][1], fmts=(SPARSE, INDICATOR))
    out["coxw_duplicated_sparse"] = (d, None, w, None)
    out["coxw_duplicated_gold"] = (cox_w(tab)[0], None, None, None)
    return out


TOL = 1e-12  # on the gradient objective: converged far below the R tests' 1e-4


def main():
    for name, (d, fixed, w, held) in problems().items():
        e = ReferenceEngine(d)
        if w is not None:
            e.set_weights(w)
        r = e.fit(GRADIENT, TOL, max_iter=10_000, fixed=fixed)
        cols = np.array([j for j in range(d.J) if fixed is None or not fixed[j]], np.int32)
        fisher = e.fisher_information(cols) if w is None else None  # refused when weighted
        pred = e.predictive_estimates()
        pred_ll = e.predictive_loglik(held) if held is not None else None
        e.close()
        arrays = dict(model_type=np.int32(d.model_type), y=d.y, col_start=d.col_start, rows=d.rows,
                      val_start=d.val_start, vals=d.vals, fmt=d.fmt, prior_type=d.prior_type,
                      prior_var=d.prior_var, offset_col0=np.int32(0), beta=r["beta"],
                      loglik=np.float64(r["loglik"]), iterations=np.int32(r["iterations"]),
                      flag=np.int32(r["flag"]), fisher_cols=cols, pred_est=pred)
        if fisher is not None:
            arrays["fisher"] = fisher
        if w is not None:
            arrays["weights"] = w
        if held is not None:
            arrays["heldout"] = held
            arrays["pred_ll"] = np.float64(pred_ll)
        if name == "bernoulli_17var":
            arrays["published_2ll"] = np.float64(large_bernoulli()[1])
        if d.time is not None:
            arrays["time"] = d.time
        if d.stratum is not None:
            arrays["stratum"] = d.stratum
        if fixed is not None:
            arrays["fixed"] = fixed
        np.savez_compressed(os.path.join(HERE, "known_" + name + ".npz"), **arrays)
        print(name, d.K, d.J, r["flag"], r["iterations"], np.round(r["beta"], 6), r["loglik"])


if __name__ == "__main__":
    main()
