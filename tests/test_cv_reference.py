"""The cross-validation drivers of ccd_b200/cv.py against the reference's own
drivers compiled from source (AutoSearchCrossValidationDriver,
GridSearchCrossValidationDriver, CrossValidationSelector, UniModalSearch),
run as CcdInterface::runCrossValidation runs them with one thread and cold
starts.  cv.py's host logic is driven here by an evaluator that fits every
(fold, variance) instance with the oracle -- which is bit-exact with the
reference engine -- on the reference selector's own fold map, so the search
path, the selected variance and the refit must agree.  The auto search's
per-step values are compared at the six significant digits the reference
logs them with; the grid's values and the selected variances exactly or to
1e-9."""
import re

import numpy as np
import pytest

from ccd_b200 import cv, native, synthetic
from ccd_b200.data import (GRADIENT, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON,
                           PRIOR_NONE)
from oracle import checker

pytestmark = pytest.mark.skipif(not checker.reference_available(),
                                reason="reference engine not built (no reference sources here)")


class OracleBatch:
    """Stands in for native.Fit.batch_find_mode: instance i fits the rows
    whose fold is not hold[i] at prior variance var[i] (cold start), and
    reports the held-out fold's predictive log-likelihood when it succeeded."""

    def __init__(self, d):
        self.d = d

    def batch_find_mode(self, var, hold, row_fold, args=None):
        args = args or native.ModeFindingArguments()
        res = []
        for v, h in zip(var, hold):
            d = self.d.with_prior(PRIOR_NONE, 1.0)
            d.prior_type = self.d.prior_type.copy()
            d.prior_var = np.where(self.d.prior_type == PRIOR_NONE, self.d.prior_var, float(v))
            w = (np.asarray(row_fold) != h).astype(np.float64)
            e = checker.RestatementEngine(d)
            e.set_weights(w)
            r = e.fit(args.convergence_type, args.tolerance, args.max_iterations)
            pred = e.predictive_loglik(1.0 - w) if r["flag"] == 0 else float("nan")
            res.append({"flag": r["flag"], "pred_loglik": pred})
            e.close()
        return None, res, 0.0

    def fold_instances(self, variances, holdout, row_fold, args=None):
        """native.Fit.fold_instances' contract: per-column variances."""
        args = args or native.ModeFindingArguments()
        res = []
        for v, h in zip(variances, holdout):
            d = self.d.with_prior(PRIOR_NONE, 1.0)
            d.prior_type = self.d.prior_type.copy()
            d.prior_var = np.array(v, dtype=np.float64)
            w = (np.asarray(row_fold) != h).astype(np.float64)
            e = checker.RestatementEngine(d)
            e.set_weights(w)
            r = e.fit(args.convergence_type, args.tolerance, args.max_iterations)
            pred = e.predictive_loglik(1.0 - w) if r["flag"] == 0 else float("nan")
            res.append({"flag": r["flag"], "pred_loglik": pred})
            e.close()
        return None, res, 0.0


def parse_auto_log(text):
    """(variance, mean, stdev) per step from the auto-search driver's log."""
    steps = re.findall(r"AvgPred = (\S+) with stdev = (\S+)\s*\nCompleted at (\S+)", text)
    return [(float(v), float(m), float(s)) for m, s, v in steps]


CASES = [
    (MODEL_LOGISTIC, dict(seed=150, K=400, P=15)),
    (MODEL_POISSON, dict(seed=151, K=300, P=10, offset=True)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=152, n_strata=60, K=360, P=10)),
    (MODEL_COX, dict(seed=153, K=300, P=8, n_strata=3, tie_days=4)),
]


@pytest.mark.parametrize("model,kw", CASES)
def test_auto_search_matches_the_reference_driver(model, kw):
    d = synthetic.small(model, **kw)
    ref = checker.ReferenceEngine(d).cross_validate(auto_search=True, fold=5, seed=123)
    args = native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6)
    got = cv.auto_search(OracleBatch(d), d, ref["row_fold"], 5, args)
    want = parse_auto_log(ref["log"])
    assert len(got.tried) == len(want)
    for (v, m, s), (wv, wm, ws) in zip(got.tried, want):
        assert v == pytest.approx(wv, rel=1e-5)
        assert m == pytest.approx(wm, rel=1e-5)
        assert s == pytest.approx(ws, rel=1e-5, abs=1e-5)
    assert got.variance == pytest.approx(ref["variance"], rel=1e-9)
    # resetForOptimal + fitModel: all rows, the selected variance, cold start
    dv = d.with_prior(PRIOR_NONE, 1.0)
    dv.prior_type = d.prior_type.copy()
    dv.prior_var = np.where(d.prior_type == PRIOR_NONE, d.prior_var, got.variance)
    refit = checker.RestatementEngine(dv).fit(GRADIENT, 1e-6)
    scale = max(1.0, np.max(np.abs(ref["beta"])))
    assert np.max(np.abs(refit["beta"] - ref["beta"])) <= 1e-8 * scale


@pytest.mark.parametrize("model,kw", CASES[:3])
def test_grid_search_matches_the_reference_driver(model, kw):
    d = synthetic.small(model, **kw)
    ref = checker.ReferenceEngine(d).cross_validate(auto_search=False, fold=5, grid_steps=6, lower=0.01,
                                                    upper=10.0, seed=7)
    args = native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6)
    got = cv.grid_search(OracleBatch(d), ref["row_fold"], 5, lower=0.01, upper=10.0, steps=6, args=args)
    assert np.array_equal([t[0] for t in got.tried], ref["points"])
    np.testing.assert_allclose([t[1] for t in got.tried], ref["values"], rtol=1e-13)
    assert got.variance == ref["variance"]


@pytest.mark.parametrize("seed", range(60))
def test_random_problems_match_the_reference_drivers(seed):
    """Seeded random problems (tests/test_oracle_fuzz.py's generator: every
    model, formats and densities, an offset, mixed priors) through a random
    driver: auto search or grid, 3 to 10 folds, the selector's seed.  Mixed
    priors give the joint prior several variance parameters, which the auto
    search tunes in turn and the grid leaves but the first alone."""
    from .test_oracle_fuzz import random_case
    d, _, _ = random_case(seed)
    rng = np.random.default_rng(20_000 + seed)
    fold = int(rng.integers(3, 11))
    cv_seed = int(rng.integers(1, 1000))
    auto = bool(rng.integers(2))
    args = native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6)
    groups = cv.variance_groups(d)
    if not groups:  # the engine's driver would read a variance parameter that does not exist
        with pytest.raises(ValueError, match="flat prior"):
            cv.auto_search(OracleBatch(d), d, np.zeros(d.K, np.int32), fold, args)
        return
    if auto:
        # the selector's fold map first (a grid run of one point gives it cheaply)
        row_fold = checker.ReferenceEngine(d).cross_validate(auto_search=False, fold=fold, grid_steps=1,
                                                             seed=cv_seed)["row_fold"]
        got = cv.auto_search(OracleBatch(d), d, row_fold, fold, args, max_cycles=20)
        if not got.converged:  # the reference's rounds would not end either
            pytest.skip("the auto search's rounds do not settle on this problem")
        ref = checker.ReferenceEngine(d).cross_validate(auto_search=True, fold=fold, seed=cv_seed)
        assert np.array_equal(ref["row_fold"], row_fold)
        want = parse_auto_log(ref["log"])
        assert len(got.tried) == len(want)
        for (v, m, s), (wv, wm, ws) in zip(got.tried, want):
            assert v == pytest.approx(wv, rel=1e-5)
            assert m == pytest.approx(wm, rel=1e-5, nan_ok=True)
            assert s == pytest.approx(ws, rel=1e-5, abs=1e-5, nan_ok=True)
        np.testing.assert_allclose(got.variances, ref["variances"], rtol=1e-9)
    else:
        ref = checker.ReferenceEngine(d).cross_validate(auto_search=False, fold=fold, grid_steps=5, lower=0.05,
                                                        upper=5.0, seed=cv_seed)
        got = cv.grid_search(OracleBatch(d), ref["row_fold"], fold, lower=0.05, upper=5.0, steps=5, args=args)
        assert np.array_equal([t[0] for t in got.tried], ref["points"])
        np.testing.assert_allclose([t[1] for t in got.tried], ref["values"], rtol=1e-13)
        assert got.variance == ref["variance"]
    # the refit: resetForOptimal's variances, all rows, cold start
    dv = d.with_prior(PRIOR_NONE, 1.0)
    dv.prior_type = d.prior_type.copy()
    dv.prior_var = cv.column_variances(d, got.variances)
    refit = checker.RestatementEngine(dv).fit(GRADIENT, 1e-6)
    scale = max(1.0, np.nanmax(np.abs(ref["beta"]), initial=0.0))
    np.testing.assert_allclose(refit["beta"], ref["beta"], rtol=0, atol=1e-8 * scale, equal_nan=True)


@pytest.mark.parametrize("flat", [False, True])
def test_quadratic_fit_is_the_references_bit_for_bit(flat):
    """cv.quadratic_log_fit against the reference's QuadrLogFit compiled from
    source, on random histories: 3 to 60 points, stdevs with zeros, and (flat)
    means equal to 1e-12 -- the badly conditioned end of a search, where the
    proposal is decided by rounding."""
    rng = np.random.default_rng(7 + flat)
    for _ in range(2000):
        n = int(rng.integers(3, 61))
        xs = np.exp(rng.uniform(-10.0, 60.0, n))
        ms = rng.normal(-13.0, 2.0) + (rng.normal(0.0, 1e-12, n) if flat else rng.normal(0.0, 1.0, n))
        sds = np.where(rng.random(n) < 0.1, 0.0, rng.uniform(0.1, 3.0, n))
        h = {float(x): (float(m), float(s)) for x, m, s in zip(xs, ms, sds)}
        assert cv.quadratic_log_fit(h) == checker.ReferenceEngine.quadr_log_fit(h)


def test_variance_parameters_in_the_references_order():
    """cv.variance_groups against the reference's getHyperprior(): a one-point
    grid moves the first variance parameter to the grid's point and leaves the
    others at the prior's values, in registration order."""
    d = synthetic.small(MODEL_LOGISTIC, seed=170, K=300, P=6, prior=PRIOR_NONE)
    d.prior_type[:] = [0, 2, 1, 2, 1, 0, 1]
    d.prior_var[:] = [1.0, 2.0, 1.0, 2.0, 3.0, 1.0, 1.0]
    groups = cv.variance_groups(d)
    assert [g.tolist() for g in groups] == [[1, 3], [2, 6], [4]]
    ref = checker.ReferenceEngine(d).cross_validate(auto_search=False, fold=3, grid_steps=1, lower=0.5,
                                                    upper=0.5, seed=3)
    assert ref["variances"].tolist() == [0.5, 1.0, 3.0]
    np.testing.assert_array_equal(cv.column_variances(d, 0.5), [1.0, 0.5, 1.0, 0.5, 3.0, 1.0, 1.0])
