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
