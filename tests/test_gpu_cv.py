"""Cross-validation drivers on the batched engine against the same drivers
run on oracle fits (one CPU fit per fold and variance, cold start)."""
import numpy as np
import pytest

from ccd_b200 import cv, native, synthetic
from ccd_b200.data import GRADIENT, MODEL_LOGISTIC

pytestmark = pytest.mark.gpu


class OracleBatch:
    """fit.batch_find_mode's contract, one oracle fit per instance."""

    def __init__(self, engine, d):
        self.engine, self.d = engine, d

    def batch_find_mode(self, variance, holdout, row_fold, args=None):
        res = []
        for v, h in zip(variance, holdout):
            e = self.engine(self.d.with_prior(int(self.d.prior_type[-1]), float(v)))
            w = (row_fold != h).astype(float)
            e.set_weights(w)
            r = e.fit(GRADIENT, 1e-6)
            res.append({"flag": r["flag"], "pred_loglik": e.predictive_loglik(1.0 - w)})
        return None, res, 0.0


def _problem():
    d = synthetic.small(MODEL_LOGISTIC, seed=80, K=900, P=25)
    fold = synthetic.cv_folds(d.K, n_folds=5, seed=9)
    return d, fold


def test_auto_search_matches_oracle_driver(gpu_ctx, oracle_engine):
    d, fold = _problem()
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    got = cv.auto_search(f, d, fold, 5)
    want = cv.auto_search(OracleBatch(oracle_engine, d), d, fold, 5)
    assert len(got.tried) == len(want.tried)
    for (v1, m1, _), (v2, m2, _) in zip(got.tried, want.tried):
        assert v1 == pytest.approx(v2, rel=1e-6)
        assert m1 == pytest.approx(m2, rel=1e-8)
    assert got.variance == pytest.approx(want.variance, rel=1e-6)
    # refit at the selected variance on all rows
    r = cv.refit_at(gpu_ctx, m, d, got.variance)
    e = oracle_engine(d.with_prior(int(d.prior_type[-1]), got.variance))
    ref = e.fit(GRADIENT, 1e-6)
    assert np.max(np.abs(r.beta - ref["beta"])) <= 1e-6 * max(np.max(np.abs(ref["beta"])), 1e-8)


def test_grid_search_matches_oracle_driver(gpu_ctx, oracle_engine):
    d, fold = _problem()
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    got = cv.grid_search(f, fold, 5, lower=0.01, upper=10.0, steps=6)
    want = cv.grid_search(OracleBatch(oracle_engine, d), fold, 5, lower=0.01, upper=10.0, steps=6)
    assert got.variance == want.variance
    for (v1, m1, _), (v2, m2, _) in zip(got.tried, want.tried):
        assert v1 == v2 and m1 == pytest.approx(m2, rel=1e-8)


def test_auto_search_mixed_precision_picks_the_same_variance(gpu_ctx):
    d, fold = _problem()
    m = native.Matrix(gpu_ctx, d)
    f64 = cv.auto_search(native.Fit(gpu_ctx, m, d), d, fold, 5)
    mixed = cv.auto_search(native.Fit(gpu_ctx, m, d, precision=native.PRECISION_MIXED), d, fold, 5)
    assert mixed.variance == pytest.approx(f64.variance, rel=1e-4)
