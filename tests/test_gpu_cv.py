"""Cross-validation drivers on the batched engine against the same drivers
run on oracle fits (one CPU fit per fold and variance, cold start)."""
import numpy as np
import pytest

from ccd_b200 import cv, native, synthetic
from ccd_b200.data import (GRADIENT, MODEL_CONDITIONAL_LOGISTIC, MODEL_LOGISTIC, PRIOR_LAPLACE, PRIOR_NONE,
                           PRIOR_NORMAL)

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

    def fold_instances(self, variances, holdout, row_fold, args=None):
        """native.Fit.fold_instances' contract: per-column variances."""
        res = []
        for v, h in zip(variances, holdout):
            d = self.d.with_prior(int(self.d.prior_type[-1]), 1.0)
            d.prior_type = self.d.prior_type.copy()
            d.prior_var = np.array(v, dtype=np.float64)
            e = self.engine(d)
            w = (row_fold != h).astype(float)
            e.set_weights(w)
            r = e.fit(GRADIENT, 1e-6)
            res.append({"flag": r["flag"],
                        "pred_loglik": e.predictive_loglik(1.0 - w) if r["flag"] == 0 else float("nan")})
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


def _agree(got, want):
    assert len(got.tried) == len(want.tried)
    for (v1, m1, _), (v2, m2, _) in zip(got.tried, want.tried):
        assert v1 == pytest.approx(v2, rel=1e-6)
        assert m1 == pytest.approx(m2, rel=1e-8)
    np.testing.assert_allclose(got.variances, want.variances, rtol=1e-6)


def test_auto_search_conditional_logistic_through_standalone_fits(gpu_ctx, oracle_engine):
    """A model the batched engine does not take: every (fold, variance) is a
    standalone device fit (native.Fit.fold_instances)."""
    # an interior optimum: the search path holds under 1e-8 relative changes of
    # the held-out values (flatter problems end at variances near 0 by rounding)
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=83, K=400, P=6, n_strata=60, prior=PRIOR_NORMAL)
    fold = synthetic.cv_folds(d.K, n_folds=4, seed=10)
    m = native.Matrix(gpu_ctx, d)
    got = cv.auto_search(native.Fit(gpu_ctx, m, d), d, fold, 4)
    want = cv.auto_search(OracleBatch(oracle_engine, d), d, fold, 4)
    _agree(got, want)


def test_auto_search_two_variance_parameters(gpu_ctx, oracle_engine):
    """Columns under two priors: the search tunes each variance parameter in
    turn (standalone device fits with per-column variances)."""
    d, fold = _problem()
    d.prior_type[1:13] = PRIOR_LAPLACE
    d.prior_var[1:13] = 1.0
    d.prior_type[13:] = PRIOR_NORMAL
    d.prior_var[13:] = 2.0
    assert len(cv.variance_groups(d)) == 2
    m = native.Matrix(gpu_ctx, d)
    got = cv.auto_search(native.Fit(gpu_ctx, m, d), d, fold, 5, max_cycles=5)
    want = cv.auto_search(OracleBatch(oracle_engine, d), d, fold, 5, max_cycles=5)
    _agree(got, want)
    assert got.rounds == want.rounds and got.converged == want.converged
    r = cv.refit_at(gpu_ctx, m, d, got.variances)
    dv = d.with_prior(PRIOR_NONE, 1.0)
    dv.prior_type = d.prior_type.copy()
    dv.prior_var = cv.column_variances(d, got.variances)
    ref = oracle_engine(dv).fit(GRADIENT, 1e-6)
    assert np.max(np.abs(r.beta - ref["beta"])) <= 1e-6 * max(np.max(np.abs(ref["beta"])), 1e-8)


def test_grid_search_two_variance_parameters(gpu_ctx, oracle_engine):
    """The grid moves the first variance parameter only (standalone device
    fits with per-column variances); the second keeps the prior's value."""
    d, fold = _problem()
    d.prior_type[13:] = PRIOR_NORMAL
    d.prior_var[13:] = 2.0
    m = native.Matrix(gpu_ctx, d)
    got = cv.grid_search(native.Fit(gpu_ctx, m, d), fold, 5, lower=0.01, upper=10.0, steps=6)
    want = cv.grid_search(OracleBatch(oracle_engine, d), fold, 5, lower=0.01, upper=10.0, steps=6)
    assert got.variance == want.variance
    for (v1, m1, _), (v2, m2, _) in zip(got.tried, want.tried):
        assert v1 == v2 and m1 == pytest.approx(m2, rel=1e-8)
