"""The mixed-precision batched engine (FP32 exp / ratios / per-entry terms with
compensated sums; FP64 xBeta, reductions, step and log-likelihoods) against
the FP64 oracle fit of every instance.

Tolerances: coefficients within 1e-6 of the oracle's, relative to the largest
coefficient (max |dbeta| / max(|beta|, 1e-8)).  The log-likelihoods are
computed in FP64 from those coefficients; at a penalised mode the likelihood's
gradient equals minus the prior's, so it moves to first order with the
coefficients, and the bound is 1e-8 relative rather than the FP64 engine's
1e-9.  The held-out predictive log-likelihood is not stationary at all in the
coefficients (its gradient on the held-out rows is O(1)), so it gets 1e-7.  The
fits converge to 1e-10 here so that the comparison measures the arithmetic,
not where each run happened to stop; the 1e-6 fits of the benchmark are
compared in the same way by bench.py."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import GRADIENT, MITTAL, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_NORMAL

pytestmark = pytest.mark.gpu

COEF_TOL = 1e-6
LL_TOL = 1e-8
PRED_TOL = 1e-7


def _rel(b, want):
    return np.max(np.abs(b - want)) / max(np.max(np.abs(want)), 1e-8)


@pytest.mark.parametrize("cluster", [1, 3])
@pytest.mark.parametrize("group", [1, 2, 4])
@pytest.mark.parametrize("model,kw,conv", [
    (MODEL_LOGISTIC, dict(seed=70, K=800, P=30), GRADIENT),
    (MODEL_LOGISTIC, dict(seed=71, K=600, P=20, formats=("sparse", "dense", "indicator")), MITTAL),
    (MODEL_POISSON, dict(seed=72, K=600, P=20, offset=True, prior=PRIOR_NORMAL), MITTAL),
])
def test_mixed_batch_matches_fp64_oracle(gpu_ctx, oracle_engine, model, kw, conv, group, cluster):
    """cluster: CTAs per group, each owning a row range of every column."""
    d = synthetic.small(model, **kw)
    fold = synthetic.cv_folds(d.K, n_folds=5, seed=4)
    hold, var = synthetic.cv_grid(n_folds=5, n_vars=3, lower=0.01, upper=10.0)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d, precision=native.PRECISION_MIXED)
    args = native.ModeFindingArguments(convergence_type=conv, tolerance=1e-10, max_iterations=2000)
    beta, res, _ = f.batch_find_mode(var, hold, fold, args, group=group, cluster=cluster)
    worst = 0.0
    for i in range(len(var)):
        di = d.with_prior(int(d.prior_type[-1]), float(var[i]))
        w = (fold != hold[i]).astype(float)
        e = oracle_engine(di)
        e.set_weights(w)
        want = e.fit(conv, 1e-10, 2000)
        assert res[i]["flag"] == want["flag"] == 0, i
        err = _rel(beta[i], want["beta"])
        worst = max(worst, err)
        assert err <= COEF_TOL, (i, err)
        assert abs(res[i]["loglik"] - want["loglik"]) <= LL_TOL * abs(want["loglik"]), i
        pred = e.predictive_loglik(1.0 - w)
        assert abs(res[i]["pred_loglik"] - pred) <= PRED_TOL * max(1.0, abs(pred)), i
    print(f"mixed group={group} cluster={cluster}: max relative coefficient error {worst:.2e}")


@pytest.mark.parametrize("cluster", [1, 4])
def test_mixed_instance_alone_equals_in_group(gpu_ctx, cluster):
    """An instance's arithmetic does not depend on its group mates: alone (its
    group padded) it gives bit-identical coefficients."""
    d = synthetic.small(MODEL_LOGISTIC, seed=73, K=700, P=25)
    fold = synthetic.cv_folds(d.K, n_folds=4, seed=2)
    hold, var = synthetic.cv_grid(n_folds=4, n_vars=3, lower=0.05, upper=5.0)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d, precision=native.PRECISION_MIXED)
    b_all, r_all, _ = f.batch_find_mode(var, hold, fold, group=4, cluster=cluster)
    for i in (0, 5, 11):
        b1, r1, _ = f.batch_find_mode(var[i:i + 1], hold[i:i + 1], fold, group=4, cluster=cluster)
        assert np.array_equal(b1[0], b_all[i])
        assert r1[0]["iterations"] == r_all[i]["iterations"]
        assert r1[0]["loglik"] == r_all[i]["loglik"]


def test_mixed_rejected_by_single_fit_calls(gpu_ctx):
    d = synthetic.small(MODEL_LOGISTIC, seed=74, K=200, P=5)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d, precision=native.PRECISION_MIXED)
    with pytest.raises(native.CcdbError, match="batched fits"):
        f.find_mode()

