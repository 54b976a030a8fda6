"""The instance-batched sweep (cross-validation grid) against standalone
oracle fits of each instance: same fold weights, same prior variance."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import GRADIENT, MITTAL, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model,kw,conv", [
    (MODEL_LOGISTIC, dict(seed=60, K=500, P=20), GRADIENT),
    (MODEL_LOGISTIC, dict(seed=61, K=400, P=15, formats=("sparse", "dense", "indicator")), MITTAL),
    (MODEL_POISSON, dict(seed=62, K=400, P=15, offset=True, prior=PRIOR_NORMAL), MITTAL),
])
def test_batch_matches_standalone_fits(gpu_ctx, oracle_engine, model, kw, conv):
    d = synthetic.small(model, **kw)
    fold = synthetic.cv_folds(d.K, n_folds=5, seed=3)
    hold, var = synthetic.cv_grid(n_folds=5, n_vars=4, lower=0.01, upper=10.0)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    beta, res, secs = f.batch_find_mode(var, hold, fold, native.ModeFindingArguments(convergence_type=conv))
    for i in range(len(var)):
        di = d.with_prior(int(d.prior_type[-1]), float(var[i]))
        w = (fold != hold[i]).astype(float)
        e = oracle_engine(di)
        e.set_weights(w)
        want = e.fit(conv, 1e-6)
        assert res[i]["iterations"] == want["iterations"], i
        assert res[i]["flag"] == want["flag"]
        err = np.max(np.abs(beta[i] - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
        assert err <= 1e-6, (i, err)
        assert abs(res[i]["loglik"] - want["loglik"]) <= 1e-9 * abs(want["loglik"])
        # held-out predictive log-likelihood: getNewPredictiveLogLikelihood with complement weights
        pred = e.predictive_loglik(1.0 - w)
        assert abs(res[i]["pred_loglik"] - pred) <= 1e-9 * max(1.0, abs(pred)), (i, res[i]["pred_loglik"], pred)


def test_batch_instance_alone_equals_in_batch(gpu_ctx):
    """An instance's result does not depend on the other instances."""
    d = synthetic.small(MODEL_LOGISTIC, seed=63, K=600, P=25)
    fold = synthetic.cv_folds(d.K, n_folds=3, seed=1)
    hold, var = synthetic.cv_grid(n_folds=3, n_vars=3, lower=0.1, upper=2.0)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    b_all, r_all, _ = f.batch_find_mode(var, hold, fold)
    for i in (0, 4, 8):
        b1, r1, _ = f.batch_find_mode(var[i:i + 1], hold[i:i + 1], fold)
        assert np.array_equal(b1[0], b_all[i])
        assert r1[0]["loglik"] == r_all[i]["loglik"]
