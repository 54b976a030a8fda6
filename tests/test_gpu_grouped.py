"""GPU parity of the grouped engine (conditional logistic / conditional
Poisson, one denominator per stratum) against the CPU oracle."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import (GRADIENT, LANGE, MITTAL, MODEL_CONDITIONAL_LOGISTIC,
                           MODEL_CONDITIONAL_POISSON, PRIOR_NORMAL)

pytestmark = pytest.mark.gpu

BETA_TOL, LL_TOL, GH_TOL = 1e-6, 1e-9, 1e-10


def rel_beta(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-8)


CASES = [
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=0, n_strata=30)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=1, n_strata=12, prior=PRIOR_NORMAL, formats=("sparse", "dense"))),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=2, K=900, n_strata=300, formats=("indicator",), P=30)),
    (MODEL_CONDITIONAL_POISSON, dict(seed=3, n_strata=20)),
]


@pytest.mark.parametrize("model,kw", CASES)
def test_grouped_gradient_hessian(gpu_ctx, oracle_engine, model, kw):
    d = synthetic.small(model, **kw)
    ref = oracle_engine(d)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    rng = np.random.default_rng(4)
    for _ in range(2):
        for j in range(d.J):
            g0, h0 = ref.grad_hess(j)
            g1, h1 = f.compute_gradient_and_hessian(j)
            assert abs(g1 - g0) <= GH_TOL * max(1.0, abs(g0)), (j, g0, g1)
            assert abs(h1 - h0) <= GH_TOL * max(1.0, abs(h0)), (j, h0, h1)
            delta = float(rng.normal(0, 0.1))
            ref.update_beta(j, delta)
            f.update_xbeta(j, delta)
    ll0, ll1 = ref.loglik(), f.get_log_likelihood()
    assert abs(ll1 - ll0) <= LL_TOL * abs(ll0)


@pytest.mark.parametrize("model,kw", CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL, LANGE])
@pytest.mark.parametrize("strategy", [native.SWEEP_AUTO, native.SWEEP_GRID_LEVELS, native.SWEEP_SPECULATIVE])
def test_grouped_find_mode(gpu_ctx, oracle_engine, model, kw, conv, strategy):
    """AUTO: one persistent launch per findMode; SPECULATIVE: host-driven batches."""
    d = synthetic.small(model, **kw)
    want = oracle_engine(d).fit(conv, 1e-6)
    got = native.fit_model(gpu_ctx, d, native.ModeFindingArguments(convergence_type=conv, strategy=strategy))
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


def test_clr_weighted(gpu_ctx, oracle_engine):
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=5, K=600, n_strata=60)
    w = (np.random.default_rng(2).random(d.K) > 0.2).astype(float)
    ref = oracle_engine(d)
    ref.set_weights(w)
    want = ref.fit(GRADIENT, 1e-6)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    f.set_weights(w)
    got = f.find_mode()
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL


@pytest.mark.parametrize("form", [native.SWEEP_LEVELS, native.SWEEP_GRID_LEVELS])
def test_clr_device_sweep_on_many_ctas(gpu_ctx, oracle_engine, form):
    """20,000 matched sets (~130,000 rows), 400 indicator columns: the persistent
    sweep's row updates and stratum runs spread over every CTA of its cluster
    form (LEVELS) and of its grid form (GRID_LEVELS)."""
    d = synthetic.conditional_logistic(seed=13, n_sets=20_000, P=400)
    want = oracle_engine(d).fit(GRADIENT, 1e-6)
    got = native.fit_model(gpu_ctx, d, native.ModeFindingArguments(convergence_type=GRADIENT, strategy=form))
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])
