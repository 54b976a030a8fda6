"""GPU parity of the independent-row engine (logistic, Poisson) against the
CPU oracle, through the C ABI."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import (GRADIENT, LANGE, MITTAL, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE,
                           PRIOR_NORMAL)

pytestmark = pytest.mark.gpu

BETA_TOL = 1e-6   # max|dbeta| / max(|beta|, 1e-8)
LL_TOL = 1e-9     # relative log-likelihood
GH_TOL = 1e-10    # relative gradient / Hessian of one coordinate


def rel_beta(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-8)


CASES = [
    (MODEL_LOGISTIC, dict(seed=0)),
    (MODEL_LOGISTIC, dict(seed=1, prior=PRIOR_NORMAL)),
    (MODEL_LOGISTIC, dict(seed=2, formats=("indicator",), P=30)),
    (MODEL_POISSON, dict(seed=0)),
    (MODEL_POISSON, dict(seed=1, offset=True, prior=PRIOR_NORMAL)),
    (MODEL_POISSON, dict(seed=2, formats=("sparse", "dense"), offset=True)),
]


@pytest.mark.parametrize("model,kw", CASES)
def test_per_coordinate_gradient_hessian(gpu_ctx, oracle_engine, model, kw):
    d = synthetic.small(model, **kw)
    ref = oracle_engine(d)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    rng = np.random.default_rng(7)
    start = 1 if d.offset_col0 else 0
    for sweep in range(2):
        for j in range(start, d.J):
            g0, h0 = ref.grad_hess(j)
            g1, h1 = f.compute_gradient_and_hessian(j)
            assert abs(g1 - g0) <= GH_TOL * max(1.0, abs(g0)), (j, g0, g1)
            assert abs(h1 - h0) <= GH_TOL * max(1.0, abs(h0)), (j, h0, h1)
            delta = float(rng.normal(0, 0.1))
            ref.update_beta(j, delta)
            f.update_xbeta(j, delta)
    np.testing.assert_allclose(f.get_xbeta(), ref.xbeta(), rtol=1e-12, atol=1e-12)
    ll0, ll1 = ref.loglik(), f.get_log_likelihood()
    assert abs(ll1 - ll0) <= LL_TOL * abs(ll0)


@pytest.mark.parametrize("model,kw", CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL, LANGE])
@pytest.mark.parametrize("mode", ["levels", "grid_levels", "speculative", "resident", "per_coordinate"])
def test_find_mode_matches_oracle(gpu_ctx, oracle_engine, model, kw, conv, mode):
    d = synthetic.small(model, **kw)
    want = oracle_engine(d).fit(conv, 1e-6)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    strategy = {"levels": native.SWEEP_LEVELS, "grid_levels": native.SWEEP_GRID_LEVELS,
                "speculative": native.SWEEP_SPECULATIVE, "resident": native.SWEEP_RESIDENT}.get(mode, 0)
    got = f.find_mode(native.ModeFindingArguments(convergence_type=conv, strategy=strategy,
                                                  per_coordinate=(mode == "per_coordinate")))
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


@pytest.mark.parametrize("strategy", [1, 2, 3, 4])
def test_logistic_l1_benchmark_problem(gpu_ctx, oracle_engine, strategy):
    """10,000 x 1,000 L1 logistic, MITTAL 1e-6, the reference's CPU-runnable case."""
    d = synthetic.logistic_l1(seed=1)
    want = oracle_engine(d).fit(MITTAL, 1e-6)
    got = native.fit_model(gpu_ctx, d, native.ModeFindingArguments(convergence_type=MITTAL,
                                                                   strategy=strategy))
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


def test_weighted_fit(gpu_ctx, oracle_engine):
    d = synthetic.small(MODEL_LOGISTIC, seed=3, K=400)
    w = (np.arange(d.K) % 5 != 0).astype(float)
    ref = oracle_engine(d)
    ref.set_weights(w)
    want = ref.fit(GRADIENT, 1e-6)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    f.set_weights(w)
    got = f.find_mode()
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL


def test_fused_is_deterministic(gpu_ctx):
    d = synthetic.small(MODEL_POISSON, seed=4, K=2000, P=60, offset=True)
    r1 = native.fit_model(gpu_ctx, d)
    r2 = native.fit_model(gpu_ctx, d)
    assert np.array_equal(r1.beta, r2.beta)
    assert r1.log_likelihood == r2.log_likelihood


@pytest.mark.parametrize("model,kw", [
    (MODEL_POISSON, dict(offset=True, prior=PRIOR_NORMAL)),
    (MODEL_LOGISTIC, dict()),
])
@pytest.mark.parametrize("strategy", [1, 3])
def test_split_columns_beyond_the_stage(gpu_ctx, oracle_engine, model, kw, strategy):
    """700,000 rows: the intercept splits over every CTA in chunks longer than a
    CTA stages, so its gradient takes the streaming path -- on the first
    dependency level, where the staged column metadata must be published to all
    threads before the level starts (both level sweeps)."""
    d = synthetic.small(model, seed=5, K=700_000, P=3, density=0.001, formats=("indicator",), **kw)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    r = f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, strategy=strategy))
    want = oracle_engine(d).fit(GRADIENT, 1e-6)
    assert r.return_flag == want["flag"] and r.iterations == want["iterations"]
    assert rel_beta(r.beta, want["beta"]) <= BETA_TOL
    assert abs(r.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


@pytest.mark.parametrize("max_ctas", [1, 3, 18])
def test_find_mode_on_a_share_of_the_sms(oracle_engine, max_ctas):
    """A context limited to a few CTAs (the serving loop's slots) builds its
    sweep schedule for that grid: longer chunks, more split columns per CTA."""
    ctx = native.Context(0)
    try:
        ctx.set_max_ctas(max_ctas)
        for d in (synthetic.small(MODEL_POISSON, seed=6, K=120_000, P=8, density=0.01, offset=True,
                                  prior=PRIOR_NORMAL, formats=("indicator", "sparse")),
                  synthetic.logistic_l1(seed=7, K=20_000, P=400)):
            m = native.Matrix(ctx, d)
            f = native.Fit(ctx, m, d)
            r = f.find_mode(native.ModeFindingArguments(strategy=native.SWEEP_LEVELS))
            want = oracle_engine(d).fit(GRADIENT, 1e-6)
            assert r.return_flag == want["flag"] and r.iterations == want["iterations"]
            assert rel_beta(r.beta, want["beta"]) <= BETA_TOL
            assert abs(r.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])
            f.close()
            m.close()
    finally:
        ctx.close()
