"""GPU parity of the Breslow Cox engine against the CPU oracle (C ABI)."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import GRADIENT, LANGE, MITTAL, MODEL_COX, PRIOR_LAPLACE, PRIOR_NORMAL

pytestmark = pytest.mark.gpu

BETA_TOL = 1e-6
LL_TOL = 1e-9
# The device gradient uses per-group suffix sums (an exact algebraic rewrite of
# the reference's risk-set walk); its rounding differs from the serial loop.
GH_TOL = 1e-9


def rel_beta(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-8)


CASES = [
    dict(seed=0),
    dict(seed=1, prior=PRIOR_NORMAL),
    dict(seed=2, formats=("indicator",), P=20, n_strata=1),
    dict(seed=3, formats=("sparse", "dense"), n_strata=7, tie_days=3),
    dict(seed=4, K=800, n_strata=40, tie_days=2),
]


@pytest.mark.parametrize("kw", CASES)
def test_cox_gradient_hessian(gpu_ctx, oracle_engine, kw):
    d = synthetic.small(MODEL_COX, **kw)
    ref = oracle_engine(d)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    rng = np.random.default_rng(3)
    for sweep in range(2):
        for j in range(d.J):
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


@pytest.mark.parametrize("kw", CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL, LANGE])
@pytest.mark.parametrize("mode", ["device", "device_grid", "host_batches", "per_coordinate"])
def test_cox_find_mode(gpu_ctx, oracle_engine, kw, conv, mode):
    """device: one persistent launch per findMode (group_sweep.cu; a small fit
    takes its cluster form); device_grid: its cooperative grid form;
    host_batches: the host-driven speculative batches; per_coordinate: the
    reference's call pattern, one round trip per coordinate."""
    d = synthetic.small(MODEL_COX, **kw)
    want = oracle_engine(d).fit(conv, 1e-6)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    got = f.find_mode(native.ModeFindingArguments(
        convergence_type=conv, per_coordinate=(mode == "per_coordinate"),
        strategy={"host_batches": native.SWEEP_SPECULATIVE, "device_grid": native.SWEEP_GRID_LEVELS}.get(
            mode, native.SWEEP_AUTO)))
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


def test_cox_zero_weights_drop_rows(gpu_ctx, oracle_engine):
    """Zero weights remove rows from the risk sets (setPidForAccumulation);
    the fit must equal the oracle's weighted fit."""
    d = synthetic.small(MODEL_COX, seed=5, K=600, n_strata=5, tie_days=3)
    w = (np.random.default_rng(1).random(d.K) > 0.3).astype(float)
    ref = oracle_engine(d)
    ref.set_weights(w)
    want = ref.fit(GRADIENT, 1e-6)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    f.set_weights(w)
    got = f.find_mode()
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


def test_cox_deterministic(gpu_ctx):
    d = synthetic.small(MODEL_COX, seed=6, K=3000, P=40, n_strata=30, tie_days=2)
    r1 = native.fit_model(gpu_ctx, d)
    r2 = native.fit_model(gpu_ctx, d)
    assert np.array_equal(r1.beta, r2.beta)
    assert r1.log_likelihood == r2.log_likelihood


@pytest.mark.parametrize("form", [native.SWEEP_LEVELS, native.SWEEP_GRID_LEVELS])
@pytest.mark.parametrize("prior,var", [(PRIOR_LAPLACE, 0.05), (PRIOR_NORMAL, 1.0)])
def test_cox_device_sweep_on_many_ctas(gpu_ctx, oracle_engine, prior, var, form):
    """A problem large enough that the persistent sweep's row updates, group
    runs and scans spread over every CTA: 60,000 rows in 150 strata of uneven
    size, daily ties, 300 indicator columns; the device sweep against the
    oracle and against the host-driven batches."""
    d = synthetic.small(MODEL_COX, seed=12, K=60_000, P=300, density=0.004, n_strata=150, tie_days=4,
                        formats=("indicator",), prior=prior, variance=var)
    want = oracle_engine(d).fit(GRADIENT, 1e-6)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    got = f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, strategy=form), beta=np.zeros(d.J))
    host = f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, strategy=native.SWEEP_SPECULATIVE),
                       beta=np.zeros(d.J))
    for r in (got, host):
        assert r.return_flag == want["flag"]
        assert r.iterations == want["iterations"]
        assert rel_beta(r.beta, want["beta"]) <= BETA_TOL
        assert abs(r.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])
    assert got.kernel_launches < host.kernel_launches


@pytest.mark.parametrize("kw", [CASES[0], CASES[3], CASES[4]])
def test_cox_mixed_precision_against_fp64_oracle(gpu_ctx, oracle_engine, kw):
    """CCDB_PRECISION_MIXED Cox: FP32 exp and per-entry gradient terms with
    compensated sums; FP64 risk-set sums, reductions, step and log-likelihood.
    Fitted to 1e-10 so that the comparison measures the arithmetic rather than
    where each run stopped: coefficients within 1e-6 of their scale of the
    FP64 oracle, log-likelihood within 1e-8."""
    d = synthetic.small(MODEL_COX, **kw)
    want = oracle_engine(d).fit(GRADIENT, 1e-10, 2000)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d, precision=native.PRECISION_MIXED)
    got = f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-10,
                                                  max_iterations=2000))
    assert got.return_flag == want["flag"] == 0
    err = rel_beta(got.beta, want["beta"])
    print(f"mixed Cox: max relative coefficient error {err:.2e}")
    assert err <= 1e-6
    assert abs(got.log_likelihood - want["loglik"]) <= 1e-8 * abs(want["loglik"])


@pytest.mark.parametrize("form", [native.SWEEP_LEVELS, native.SWEEP_GRID_LEVELS])
def test_cox_device_sweep_direct_rebuild_on_two_ctas(oracle_engine, form):
    """Two CTAs for about 45,000 groups: each CTA's group range is larger than
    the staged rebuild holds in shared memory, so the risk-set sums are rebuilt
    straight from global memory (the direct form)."""
    d = synthetic.small(MODEL_COX, seed=12, K=60_000, P=120, density=0.004, n_strata=150, tie_days=4,
                        formats=("indicator",), prior=PRIOR_LAPLACE, variance=0.05)
    want = oracle_engine(d).fit(GRADIENT, 1e-6)
    ctx = native.Context(0)
    ctx.set_max_ctas(2)
    try:
        got = native.fit_model(ctx, d, native.ModeFindingArguments(convergence_type=GRADIENT, strategy=form))
    finally:
        ctx.close()
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


@pytest.mark.parametrize("form", [native.SWEEP_LEVELS, native.SWEEP_GRID_LEVELS])
@pytest.mark.parametrize("kind", ["cox", "clr"])
def test_group_sweep_on_one_cta(oracle_engine, kind, form):
    """A context limited to one CTA (a serving slot for small fits): the group
    sweep runs as a one-CTA cluster (LEVELS) or a one-CTA grid (GRID_LEVELS);
    every row, stratum run and risk-set sum is that CTA's."""
    if kind == "cox":
        d = synthetic.small(MODEL_COX, seed=21, K=8_000, P=60, density=0.02, n_strata=8, tie_days=3,
                            formats=("indicator", "sparse"), prior=PRIOR_LAPLACE, variance=0.1)
    else:
        d = synthetic.conditional_logistic(seed=22, n_sets=900, P=80)
    want = oracle_engine(d).fit(GRADIENT, 1e-6)
    ctx = native.Context(0)
    ctx.set_max_ctas(1)
    try:
        got = native.fit_model(ctx, d, native.ModeFindingArguments(convergence_type=GRADIENT, strategy=form))
    finally:
        ctx.close()
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])
