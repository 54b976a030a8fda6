"""GPU parity of the resident sweep (one CTA, the row state in shared memory,
or in global memory for larger fits) against the CPU oracle: short columns in
speculative warp batches, long columns on the whole CTA, weights, fixed
columns, the global form and AUTO's choice of it."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import GRADIENT, LANGE, MITTAL, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL

pytestmark = pytest.mark.gpu

BETA_TOL = 1e-6
LL_TOL = 1e-9


def rel_beta(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-8)


def check(got, want):
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    assert rel_beta(got.beta, want["beta"]) <= BETA_TOL
    assert abs(got.log_likelihood - want["loglik"]) <= LL_TOL * abs(want["loglik"])


RESIDENT = native.ModeFindingArguments(strategy=native.SWEEP_RESIDENT)

CASES = [
    # K = 300: every column is short (one warp each)
    (MODEL_LOGISTIC, dict(seed=10)),
    (MODEL_POISSON, dict(seed=11, offset=True, prior=PRIOR_NORMAL)),
    # K = 3000 with dense columns: long columns on the whole CTA between warp batches
    (MODEL_LOGISTIC, dict(seed=12, K=3000, P=80, density=0.05)),
    (MODEL_POISSON, dict(seed=13, K=3000, P=80, density=0.05, formats=("sparse", "dense"), offset=True)),
    # denser sparse columns: some above the warp limit
    (MODEL_LOGISTIC, dict(seed=14, K=4000, P=50, density=0.12, formats=("indicator", "sparse"))),
]


@pytest.mark.parametrize("model,kw", CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL, LANGE])
def test_resident_matches_oracle(gpu_ctx, oracle_engine, model, kw, conv):
    d = synthetic.small(model, **kw)
    want = oracle_engine(d).fit(conv, 1e-6)
    args = native.ModeFindingArguments(convergence_type=conv, strategy=native.SWEEP_RESIDENT)
    check(native.fit_model(gpu_ctx, d, args), want)


def test_resident_weighted(gpu_ctx, oracle_engine):
    d = synthetic.small(MODEL_LOGISTIC, seed=15, K=2000, P=40)
    w = np.random.default_rng(3).uniform(0.0, 2.0, d.K)
    w[::7] = 0.0
    ref = oracle_engine(d)
    ref.set_weights(w)
    want = ref.fit(GRADIENT, 1e-6)
    f = native.Fit(gpu_ctx, native.Matrix(gpu_ctx, d), d)
    f.set_weights(w)
    check(f.find_mode(RESIDENT), want)


def test_resident_fixed_columns(gpu_ctx, oracle_engine):
    d = synthetic.small(MODEL_POISSON, seed=16, K=1500, P=30, offset=True)
    fixed = np.zeros(d.J, np.uint8)
    fixed[[0, 3, 7, 20]] = 1
    want = oracle_engine(d).fit(GRADIENT, 1e-6, fixed=fixed)
    f = native.Fit(gpu_ctx, native.Matrix(gpu_ctx, d), d)
    args = native.ModeFindingArguments(strategy=native.SWEEP_RESIDENT, fixed=fixed)
    check(f.find_mode(args), want)


def test_resident_same_as_cluster_sweep_within_tolerance(gpu_ctx):
    d = synthetic.logistic_l1(seed=1)
    a = native.fit_model(gpu_ctx, d, native.ModeFindingArguments(convergence_type=MITTAL,
                                                                 strategy=native.SWEEP_RESIDENT))
    b = native.fit_model(gpu_ctx, d, native.ModeFindingArguments(convergence_type=MITTAL,
                                                                 strategy=native.SWEEP_LEVELS))
    assert a.iterations == b.iterations
    assert rel_beta(a.beta, b.beta) <= BETA_TOL
    assert a.kernel_launches == b.kernel_launches  # one sweep launch per attempt either way


def test_resident_is_deterministic(gpu_ctx):
    d = synthetic.small(MODEL_LOGISTIC, seed=17, K=5000, P=200, density=0.02)
    r1 = native.fit_model(gpu_ctx, d, RESIDENT)
    r2 = native.fit_model(gpu_ctx, d, RESIDENT)
    assert np.array_equal(r1.beta, r2.beta)
    assert r1.log_likelihood == r2.log_likelihood


def test_auto_takes_resident_for_small_fits(gpu_ctx):
    d = synthetic.small(MODEL_LOGISTIC, seed=18, K=800, P=20)
    r0 = native.fit_model(gpu_ctx, d, native.ModeFindingArguments())
    r1 = native.fit_model(gpu_ctx, d, RESIDENT)
    assert np.array_equal(r0.beta, r1.beta)


GLOBAL_CASES = [
    # 40,000 rows: the row state in global memory; columns of ~400 entries, two
    # chunks of one warp each
    (MODEL_LOGISTIC, dict(seed=19, K=40_000, P=60, density=0.01, formats=("indicator", "sparse"))),
    (MODEL_POISSON, dict(seed=20, K=30_000, P=40, density=0.02, offset=True, prior=PRIOR_NORMAL,
                         formats=("indicator", "sparse"))),
    # ~3,000-entry columns (above the warp limit) and dense ones on the whole CTA
    (MODEL_LOGISTIC, dict(seed=21, K=25_000, P=24, density=0.12)),
]


@pytest.mark.parametrize("model,kw", GLOBAL_CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL])
def test_resident_global_form_matches_oracle(gpu_ctx, oracle_engine, model, kw, conv):
    """More rows than shared memory holds: the same sweep with the row state in
    a global array, asked for by CCDB_SWEEP_RESIDENT."""
    d = synthetic.small(model, **kw)
    want = oracle_engine(d).fit(conv, 1e-6)
    args = native.ModeFindingArguments(convergence_type=conv, strategy=native.SWEEP_RESIDENT)
    check(native.fit_model(gpu_ctx, d, args), want)


def test_auto_leaves_large_fits_to_the_cluster_sweep(gpu_ctx, oracle_engine):
    """Beyond shared memory AUTO runs the cluster sweep (the same bits as
    asking for it); the global resident form, asked for, matches the oracle."""
    d = synthetic.logistic_l1(seed=22, K=30_000, P=400, density=0.01)
    want = oracle_engine(d).fit(GRADIENT, 1e-6)
    a = native.fit_model(gpu_ctx, d, native.ModeFindingArguments())
    b = native.fit_model(gpu_ctx, d, native.ModeFindingArguments(strategy=native.SWEEP_LEVELS))
    assert np.array_equal(a.beta, b.beta)
    check(a, want)
    check(native.fit_model(gpu_ctx, d, RESIDENT), want)
