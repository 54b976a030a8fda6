"""Known answers of the reference's own R tests (test-smallBernoulli.R,
test-smallPoisson.R, test-smallCox.R, test-smallCLR.R), whose gold values
come from glm / coxph / clogit.  The data sets are read out of those files by
tests/golden/make_known_answers.py; here the oracle must reproduce the
reference engine's fixtures, and the fixtures must match an independent Newton
solve of the same likelihood (tests/newton.py) to far below the R tests' 1e-4
tolerance.  The R tests' invariants are checked too: dense and sparse
representations give the same fit, fixed coefficients stay at zero."""
import numpy as np
import pytest

from ccd_b200.data import GRADIENT, MODEL_COX
from oracle import checker

from .golden_io import known_names, load_known
from .newton import newton_mle

NAMES = known_names()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_the_reference(name):
    d, want = load_known(name)
    e = checker.RestatementEngine(d)
    r = e.fit(GRADIENT, 1e-12, max_iter=10_000, fixed=want["fixed"])
    assert r["flag"] == want["flag"] and r["iterations"] == want["iterations"]
    np.testing.assert_allclose(r["beta"], want["beta"], rtol=1e-12, atol=1e-14)
    assert abs(r["loglik"] - want["loglik"]) <= 1e-12 * abs(want["loglik"])
    f = e.fisher_information(want["fisher_cols"])
    assert np.max(np.abs(f - want["fisher"])) <= 1e-12 * max(1.0, np.max(np.abs(want["fisher"])))
    np.testing.assert_allclose(e.predictive_estimates(), want["pred_est"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", NAMES)
def test_reference_fit_is_the_mle(name):
    """The gold standard of the R test: the unpenalised MLE (glm / clogit /
    coxph with Breslow ties), here from an independent Newton solve."""
    d, want = load_known(name)
    beta, ll, info = newton_mle(d, want["fixed"])
    scale = max(1.0, np.max(np.abs(beta)))
    assert np.max(np.abs(want["beta"] - beta)) <= 1e-7 * scale
    assert abs(want["loglik"] - ll) <= 1e-10 * abs(ll)
    if d.model_type != MODEL_COX:
        # getSEs / vcov: the inverse Fisher information is the MLE's covariance
        # (the canonical GLMs and the conditional logistic likelihood: expected
        # = observed information)
        se_ref = np.sqrt(np.diag(np.linalg.inv(want["fisher"])))
        se_newton = np.sqrt(np.diag(np.linalg.inv(info)))
        np.testing.assert_allclose(se_ref, se_newton, rtol=1e-6)


def test_representations_agree():
    """test-smallBernoulli.R:54-73, test-smallPoisson.R:96-136: the same
    covariate stored dense, sparse or as indicators gives the same fit."""
    for a, b in (("bernoulli_dense", "bernoulli_sparse"), ("dobson_dense", "dobson_indicator")):
        wa, wb = load_known(a)[1], load_known(b)[1]
        np.testing.assert_allclose(wa["beta"], wb["beta"], rtol=1e-10, atol=1e-12)
        assert abs(wa["loglik"] - wb["loglik"]) <= 1e-12 * abs(wa["loglik"])


def test_fixed_coefficients_stay_at_zero():
    """test-smallPoisson.R:29-46: fixedCoefficients hold their starting value."""
    d, want = load_known("dobson_fixed")
    assert want["beta"][1] == 0.0 and want["beta"][3] == 0.0
