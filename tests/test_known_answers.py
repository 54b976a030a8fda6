"""Known answers of the reference's own R tests (test-smallBernoulli.R,
test-smallPoisson.R, test-smallCox.R, test-smallCLR.R, test-weighting.R),
whose gold values come from glm / coxph / clogit.  The data sets are read out of those files by
tests/golden/make_known_answers.py; here the oracle must reproduce the
reference engine's fixtures, and the fixtures must match an independent Newton
solve of the same likelihood (tests/newton.py) to far below the R tests' 1e-4
tolerance.  The R tests' invariants are checked too: dense and sparse
representations give the same fit, fixed coefficients stay at zero, zero
weights give the subset fit, duplicated rows re-weighted give the original
fit, and the Cox predictive log-likelihood of held-out rows is their fit's
log-likelihood."""
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
    if want["weights"] is not None:
        e.set_weights(want["weights"])
    r = e.fit(GRADIENT, 1e-12, max_iter=10_000, fixed=want["fixed"])
    assert r["flag"] == want["flag"] and r["iterations"] == want["iterations"]
    np.testing.assert_allclose(r["beta"], want["beta"], rtol=1e-12, atol=1e-14)
    assert abs(r["loglik"] - want["loglik"]) <= 1e-12 * abs(want["loglik"])
    if want["fisher"] is not None:
        f = e.fisher_information(want["fisher_cols"])
        assert np.max(np.abs(f - want["fisher"])) <= 1e-12 * max(1.0, np.max(np.abs(want["fisher"])))
    np.testing.assert_allclose(e.predictive_estimates(), want["pred_est"], rtol=1e-12, atol=1e-15)
    if want["pred_ll"] is not None:
        assert abs(e.predictive_loglik(want["heldout"]) - want["pred_ll"]) <= 1e-12 * abs(want["pred_ll"])


@pytest.mark.parametrize("name", NAMES)
def test_reference_fit_is_the_mle(name):
    """The gold standard of the R test: the unpenalised MLE (glm / clogit /
    coxph with Breslow ties), here from an independent Newton solve."""
    d, want = load_known(name)
    beta, ll, info = newton_mle(d, want["fixed"], want["weights"])
    scale = max(1.0, np.max(np.abs(beta)))
    assert np.max(np.abs(want["beta"] - beta)) <= 1e-7 * scale
    assert abs(want["loglik"] - ll) <= 1e-10 * abs(ll)
    if d.model_type != MODEL_COX and want["fisher"] is not None:
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


def _same_fit(a, b, rtol=1e-9):
    wa, wb = load_known(a)[1], load_known(b)[1]
    np.testing.assert_allclose(wa["beta"], wb["beta"], rtol=rtol, atol=1e-12)
    assert abs(wa["loglik"] - wb["loglik"]) <= rtol * abs(wa["loglik"])


def test_zero_weights_are_the_subset_fit():
    """test-weighting.R:192-227: weights 0/1 give the fit of the weight-1 rows."""
    _same_fit("bernoulli_zero_weights", "bernoulli_subset", rtol=1e-12)


def test_reweighted_duplicates_are_the_original_fit():
    """test-weighting.R:107-142: three rows duplicated and both copies weighted
    0.5 give the original fit, dense or sparse / indicator columns."""
    _same_fit("coxw_duplicated", "coxw_duplicated_gold")
    _same_fit("coxw_duplicated_sparse", "coxw_duplicated")


def test_cox_predictive_loglik_of_held_out_rows():
    """test-weighting.R:74-105: every row twice, the second copies fitted; the
    predictive log-likelihood of the first copies is the stratified fit's."""
    _same_fit("coxw_predictive", "coxw_predictive_gold")
    _, want = load_known("coxw_predictive")
    _, gold = load_known("coxw_predictive_gold")
    assert abs(want["pred_ll"] - gold["loglik"]) <= 1e-10 * abs(gold["loglik"])


def test_published_sas_fit():
    """test-largeBernoulli.R quotes the SAS fit of CCD_LOGISTIC_TEST_17var.txt
    (22,296 rows, 17 covariates + intercept) as 2 x log-likelihood, to the
    three decimals it prints."""
    _, want = load_known("bernoulli_17var")
    assert abs(2 * want["loglik"] - want["published_2ll"]) <= 5e-4
