"""Calls on a fitted state on the GPU, through the C ABI: Fisher information
(ccdb_fisher_information), predictive log-likelihood and predictive estimates,
against the golden fixtures of the reference engine and the CPU oracle, and
through the reference's own CyclicCoordinateDescent over the drop-in adapter.

Tolerances (FP64 throughout; only the summation order differs from the
reference): Fisher entries within 1e-10 of the matrix's largest entry at the
reference's coefficients; predictions 1e-12 relative; predictive
log-likelihood 1e-11 relative."""
import os

import numpy as np
import pytest

from ccd_b200 import inference, native, synthetic
from ccd_b200.data import (GRADIENT, MITTAL, MODEL_CONDITIONAL_LOGISTIC, MODEL_CONDITIONAL_POISSON,
                           MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_NORMAL)
from oracle import checker

from .golden_io import case_names, load_case

pytestmark = pytest.mark.gpu

FISHER_TOL = 1e-10


def _fit_at(gpu_ctx, d, beta, w=None):
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    if w is not None:
        f.set_weights(w)
    f.set_beta(beta)
    return m, f


@pytest.mark.parametrize("name", case_names())
def test_postfit_calls_match_golden(gpu_ctx, name):
    d, w, want = load_case(name)
    m, f = _fit_at(gpu_ctx, d, want["beta"], w)
    if "fisher" in want:
        got = f.compute_fisher_information(want["fisher_cols"])
        scale = np.max(np.abs(want["fisher"]))
        assert np.max(np.abs(got - want["fisher"])) <= FISHER_TOL * scale
        assert np.array_equal(got, got.T)
    else:
        with pytest.raises(native.CcdbError) as ei:
            f.compute_fisher_information(np.arange(d.J))
        assert ei.value.code == native.ERR_UNSUPPORTED
    np.testing.assert_allclose(f.get_predictive_estimates(), want["pred_est"], rtol=1e-12, atol=1e-15)
    ll = f.get_predictive_log_likelihood(want["heldout"])
    assert abs(ll - want["pred_ll"]) <= 1e-11 * max(1.0, abs(want["pred_ll"]))


@pytest.mark.parametrize("model,kw", [
    (MODEL_LOGISTIC, dict(seed=80, P=30, formats=("sparse", "dense", "indicator"))),
    (MODEL_POISSON, dict(seed=81, P=20, offset=True, prior=PRIOR_NORMAL)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=82, P=20, n_strata=40, formats=("sparse", "dense", "indicator"))),
    (MODEL_CONDITIONAL_POISSON, dict(seed=83, P=12, n_strata=30)),
    (MODEL_COX, dict(seed=84, P=20, n_strata=6, tie_days=2, formats=("sparse", "dense", "indicator"))),
])
def test_fisher_after_a_gpu_fit_matches_oracle(gpu_ctx, model, kw):
    """Several passes of kFisherSlots columns, every format, on the GPU's own
    mode; the oracle evaluates the same coefficients."""
    d = synthetic.small(model, **kw)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    r = f.find_mode(native.ModeFindingArguments(convergence_type=MITTAL, tolerance=1e-8))
    assert r.return_flag == 0
    cols = np.arange(1 if d.offset_col0 else 0, d.J, dtype=np.int32)
    got = f.compute_fisher_information(cols)
    e = checker.RestatementEngine(d)
    e.set_beta(r.beta)
    want = e.fisher_information(cols)
    assert np.max(np.abs(got - want)) <= FISHER_TOL * np.max(np.abs(want))
    # a subset with a repeat is the matching block of the full matrix
    sub = np.array([3, 0, 3, len(cols) - 1], np.int32)
    part = f.compute_fisher_information(cols[sub])
    assert np.max(np.abs(part - got[np.ix_(sub, sub)])) <= FISHER_TOL * np.max(np.abs(want))
    # standard errors as getSEs forms them
    se = inference.standard_errors(f)
    np.testing.assert_allclose(se, np.sqrt(np.diag(np.linalg.inv(want))), rtol=1e-8)


def test_fisher_arguments(gpu_ctx):
    d = synthetic.small(MODEL_LOGISTIC, seed=85, K=200, P=5)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    assert f.compute_fisher_information(np.array([], np.int32)).shape == (0, 0)
    with pytest.raises(native.CcdbError) as ei:
        f.compute_fisher_information([0, d.J])
    assert ei.value.code == native.ERR_INVALID


def test_cox_predictive_call_restores_the_fit(gpu_ctx):
    """The Cox predictive log-likelihood regroups under the held-out weights
    and returns to the fit's own risk sets: the fit's log-likelihood and its
    next gradients are unchanged."""
    d = synthetic.small(MODEL_COX, seed=86, n_strata=5, tie_days=3)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT))
    ll0 = f.get_log_likelihood()
    gh0 = [f.compute_gradient_and_hessian(j) for j in range(d.J)]
    held = (np.arange(d.K) % 3 == 0).astype(float)
    e = checker.RestatementEngine(d)
    e.set_beta(f.get_beta())
    want = e.predictive_loglik(held)
    got = f.get_predictive_log_likelihood(held)
    assert abs(got - want) <= 1e-11 * abs(want)
    assert abs(f.get_log_likelihood() - ll0) <= 1e-13 * abs(ll0)
    np.testing.assert_allclose([f.compute_gradient_and_hessian(j) for j in range(d.J)], gh0,
                               rtol=1e-12, atol=1e-13)


dropin = pytest.mark.skipif(not (os.path.exists(checker.REF_B200_LIB) and checker.reference_available()),
                            reason="reference solver / adapter not built here")


@dropin
@pytest.mark.parametrize("model,kw", [
    (MODEL_LOGISTIC, dict(seed=87)),
    (MODEL_POISSON, dict(seed=88, offset=True, prior=PRIOR_NORMAL, P=8)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=89, n_strata=30)),
    (MODEL_COX, dict(seed=90, n_strata=4, tie_days=3, prior=PRIOR_NORMAL)),
])
def test_reference_solver_postfit_calls_on_b200(model, kw):
    """The reference's CyclicCoordinateDescent asks the adapter for the Fisher
    information pair by pair, for the asymptotic variance (its own Eigen
    inverse) and for the predictive log-likelihood / estimates."""
    d = synthetic.small(model, **kw)
    a, b = checker.ReferenceEngine(d), checker.ReferenceOnB200Engine(d)
    a.fit(MITTAL, 1e-8)
    b.fit(MITTAL, 1e-8)
    cols = np.arange(1 if d.offset_col0 else 0, d.J, dtype=np.int32)
    fa, fb = a.fisher_information(cols), b.fisher_information(cols)
    # the two fits agree to the solver tolerance, and so do calls on them
    assert np.max(np.abs(fa - fb)) <= 1e-6 * np.max(np.abs(fa))
    held = (np.arange(d.K) % 4 == 1).astype(float)
    assert abs(a.predictive_loglik(held) - b.predictive_loglik(held)) <= 1e-7 * abs(a.predictive_loglik(held))
    np.testing.assert_allclose(b.predictive_estimates(held), a.predictive_estimates(held), rtol=1e-6, atol=1e-10)
    if kw.get("prior") == PRIOR_NORMAL:
        i, j = int(cols[0]), int(cols[-1])
        va, vb = a.asymptotic_variance(i, j), b.asymptotic_variance(i, j)
        assert abs(va - vb) <= 1e-6 * max(abs(a.asymptotic_variance(i, i)), 1e-12)
    w = (np.arange(d.K) % 5 != 0).astype(float)
    b.set_weights(w)
    with pytest.raises(checker.FisherRefused):
        b.fisher_information(cols)
