"""Mode-finding variants on the GPU, through the C ABI, against the oracle
(which is bit-exact with the reference for them): the KKT swindle, the MM
algorithm, fixed coefficients; and the reference's own solver running the
same variants over the drop-in adapter.

Tolerances as for plain fits: same iteration count and return flag,
coefficients within 1e-6 relative to the largest, log-likelihood 1e-9."""
import os
import re

import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import (GRADIENT, LANGE, MITTAL, MODEL_CONDITIONAL_LOGISTIC, MODEL_CONDITIONAL_POISSON,
                           MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL)
from oracle import checker

from .test_oracle_postfit import _dense

pytestmark = pytest.mark.gpu

CASES = [
    (MODEL_LOGISTIC, dict(seed=130, P=24)),
    (MODEL_POISSON, dict(seed=131, offset=True)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=132, n_strata=40)),
    (MODEL_CONDITIONAL_POISSON, dict(seed=133, n_strata=30)),
    (MODEL_COX, dict(seed=134, n_strata=6, tie_days=3)),
]
STRATIFIED = CASES[2:]


def _gpu_fit(gpu_ctx, d, w=None, **args):
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    if w is not None:
        f.set_weights(w)
    return f.find_mode(native.ModeFindingArguments(**args))


def _oracle_fit(d, w=None, **kw):
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    return e.fit(**kw)


def _agree(got, want):
    assert got.return_flag == want["flag"]
    assert got.iterations == want["iterations"]
    err = np.max(np.abs(got.beta - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
    assert err <= 1e-6, err
    assert abs(got.log_likelihood - want["loglik"]) <= 1e-9 * abs(want["loglik"])


@pytest.mark.parametrize("model,kw", CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL])
def test_kkt_swindle_matches_oracle(gpu_ctx, model, kw, conv):
    d = synthetic.small(model, **kw)
    want = _oracle_fit(d, conv_type=conv, tol=1e-7, kkt_swindle=True)
    got = _gpu_fit(gpu_ctx, d, convergence_type=conv, tolerance=1e-7, kkt_swindle=True)
    _agree(got, want)


@pytest.mark.parametrize("strategy", [1, 2])
def test_kkt_swindle_weighted_fixed_mixed_priors(gpu_ctx, strategy):
    """Both sweep strategies of the independent-row engine under the swindle's
    changing fixed sets."""
    d = synthetic.small(MODEL_LOGISTIC, seed=135, P=16)
    d.prior_type[3] = PRIOR_NORMAL
    w = (np.arange(d.K) % 6 != 0).astype(float)
    fixed = np.zeros(d.J, np.uint8)
    fixed[5] = 1
    want = _oracle_fit(d, w, conv_type=GRADIENT, tol=1e-7, kkt_swindle=True, fixed=fixed)
    got = _gpu_fit(gpu_ctx, d, w, convergence_type=GRADIENT, tolerance=1e-7, kkt_swindle=True,
                   fixed=fixed, strategy=strategy)
    _agree(got, want)
    assert got.beta[5] == 0.0


def test_kkt_swindle_limited_passes(gpu_ctx):
    d = synthetic.small(MODEL_LOGISTIC, seed=136, P=20, variance=100.0)
    want = _oracle_fit(d, conv_type=GRADIENT, tol=1e-8, max_iter=2, kkt_swindle=True)
    got = _gpu_fit(gpu_ctx, d, convergence_type=GRADIENT, tolerance=1e-8, max_iterations=2,
                   kkt_swindle=True)
    _agree(got, want)


@pytest.mark.parametrize("model,kw", STRATIFIED)
@pytest.mark.parametrize("prior", [PRIOR_LAPLACE, PRIOR_NORMAL])
def test_mm_matches_oracle(gpu_ctx, model, kw, prior):
    d = synthetic.small(model, prior=prior, **kw)
    want = _oracle_fit(d, conv_type=MITTAL, tol=1e-8, algorithm=1)
    got = _gpu_fit(gpu_ctx, d, convergence_type=MITTAL, tolerance=1e-8, algorithm=native.ALGORITHM_MM)
    _agree(got, want)


def test_mm_with_kkt_swindle_matches_oracle(gpu_ctx):
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=137, n_strata=40)
    want = _oracle_fit(d, conv_type=GRADIENT, tol=1e-7, algorithm=1, kkt_swindle=True)
    got = _gpu_fit(gpu_ctx, d, convergence_type=GRADIENT, tolerance=1e-7, algorithm=native.ALGORITHM_MM,
                   kkt_swindle=True)
    _agree(got, want)


@pytest.mark.parametrize("formats", [("sparse", "indicator"), ("sparse",), ("indicator", "dense", "sparse")])
def test_mm_product_follows_the_transpose_format(gpu_ctx, formats):
    """The MM cycle's xBeta over the reference's one-format transpose
    (CompressedDataMatrix.cpp:151-209): SPARSE + INDICATOR without DENSE counts
    each non-zero entry as 1, which on this problem makes the log posterior
    fall by 0.05 in the third cycle ("Non-increasing!", as the reference)."""
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=150, n_strata=20, formats=formats,
                        prior=PRIOR_NORMAL, variance=4.0)
    try:
        want = _oracle_fit(d, conv_type=MITTAL, tol=1e-8, algorithm=1)
    except RuntimeError as ex:
        with pytest.raises(native.CcdbError, match=re.escape(str(ex))):
            _gpu_fit(gpu_ctx, d, convergence_type=MITTAL, tolerance=1e-8, algorithm=native.ALGORITHM_MM)
        return
    got = _gpu_fit(gpu_ctx, d, convergence_type=MITTAL, tolerance=1e-8, algorithm=native.ALGORITHM_MM)
    _agree(got, want)


@pytest.mark.parametrize("formats,unit", [(("sparse", "indicator"), True), (("sparse", "indicator", "dense"), False)])
def test_mm_cycle_xbeta_is_the_transpose_product(gpu_ctx, formats, unit):
    """After one MM cycle the device xBeta is X' beta, X' = X with every
    non-zero entry 1 when the matrix has INDICATOR and no DENSE columns."""
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=151, n_strata=15, formats=formats,
                        prior=PRIOR_NORMAL, variance=4.0)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    r = f.find_mode(native.ModeFindingArguments(convergence_type=MITTAL, tolerance=1e-8, max_iterations=1,
                                                algorithm=native.ALGORITHM_MM))
    X = _dense(d)
    if unit:
        X = (X != 0).astype(float)
    np.testing.assert_allclose(f.get_xbeta(), X @ r.beta, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("formats,unit", [(("sparse", "indicator"), True), (("indicator",), True),
                                          (("sparse", "dense"), False), (("sparse",), False)])
def test_compute_xbeta_from_beta(gpu_ctx, formats, unit):
    """ccdb_compute_xbeta, ModelSpecifics::computeXBeta(double* beta, bool):
    X' beta against numpy, X' = X with non-zero entries 1 exactly when the
    matrix has INDICATOR and no DENSE columns; the statistics follow on demand."""
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=152, n_strata=15, formats=formats)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    beta = np.random.default_rng(152).normal(0.0, 0.5, d.J)
    f.compute_xbeta(beta)
    X = _dense(d)
    if unit:
        X = (X != 0).astype(float)
    np.testing.assert_allclose(f.get_xbeta(), X @ beta, rtol=1e-12, atol=1e-12)
    f.compute_remaining_statistics()
    e = checker.RestatementEngine(d)
    e.set_beta(beta)
    if not unit:  # the oracle's state from beta is X beta
        assert abs(f.get_log_likelihood() - e.loglik()) <= 1e-11 * abs(e.loglik())


@pytest.mark.parametrize("model", [MODEL_LOGISTIC, MODEL_POISSON])
def test_mm_refused_without_strata(gpu_ctx, model):
    d = synthetic.small(model, seed=138, offset=(model == MODEL_POISSON))
    with pytest.raises(native.CcdbError) as ei:
        _gpu_fit(gpu_ctx, d, algorithm=native.ALGORITHM_MM)
    assert ei.value.code == native.ERR_UNSUPPORTED


def test_mm_gradient_hessian_is_the_bound(gpu_ctx):
    """Against numpy on the GPU's own state (conditional logistic):
    g_j = sum_k nEv_s e_k x_kj / d_s - XjY_j, h_j = sum_k nEv_s e_k x_kj^2 / d_s
    (indicator columns drop one x), fixed columns (0, 0)."""
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=139, n_strata=25,
                        formats=("sparse", "dense", "indicator"))
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, max_iterations=3))
    fixed = np.zeros(d.J, np.uint8)
    fixed[1] = 1
    g, h = f.compute_mm_gradient_and_hessian(fixed)
    xb = f.get_xbeta()
    e = np.exp(xb)
    s = np.unique(d.stratum, return_inverse=True)[1]
    den = np.bincount(s, weights=e)
    nev = np.bincount(s, weights=d.y)
    fac = nev[s] * e / den[s]
    for j in range(d.J):
        if fixed[j]:
            assert g[j] == 0.0 and h[j] == 0.0
            continue
        f_ = int(d.fmt[j])
        if f_ == 0:
            r, x = np.arange(d.K), d.vals[d.val_start[j]:d.val_start[j] + d.K]
        else:
            r = d.rows[d.col_start[j]:d.col_start[j + 1]]
            x = d.vals[d.val_start[j]:d.val_start[j] + len(r)] if f_ == 1 else np.ones(len(r))
        gw = np.sum(fac[r] * x) - np.sum(x * d.y[r])
        hw = np.sum(fac[r] * x * (x if f_ != 2 else 1.0))
        assert abs(g[j] - gw) <= 1e-10 * max(1.0, abs(gw))
        assert abs(h[j] - hw) <= 1e-10 * max(1.0, abs(hw))


@pytest.mark.parametrize("model,kw", CASES)
@pytest.mark.parametrize("strategy", [0, 2])
def test_fixed_coefficients_match_oracle(gpu_ctx, model, kw, strategy):
    d = synthetic.small(model, prior=PRIOR_NORMAL, **kw)
    fixed = np.zeros(d.J, np.uint8)
    fixed[[2, 4]] = 1
    want = _oracle_fit(d, conv_type=GRADIENT, tol=1e-7, fixed=fixed)
    got = _gpu_fit(gpu_ctx, d, convergence_type=GRADIENT, tolerance=1e-7, fixed=fixed, strategy=strategy)
    _agree(got, want)
    assert got.beta[2] == 0.0 and got.beta[4] == 0.0


dropin = pytest.mark.skipif(not (os.path.exists(checker.REF_B200_LIB) and checker.reference_available()),
                            reason="reference solver / adapter not built here")


@dropin
@pytest.mark.parametrize("model,kw,fit_kw", [
    (MODEL_LOGISTIC, dict(seed=140), dict(kkt_swindle=True)),
    (MODEL_COX, dict(seed=141, n_strata=4, tie_days=3), dict(kkt_swindle=True)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=142, n_strata=30), dict(algorithm=1)),
    (MODEL_CONDITIONAL_POISSON, dict(seed=143, n_strata=25, prior=PRIOR_NORMAL), dict(algorithm=1)),
])
def test_reference_solver_variants_on_b200(model, kw, fit_kw):
    """The reference's CyclicCoordinateDescent runs the swindle and the MM
    cycle itself, asking the adapter for gradients, MM bounds and xBeta."""
    d = synthetic.small(model, **kw)
    want = checker.ReferenceEngine(d).fit(LANGE, 1e-7, **fit_kw)
    got = checker.ReferenceOnB200Engine(d).fit(LANGE, 1e-7, **fit_kw)
    assert got["flag"] == want["flag"] and got["iterations"] == want["iterations"]
    err = np.max(np.abs(got["beta"] - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
    assert err <= 1e-6
    assert abs(got["loglik"] - want["loglik"]) <= 1e-9 * abs(want["loglik"])


@dropin
@pytest.mark.parametrize("formats", [("sparse", "indicator"), ("sparse", "dense")])
def test_reference_solver_mm_over_the_transpose_product(formats):
    """The reference's MM cycle calls computeXBeta(beta) on the adapter, which
    forms the one-format transpose product as the reference's own
    ModelSpecifics does: the same end, a fit or "Non-increasing!"."""
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=150, n_strata=20, formats=formats,
                        prior=PRIOR_NORMAL, variance=4.0)
    out = []
    for E in (checker.ReferenceEngine, checker.ReferenceOnB200Engine):
        try:
            out.append(E(d).fit(MITTAL, 1e-8, algorithm=1))
        except RuntimeError as ex:
            out.append(str(ex))
    want, got = out
    if isinstance(want, str):
        assert got == want
        return
    assert got["flag"] == want["flag"] and got["iterations"] == want["iterations"]
    err = np.max(np.abs(got["beta"] - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
    assert err <= 1e-6
