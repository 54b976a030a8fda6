"""Mode-finding variants of CyclicCoordinateDescent::update in the oracle,
pinned bit for bit against the reference compiled from source:

* the KKT swindle (CyclicCoordinateDescent.cpp:636-826): Laplace columns start
  inactive and join the active set when their |gradient| exceeds lambda;
* the MM algorithm (AlgorithmType::MM, .cpp:957-1001, 1354-1391;
  ModelSpecifics.hpp:776-889): every coordinate's step from one
  all-coordinate (g, h), then xBeta from beta;
* fixed coefficients (setFixedBeta).

The reference's MM reads out of bounds on unstratified data (initializeMM's
per-stratum reduction, ModelData.h:606-660), so it is run here only on the
stratified models; the oracle refuses the others."""
import numpy as np
import pytest

from ccd_b200 import synthetic
from ccd_b200.data import (GRADIENT, LANGE, MITTAL, MODEL_CONDITIONAL_LOGISTIC, MODEL_CONDITIONAL_POISSON,
                           MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL)
from oracle import checker

from .test_oracle_postfit import _dense

needs_ref = pytest.mark.skipif(not checker.reference_available(),
                               reason="reference engine not built (no reference sources here)")

CASES = [
    (MODEL_LOGISTIC, dict(seed=120, P=20)),
    (MODEL_POISSON, dict(seed=121, offset=True)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=122, n_strata=40)),
    (MODEL_CONDITIONAL_POISSON, dict(seed=123, n_strata=30)),
    (MODEL_COX, dict(seed=124, n_strata=6, tie_days=3)),
]
STRATIFIED = [c for c in CASES if c[0] in (MODEL_CONDITIONAL_LOGISTIC, MODEL_CONDITIONAL_POISSON, MODEL_COX)]


def _both(d, w=None, **fit_kw):
    out = []
    for E in (checker.ReferenceEngine, checker.RestatementEngine):
        e = E(d)
        if w is not None:
            e.set_weights(w)
        out.append(e.fit(**fit_kw))
    return out


def _same(a, b):
    assert a["iterations"] == b["iterations"] and a["flag"] == b["flag"]
    assert np.array_equal(a["beta"], b["beta"])
    assert a["loglik"] == b["loglik"]


@needs_ref
@pytest.mark.parametrize("model,kw", CASES)
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL, LANGE])
def test_kkt_swindle_bit_exact(model, kw, conv):
    d = synthetic.small(model, **kw)
    a, b = _both(d, conv_type=conv, tol=1e-7, kkt_swindle=True)
    _same(a, b)


@needs_ref
def test_kkt_swindle_weighted_with_fixed_and_mixed_priors():
    d = synthetic.small(MODEL_LOGISTIC, seed=125, P=16)
    d.prior_type[3] = PRIOR_NORMAL  # a non-Laplace column starts active
    w = (np.arange(d.K) % 6 != 0).astype(float)
    fixed = np.zeros(d.J, np.uint8)
    fixed[5] = 1
    a, b = _both(d, w, conv_type=GRADIENT, tol=1e-7, kkt_swindle=True, fixed=fixed)
    _same(a, b)
    assert a["beta"][5] == 0.0


@needs_ref
def test_kkt_swindle_limited_passes():
    """maxIterations also bounds the number of swindle passes (MAX_ITERATIONS)."""
    d = synthetic.small(MODEL_LOGISTIC, seed=126, P=20, variance=100.0)
    a, b = _both(d, conv_type=GRADIENT, tol=1e-8, max_iter=2, kkt_swindle=True)
    _same(a, b)


@needs_ref
@pytest.mark.parametrize("model,kw", STRATIFIED)
@pytest.mark.parametrize("prior", [PRIOR_LAPLACE, PRIOR_NORMAL])
def test_mm_bit_exact(model, kw, prior):
    d = synthetic.small(model, prior=prior, **kw)
    a, b = _both(d, conv_type=MITTAL, tol=1e-8, algorithm=1)
    _same(a, b)


@needs_ref
@pytest.mark.parametrize("model,kw", STRATIFIED[:2])
def test_mm_with_kkt_swindle_bit_exact(model, kw):
    d = synthetic.small(model, **kw)
    a, b = _both(d, conv_type=GRADIENT, tol=1e-7, algorithm=1, kkt_swindle=True)
    _same(a, b)


@needs_ref
@pytest.mark.parametrize("formats", [("sparse", "indicator"), ("sparse", "dense"), ("sparse",),
                                     ("indicator", "dense", "sparse")])
@pytest.mark.parametrize("model", [MODEL_CONDITIONAL_LOGISTIC, MODEL_COX])
def test_mm_product_follows_the_transpose_format(model, formats):
    """The MM cycle's xBeta runs over hX.transpose(), whose rows take one
    format (CompressedDataMatrix.cpp:151-209): with INDICATOR and SPARSE columns
    and no DENSE one the transpose is INDICATOR and a SPARSE entry counts 1.
    The restatement follows the same rule, bit for bit, under every mix; the
    inconsistent product often ends the reference's fit with "Non-increasing!",
    and then the restatement's too."""
    d = synthetic.small(model, seed=150, n_strata=20, formats=formats, prior=PRIOR_NORMAL, variance=4.0)
    out = []
    for E in (checker.ReferenceEngine, checker.RestatementEngine):
        try:
            out.append(E(d).fit(MITTAL, 1e-8, algorithm=1))
        except RuntimeError as ex:
            out.append(str(ex))
    if isinstance(out[0], str) or isinstance(out[1], str):
        assert out[0] == out[1]
    else:
        _same(*out)


def test_mm_product_counts_sparse_entries_as_one_without_dense_columns():
    """The same rule shown on the restatement alone: after one MM cycle on a
    SPARSE + INDICATOR matrix the state's xBeta is X' beta with every non-zero
    entry of X' equal to 1; with a DENSE column added it is X beta."""
    for formats, unit in ((("sparse", "indicator"), True), (("sparse", "indicator", "dense"), False)):
        d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=151, n_strata=15, formats=formats,
                            prior=PRIOR_NORMAL, variance=4.0)
        e = checker.RestatementEngine(d)
        r = e.fit(MITTAL, 1e-8, max_iter=1, algorithm=1)
        X = _dense(d)
        if unit:
            X = (X != 0).astype(float)
        np.testing.assert_allclose(e.xbeta(), X @ r["beta"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("model", [MODEL_LOGISTIC, MODEL_POISSON])
def test_mm_refused_without_strata(model):
    d = synthetic.small(model, seed=127, offset=(model == MODEL_POISSON))
    with pytest.raises(RuntimeError, match="stratified|Not model-specific"):
        checker.RestatementEngine(d).fit(MITTAL, 1e-6, algorithm=1)


@needs_ref
@pytest.mark.parametrize("model,kw", CASES)
def test_fixed_coefficients_bit_exact(model, kw):
    d = synthetic.small(model, **kw)
    fixed = np.zeros(d.J, np.uint8)
    fixed[[2, 4]] = 1
    a, b = _both(d, conv_type=GRADIENT, tol=1e-7, fixed=fixed)
    _same(a, b)
    assert a["beta"][2] == 0.0 and a["beta"][4] == 0.0
