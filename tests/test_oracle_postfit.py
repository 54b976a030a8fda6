"""The oracle's calls on a fitted state -- Fisher information, predictive
estimates, predictive log-likelihood -- pinned against the reference engine:
the committed golden fixtures, and the compiled reference where it is built.

Fisher information (ModelSpecifics.hpp:1203-1337) is FP64 sums in the
reference's own order in the restatement, so on the reference's mode it is
compared to 1e-13 relative to the matrix's largest entry; an independent
check rebuilds the unweighted GLM information X' diag(v) X with numpy."""
import numpy as np
import pytest

from ccd_b200 import synthetic
from ccd_b200.data import (MODEL_CONDITIONAL_LOGISTIC, MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON,
                           PRIOR_NORMAL)
from oracle import checker

from .golden_io import case_names, load_case

FISHER_TOL = 1e-13


def _dense(d) -> np.ndarray:
    """The K x J design matrix of a CyclopsData (formats DENSE 0, SPARSE 1,
    INDICATOR 2, INTERCEPT 3)."""
    X = np.zeros((d.K, d.J))
    for j in range(d.J):
        f = int(d.fmt[j])
        if f == 3:
            X[:, j] = 1.0
        elif f == 0:
            X[:, j] = d.vals[d.val_start[j]:d.val_start[j] + d.K]
        else:
            r = d.rows[d.col_start[j]:d.col_start[j + 1]]
            X[r, j] = d.vals[d.val_start[j]:d.val_start[j] + len(r)] if f == 1 else 1.0
    return X


def _fitted(name):
    d, w, want = load_case(name)
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    e.fit(want["conv"], 1e-6)
    return d, w, want, e


@pytest.mark.parametrize("name", case_names())
def test_postfit_calls_match_golden(name):
    d, w, want, e = _fitted(name)
    if "fisher" in want:
        got = e.fisher_information(want["fisher_cols"])
        scale = np.max(np.abs(want["fisher"]))
        assert np.max(np.abs(got - want["fisher"])) <= FISHER_TOL * scale
        assert np.array_equal(got, got.T)
    else:  # a weighted fit: the reference refuses it
        with pytest.raises(checker.FisherRefused):
            e.fisher_information(np.arange(d.J, dtype=np.int32))
    np.testing.assert_allclose(e.predictive_estimates(), want["pred_est"], rtol=1e-13, atol=1e-15)
    assert abs(e.predictive_loglik(want["heldout"]) - want["pred_ll"]) <= 1e-12 * max(1.0, abs(want["pred_ll"]))


def test_fisher_of_a_glm_is_x_weighted_x():
    """Independent of both engines: for LR and Poisson the information is
    X' diag(v) X with v = p(1-p) (LR) or mu (Poisson) at the current xBeta."""
    for model, v_of in ((MODEL_LOGISTIC, lambda xb: np.exp(xb) / (1 + np.exp(xb)) ** 2),
                        (MODEL_POISSON, np.exp)):
        d = synthetic.small(model, seed=61, K=300, P=8, formats=("sparse", "dense", "indicator"),
                            prior=PRIOR_NORMAL)
        e = checker.RestatementEngine(d)
        e.fit(0, 1e-8)
        X = _dense(d)
        v = v_of(e.xbeta())
        want = X.T @ (v[:, None] * X)
        got = e.fisher_information(np.arange(d.J, dtype=np.int32))
        assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))


def test_fisher_subsets_and_repeats_are_entries_of_the_full_matrix():
    d = synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=62, n_strata=30)
    e = checker.RestatementEngine(d)
    e.fit(0, 1e-8)
    full = e.fisher_information(np.arange(d.J, dtype=np.int32))
    sub = np.array([5, 2, 5, 0], np.int32)
    got = e.fisher_information(sub)
    assert np.array_equal(got, full[np.ix_(sub, sub)])


needs_ref = pytest.mark.skipif(not checker.reference_available(),
                               reason="reference engine not built (no reference sources here)")


@needs_ref
@pytest.mark.parametrize("model,kw", [
    (MODEL_LOGISTIC, dict(seed=63, formats=("sparse", "dense", "indicator"))),
    (MODEL_POISSON, dict(seed=64, offset=True, prior=PRIOR_NORMAL)),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=65, n_strata=35, formats=("sparse", "dense", "indicator"))),
    (MODEL_COX, dict(seed=66, n_strata=5, tie_days=2, formats=("sparse", "dense", "indicator"))),
])
def test_fisher_bit_exact_with_reference(model, kw):
    d = synthetic.small(model, **kw)
    cols = np.arange(1 if d.offset_col0 else 0, d.J, dtype=np.int32)
    a, b = checker.ReferenceEngine(d), checker.RestatementEngine(d)
    a.fit(0, 1e-7)
    b.fit(0, 1e-7)
    assert np.array_equal(a.fisher_information(cols), b.fisher_information(cols))
    w = (np.arange(d.K) % 4 != 1).astype(float)
    assert np.array_equal(a.predictive_estimates(w), b.predictive_estimates(w))
    assert a.predictive_loglik(w) == b.predictive_loglik(w)


@needs_ref
def test_reference_variance_is_the_inverse_information():
    """getAsymptoticVariance (CyclicCoordinateDescent.cpp:1249-1269) inverts
    the information of the free columns; with a Normal prior every column is
    kept, so it equals inv(fisher) of all coefficient columns."""
    d = synthetic.small(MODEL_POISSON, seed=67, offset=True, prior=PRIOR_NORMAL, P=6)
    e = checker.ReferenceEngine(d)
    e.fit(0, 1e-8)
    cols = np.arange(1, d.J, dtype=np.int32)
    inv = np.linalg.inv(e.fisher_information(cols))
    for a in range(len(cols)):
        for b in range(len(cols)):
            v = e.asymptotic_variance(int(cols[a]), int(cols[b]))
            assert abs(v - inv[a, b]) <= 1e-9 * np.max(np.abs(inv))
