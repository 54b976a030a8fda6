"""The drop-in, end to end: the reference's own, unchanged
CyclicCoordinateDescent (compiled from the reference sources) driving the B200
engine through B200ModelSpecifics, an AbstractModelSpecifics over the C ABI,
must give the reference CPU engine's fits."""
import os

import numpy as np
import pytest

from ccd_b200 import synthetic
from ccd_b200.data import (GRADIENT, MITTAL, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX, MODEL_LOGISTIC,
                           MODEL_POISSON, PRIOR_NORMAL)
from oracle import checker

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(checker.REF_B200_LIB) and checker.reference_available()),
                                 reason="reference solver / adapter not built here")]


@pytest.mark.parametrize("model,kw,conv", [
    (MODEL_LOGISTIC, dict(seed=40), GRADIENT),
    (MODEL_POISSON, dict(seed=41, offset=True, prior=PRIOR_NORMAL), MITTAL),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=42, n_strata=30), GRADIENT),
    (MODEL_COX, dict(seed=43, n_strata=4, tie_days=3), MITTAL),
])
def test_reference_solver_on_b200_engine(model, kw, conv):
    d = synthetic.small(model, **kw)
    want = checker.ReferenceEngine(d).fit(conv, 1e-6)
    got = checker.ReferenceOnB200Engine(d).fit(conv, 1e-6)
    assert got["flag"] == want["flag"] and got["iterations"] == want["iterations"]
    err = np.max(np.abs(got["beta"] - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
    assert err <= 1e-6
    assert abs(got["loglik"] - want["loglik"]) <= 1e-9 * abs(want["loglik"])


def test_reference_solver_on_b200_with_weights():
    d = synthetic.small(MODEL_LOGISTIC, seed=44, K=400)
    w = (np.arange(d.K) % 7 != 0).astype(float)
    a, b = checker.ReferenceEngine(d), checker.ReferenceOnB200Engine(d)
    a.set_weights(w)
    b.set_weights(w)
    want, got = a.fit(GRADIENT, 1e-6), b.fit(GRADIENT, 1e-6)
    assert got["iterations"] == want["iterations"]
    assert np.max(np.abs(got["beta"] - want["beta"])) <= 1e-6 * max(np.max(np.abs(want["beta"])), 1e-8)


# The fused reference-side path: B200CyclicCoordinateDescent runs each findMode
# of update() as one ccdb_find_mode call; results as the reference's own.
@pytest.mark.parametrize("model,kw,conv,fit_kw", [
    (MODEL_LOGISTIC, dict(seed=40), GRADIENT, {}),
    (MODEL_LOGISTIC, dict(seed=45, K=600, P=30), MITTAL, dict(kkt_swindle=True)),
    (MODEL_POISSON, dict(seed=41, offset=True, prior=PRIOR_NORMAL), MITTAL, {}),
    (MODEL_CONDITIONAL_LOGISTIC, dict(seed=42, n_strata=30), GRADIENT, {}),
    (MODEL_COX, dict(seed=43, n_strata=4, tie_days=3), MITTAL, {}),
    (MODEL_COX, dict(seed=46, n_strata=6, tie_days=2), GRADIENT, dict(algorithm=1)),
])
def test_fused_reference_solver_on_b200(model, kw, conv, fit_kw):
    d = synthetic.small(model, **kw)
    want = checker.ReferenceEngine(d).fit(conv, 1e-6, **fit_kw)
    e = checker.ReferenceOnB200FusedEngine(d)
    got = e.fit(conv, 1e-6, **fit_kw)
    assert e.device_calls() == 1
    assert got["flag"] == want["flag"]
    if not fit_kw.get("kkt_swindle"):
        assert got["iterations"] == want["iterations"]
    err = np.max(np.abs(got["beta"] - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
    assert err <= 1e-6
    assert abs(got["loglik"] - want["loglik"]) <= 1e-9 * abs(want["loglik"])
    # a second update continues from the mode, as the reference's does
    want2 = checker.ReferenceEngine(d)
    want2.fit(conv, 1e-6, **fit_kw)
    w2 = want2.fit(conv, 1e-6, **fit_kw)
    g2 = e.fit(conv, 1e-6, **fit_kw)
    assert e.device_calls() == 2
    assert g2["flag"] == w2["flag"]
    assert np.max(np.abs(g2["beta"] - w2["beta"])) <= 1e-6 * max(np.max(np.abs(w2["beta"])), 1e-8)


def test_fused_reference_solver_with_weights_and_fixed():
    d = synthetic.small(MODEL_LOGISTIC, seed=44, K=400)
    w = (np.arange(d.K) % 7 != 0).astype(float)
    fixed = np.zeros(d.J, np.uint8)
    fixed[2] = 1
    a, b = checker.ReferenceEngine(d), checker.ReferenceOnB200FusedEngine(d)
    a.set_weights(w)
    b.set_weights(w)
    want, got = a.fit(GRADIENT, 1e-6, fixed=fixed), b.fit(GRADIENT, 1e-6, fixed=fixed)
    assert b.device_calls() == 1
    assert got["iterations"] == want["iterations"] and got["flag"] == want["flag"]
    assert np.max(np.abs(got["beta"] - want["beta"])) <= 1e-6 * max(np.max(np.abs(want["beta"])), 1e-8)
    assert got["beta"][2] == 0.0
