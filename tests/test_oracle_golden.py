"""The CPU oracle (plain-C restatement) pinned against the reference engine:
golden fixtures produced by the reference compiled from source, plus direct
comparisons with the reference where it is built."""
import hashlib

import numpy as np
import pytest

from ccd_b200 import synthetic
from ccd_b200.data import (GRADIENT, LANGE, MITTAL, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX,
                           MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL, cox_groups)
from oracle import checker

from .golden_io import case_names, index, load_case


@pytest.mark.parametrize("name", case_names())
def test_restatement_matches_golden(name):
    d, w, want = load_case(name)
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    gh = np.array([e.grad_hess(j) for j in range(d.J)])
    np.testing.assert_allclose(gh, want["gh0"], rtol=1e-13, atol=1e-13)
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    r = e.fit(want["conv"], 1e-6)
    assert r["iterations"] == want["iterations"] and r["flag"] == want["flag"]
    np.testing.assert_allclose(r["beta"], want["beta"], rtol=1e-12, atol=1e-14)
    assert abs(r["loglik"] - want["loglik"]) <= 1e-12 * abs(want["loglik"])


def test_logistic_l1_benchmark_golden():
    ix = index()["logistic_l1_10000x1000"]
    d = synthetic.logistic_l1(seed=ix["seed"])
    h = hashlib.sha256()
    for a in (d.y, d.col_start, d.rows, d.fmt):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == ix["input_sha256"], "synthetic generator drifted"
    import os
    from .golden_io import GOLDEN
    z = np.load(os.path.join(GOLDEN, "logistic_l1_10000x1000.npz"))
    r = checker.RestatementEngine(d).fit(MITTAL, 1e-6)
    assert r["iterations"] == int(z["iterations"]) and r["flag"] == int(z["flag"])
    np.testing.assert_allclose(r["beta"], z["beta"], rtol=1e-12, atol=1e-14)


needs_ref = pytest.mark.skipif(not checker.reference_available(),
                               reason="reference engine not built (no reference sources here)")


@needs_ref
@pytest.mark.parametrize("model", [MODEL_LOGISTIC, MODEL_POISSON, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX])
@pytest.mark.parametrize("seed", range(4))
def test_restatement_bit_exact_with_reference(model, seed):
    kw = dict(seed=100 + seed, prior=PRIOR_LAPLACE if seed % 2 else PRIOR_NORMAL,
              offset=(model == MODEL_POISSON and seed % 2 == 0))
    d = synthetic.small(model, **kw)
    conv = [GRADIENT, MITTAL, LANGE, GRADIENT][seed]
    w = None
    if seed == 3:
        w = (np.random.default_rng(seed).random(d.K) > 0.2).astype(float)
    out = []
    for E in (checker.ReferenceEngine, checker.RestatementEngine):
        e = E(d)
        if w is not None:
            e.set_weights(w)
        out.append(e.fit(conv, 1e-6))
    a, b = out
    assert a["iterations"] == b["iterations"] and a["flag"] == b["flag"]
    assert np.array_equal(a["beta"], b["beta"])
    assert a["loglik"] == b["loglik"]


@needs_ref
def test_per_coordinate_traces_match_reference():
    d = synthetic.small(MODEL_COX, seed=7, n_strata=5, tie_days=3)
    ref, port = checker.ReferenceEngine(d), checker.RestatementEngine(d)
    rng = np.random.default_rng(0)
    for j in list(range(d.J)) * 2:
        assert ref.grad_hess(j) == port.grad_hess(j)
        delta = float(rng.normal(0, 0.2))
        ref.update_beta(j, delta)
        port.update_beta(j, delta)
    assert np.array_equal(ref.xbeta(), port.xbeta())
    assert ref.loglik() == port.loglik()


@pytest.mark.parametrize("weighted", [False, True])
def test_cox_grouping_matches_restatement(weighted):
    """Risk-set tie groups (setPidForAccumulation) are integer work: bit-exact."""
    import ctypes as C
    d = synthetic.small(MODEL_COX, seed=8, K=700, n_strata=9, tie_days=2)
    w = (np.random.default_rng(2).random(d.K) > 0.3).astype(float) if weighted else None
    grp, acc_reset, N = cox_groups(d.stratum, d.time, d.y, w)
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    lib = e.lib()
    lib.orc_cox_groups.argtypes = [C.c_void_p] * 4
    g2 = np.zeros(d.K, np.int32)
    r2 = np.zeros(d.K + 2, np.int32)
    nr = C.c_int()
    N2 = lib.orc_cox_groups(e.h, g2.ctypes.data_as(C.c_void_p), r2.ctypes.data_as(C.c_void_p), C.byref(nr))
    assert N == N2
    assert np.array_equal(grp, g2)
    assert np.array_equal(acc_reset, r2[:nr.value])


def test_edge_empty_column_and_all_zero_weights_stratum():
    """An empty indicator column gives (g, h) = (0, 0) (ModelSpecifics.hpp:720-723)."""
    from ccd_b200.data import INDICATOR, INTERCEPT, CyclopsData, build_columns
    K = 50
    rng = np.random.default_rng(1)
    cols = [(None, None), (np.array([], np.int32), None), (np.sort(rng.choice(K, 10, replace=False)).astype(np.int32), None)]
    cs, r, vs, v, fm = build_columns(K, cols, [INTERCEPT, INDICATOR, INDICATOR])
    y = (rng.random(K) < 0.4).astype(float)
    d = CyclopsData(MODEL_LOGISTIC, y, cs, r, vs, v, fm, np.array([0, 1, 1], np.int32), np.ones(3))
    e = checker.RestatementEngine(d)
    assert e.grad_hess(1) == (0.0, 0.0)
    res = e.fit(GRADIENT, 1e-6)
    assert res["beta"][1] == 0.0
