"""The oracle on edge-case inputs (tests/edge_cases.py), bit for bit against
the reference engine compiled from source: fits under every convergence
criterion, per-coordinate gradients, predictive calls, and the Fisher
information where the fit is unweighted."""
import numpy as np
import pytest

from ccd_b200.data import GRADIENT, LANGE, MITTAL
from oracle import checker

from .edge_cases import cases

pytestmark = pytest.mark.skipif(not checker.reference_available(),
                                reason="reference engine not built (no reference sources here)")

CASES = cases()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL, LANGE])
def test_edge_case_bit_exact(name, conv):
    d, w = CASES[name]
    out = []
    for E in (checker.ReferenceEngine, checker.RestatementEngine):
        e = E(d)
        if w is not None:
            e.set_weights(w)
        gh = [e.grad_hess(j) for j in range(d.J)]
        r = e.fit(conv, 1e-7)
        held = (np.arange(d.K) % 3 == 0).astype(float)
        extra = {"gh": gh, "pred_ll": e.predictive_loglik(held), "pred": e.predictive_estimates()}
        if w is None:
            extra["fisher"] = e.fisher_information(np.arange(d.J, dtype=np.int32))
        out.append((r, extra))
    (a, xa), (b, xb) = out
    assert a["iterations"] == b["iterations"] and a["flag"] == b["flag"]
    assert np.array_equal(a["beta"], b["beta"]) and a["loglik"] == b["loglik"]
    assert xa["gh"] == xb["gh"]
    assert xa["pred_ll"] == xb["pred_ll"] or (np.isnan(xa["pred_ll"]) and np.isnan(xb["pred_ll"]))
    assert np.array_equal(xa["pred"], xb["pred"])
    if "fisher" in xa:
        assert np.array_equal(xa["fisher"], xb["fisher"])
