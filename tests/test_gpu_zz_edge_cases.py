"""Edge-case inputs (tests/edge_cases.py) on the GPU through the C ABI,
against the oracle (bit-exact with the reference on the same inputs): the
starting gradients, the fit, and the calls on the oracle's mode.  Slowly
converging problems (a column equal to the intercept) may settle a cycle
either side of the oracle's count."""
import numpy as np
import pytest

from ccd_b200 import native
from ccd_b200.data import GRADIENT, MITTAL, MODEL_COX
from oracle import checker

from .edge_cases import cases

pytestmark = pytest.mark.gpu

CASES = cases()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("conv", [GRADIENT, MITTAL])
def test_gpu_edge_case(gpu_ctx, name, conv):
    d, w = CASES[name]
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    gh_want = np.array([e.grad_hess(j) for j in range(d.J)])
    want = e.fit(conv, 1e-7)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    if w is not None:
        f.set_weights(w)
    gh = np.array([f.compute_gradient_and_hessian(j) for j in range(d.J)])
    # 1e-10 as the other per-coordinate tests; 1e-9 for Cox, whose gradient is
    # reassociated through per-group suffix sums
    tol = 1e-9 if d.model_type == MODEL_COX else 1e-10
    np.testing.assert_allclose(gh, gh_want, rtol=tol, atol=tol)
    r = f.find_mode(native.ModeFindingArguments(convergence_type=conv, tolerance=1e-7))
    assert r.return_flag == want["flag"]
    assert abs(r.iterations - want["iterations"]) <= 2
    scale = max(np.max(np.abs(want["beta"])), 1e-8)
    assert np.max(np.abs(r.beta - want["beta"])) <= 1e-6 * scale
    assert abs(r.log_likelihood - want["loglik"]) <= 1e-9 * abs(want["loglik"])
    # calls at the oracle's mode
    g = native.Fit(gpu_ctx, m, d)
    if w is not None:
        g.set_weights(w)
    g.set_beta(want["beta"])
    np.testing.assert_allclose(g.get_predictive_estimates(), e.predictive_estimates(), rtol=1e-12, atol=1e-15)
    held = (np.arange(d.K) % 3 == 0).astype(float)
    pl = e.predictive_loglik(held)
    assert abs(g.get_predictive_log_likelihood(held) - pl) <= 1e-11 * max(1.0, abs(pl))
    if w is None:
        cols = np.arange(d.J, dtype=np.int32)
        fi = e.fisher_information(cols)
        assert np.max(np.abs(g.compute_fisher_information(cols) - fi)) <= 1e-10 * max(1.0, np.max(np.abs(fi)))
