"""The known answers of the reference's own R tests (see
test_known_answers.py) on the GPU, through the C ABI: fits from a cold start
against the independent Newton MLE and the reference's fixtures (weights,
fixed coefficients, every model of the tests), and the Fisher information,
predictions and held-out predictive log-likelihood at the reference's
coefficients."""
import numpy as np
import pytest

from ccd_b200 import native
from ccd_b200.data import GRADIENT

from .golden_io import known_names, load_known
from .newton import newton_mle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", known_names())
def test_gpu_known_answer(gpu_ctx, name):
    d, want = load_known(name)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    if want["weights"] is not None:
        f.set_weights(want["weights"])
    r = f.find_mode(native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-12,
                                                max_iterations=10_000, fixed=want["fixed"]))
    assert r.return_flag == want["flag"]
    # the convergence test at 1e-12 may settle one cycle either side of the reference's
    assert abs(r.iterations - want["iterations"]) <= 2
    beta, ll, _ = newton_mle(d, want["fixed"], want["weights"])
    scale = max(1.0, np.max(np.abs(beta)))
    assert np.max(np.abs(r.beta - beta)) <= 1e-7 * scale
    assert np.max(np.abs(r.beta - want["beta"])) <= 1e-7 * scale
    assert abs(r.log_likelihood - ll) <= 1e-10 * abs(ll)
    # calls on the reference's own mode
    g = native.Fit(gpu_ctx, m, d)
    if want["weights"] is not None:
        g.set_weights(want["weights"])
    g.set_beta(want["beta"])
    if want["fisher"] is not None:
        info = g.compute_fisher_information(want["fisher_cols"])
        assert np.max(np.abs(info - want["fisher"])) <= 1e-10 * max(1.0, np.max(np.abs(want["fisher"])))
    np.testing.assert_allclose(g.get_predictive_estimates(), want["pred_est"], rtol=1e-12, atol=1e-15)
    if want["pred_ll"] is not None:
        got = g.get_predictive_log_likelihood(want["heldout"])
        assert abs(got - want["pred_ll"]) <= 1e-11 * abs(want["pred_ll"])
