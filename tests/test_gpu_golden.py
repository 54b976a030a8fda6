"""GPU fits against the committed golden fixtures produced by the reference
engine compiled from source (no CPU checker needed at run time)."""
import numpy as np
import pytest

from ccd_b200 import native

from .golden_io import case_names, load_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", case_names())
def test_gpu_matches_golden(gpu_ctx, name):
    d, w, want = load_case(name)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    if w is not None:
        f.set_weights(w)
    gh = np.array([f.compute_gradient_and_hessian(j) for j in range(d.J)])
    np.testing.assert_allclose(gh, want["gh0"], rtol=1e-9, atol=1e-10)
    f2 = native.Fit(gpu_ctx, m, d)
    if w is not None:
        f2.set_weights(w)
    r = f2.find_mode(native.ModeFindingArguments(convergence_type=want["conv"]))
    assert r.iterations == want["iterations"] and r.return_flag == want["flag"]
    err = np.max(np.abs(r.beta - want["beta"])) / max(np.max(np.abs(want["beta"])), 1e-8)
    assert err <= 1e-6
    assert abs(r.log_likelihood - want["loglik"]) <= 1e-9 * abs(want["loglik"])
