"""Seeded random problems (the ones tests/test_oracle_fuzz.py pins the oracle
on, bit for bit against the reference) on the GPU through the C ABI, against
the oracle: random model, column formats, densities, per-column priors, an
offset, weights with zeros, fixed columns, convergence criterion and
algorithm (CCD, KKT swindle, MM).

The device reductions associate differently from the oracle's sequential sums
(1e-10 per coordinate, as the other parity tests), so a fit may settle a cycle
or two either side of the oracle's count; coefficients agree to 1e-6 of their
scale.  Fits the oracle ends without a finite mode (ILLCONDITIONED, NaN) must
end with the same flag."""
import re

import numpy as np
import pytest

from ccd_b200 import native
from oracle import checker

from .test_oracle_fuzz import random_case

pytestmark = pytest.mark.gpu

R_SUCCESS = 0


def _args(fit_kw):
    return native.ModeFindingArguments(convergence_type=fit_kw["conv_type"], tolerance=fit_kw["tol"],
                                       fixed=fit_kw["fixed"], kkt_swindle=fit_kw["kkt_swindle"],
                                       algorithm=fit_kw.get("algorithm", native.ALGORITHM_CCD))


@pytest.mark.parametrize("seed", range(100))
def test_gpu_random_problem(gpu_ctx, seed):
    d, w, fit_kw = random_case(seed)
    e = checker.RestatementEngine(d)
    if w is not None:
        e.set_weights(w)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    if w is not None:
        f.set_weights(w)
    # the starting gradients, every column
    gh_want = np.array([e.grad_hess(j) for j in range(d.J)])
    gh = np.array([f.compute_gradient_and_hessian(j) for j in range(d.J)])
    np.testing.assert_allclose(gh, gh_want, rtol=1e-9, atol=1e-9)
    try:
        want = e.fit(**fit_kw)
    except RuntimeError as ex:  # the MM cycle's "Non-increasing!"
        with pytest.raises(native.CcdbError, match=re.escape(str(ex))):
            f.find_mode(_args(fit_kw))
        return
    r = f.find_mode(_args(fit_kw))
    assert r.return_flag == want["flag"]
    finite = np.all(np.isfinite(want["beta"])) and np.isfinite(want["loglik"])
    if want["flag"] != R_SUCCESS or not finite:
        return
    if not fit_kw["kkt_swindle"]:
        assert abs(r.iterations - want["iterations"]) <= 2
    scale = max(np.max(np.abs(want["beta"])), 1e-8)
    assert np.max(np.abs(r.beta - want["beta"])) <= 1e-6 * scale
    assert abs(r.log_likelihood - want["loglik"]) <= 1e-9 * max(1.0, abs(want["loglik"]))
    # the post-fit calls at the oracle's mode, both sides from beta (an MM fit
    # leaves the reference's own xBeta behind, see the MM product's rule)
    e = checker.RestatementEngine(d)
    g = native.Fit(gpu_ctx, m, d)
    if w is not None:
        e.set_weights(w)
        g.set_weights(w)
    e.set_beta(want["beta"])
    g.set_beta(want["beta"])
    np.testing.assert_allclose(g.get_predictive_estimates(), e.predictive_estimates(), rtol=1e-12, atol=1e-15)
    held = (np.arange(d.K) % 4 == 0).astype(float)
    pl = e.predictive_loglik(held)
    assert abs(g.get_predictive_log_likelihood(held) - pl) <= 1e-11 * max(1.0, abs(pl))
