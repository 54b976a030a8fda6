"""Seeded random problems (the ones tests/test_oracle_fuzz.py pins the oracle
on, bit for bit against the reference) on the GPU through the C ABI, against
the oracle: random model, column formats, densities, per-column priors, an
offset, weights with zeros, fixed columns, convergence criterion and
algorithm (CCD, KKT swindle, MM).

A fit must end with the oracle's return flag and iteration count, its
coefficients within 1e-6 of their scale and its log-likelihood within 1e-9.

One exception, checked rather than assumed: a problem whose result is decided
by rounding.  The device sums a column in a fixed tree order and uses CUDA's
exp; the reference sums serially and uses glibc's exp, which is itself not
correctly rounded on every argument.  Where a fit drives a coefficient to
infinity (complete or quasi-complete separation), its last cycles see
gradients and Hessians that are rounding noise, and the cycle it stops at and
the coefficient it stops with follow that noise.  The test detects such a
problem by re-running the oracle with exp moved by one unit in the last place
on a seeded fifth of its arguments (three patterns): when those runs
themselves leave the tolerances above, the exact iteration count and the
diverging coefficients are not a property of the problem.  There the GPU must
still end SUCCESS or ILLCONDITIONED and match every coefficient on which all
oracle runs agree.  Of seeds 0-99, seed 25 is such a problem (logistic,
KKT swindle, no prior on column 3, which separates its two rows): the oracle
stops after 49 cycles with beta_3 = 92.57, its three perturbed runs after 47,
50 and 52 cycles with beta_3 between 91.5 and 94.2; the other coefficients
agree to 1e-8."""
import re

import numpy as np
import pytest

from ccd_b200 import native
from oracle import checker

from .test_oracle_fuzz import random_case

pytestmark = pytest.mark.gpu

R_SUCCESS, R_ILLCONDITIONED = 0, 3
PERTURBATION_ONE_IN = 10
PERTURBATION_SALTS = (1, 2, 3)


def _args(fit_kw):
    return native.ModeFindingArguments(convergence_type=fit_kw["conv_type"], tolerance=fit_kw["tol"],
                                       fixed=fit_kw["fixed"], kkt_swindle=fit_kw["kkt_swindle"],
                                       algorithm=fit_kw.get("algorithm", native.ALGORITHM_CCD))


def _agree(a, b, check_iterations: bool) -> bool:
    """Two fit results within the parity tolerances."""
    if a["flag"] != b["flag"]:
        return False
    if check_iterations and a["iterations"] != b["iterations"]:
        return False
    fa = np.all(np.isfinite(a["beta"])) and np.isfinite(a["loglik"])
    fb = np.all(np.isfinite(b["beta"])) and np.isfinite(b["loglik"])
    if a["flag"] != R_SUCCESS or not (fa and fb):
        return fa == fb
    scale = max(np.max(np.abs(a["beta"])), 1e-8)
    return (np.max(np.abs(a["beta"] - b["beta"])) <= 1e-6 * scale
            and abs(a["loglik"] - b["loglik"]) <= 1e-9 * max(1.0, abs(a["loglik"])))


def _perturbed_runs(d, w, fit_kw):
    out = []
    try:
        for salt in PERTURBATION_SALTS:
            checker.RestatementEngine.set_exp_perturbation(PERTURBATION_ONE_IN, salt)
            e = checker.RestatementEngine(d)
            if w is not None:
                e.set_weights(w)
            out.append(e.fit(**fit_kw))
    finally:
        checker.RestatementEngine.set_exp_perturbation(0)
    return out


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
    got = {"beta": r.beta, "loglik": r.log_likelihood, "iterations": r.iterations, "flag": r.return_flag}
    # a swindle's count is that of its last findMode, which may run no cycle at all
    check_iterations = not fit_kw["kkt_swindle"]
    if not _agree(want, got, check_iterations):
        runs = _perturbed_runs(d, w, fit_kw)
        decided_by_rounding = any(not _agree(want, p, True) for p in runs)
        assert decided_by_rounding, (seed, want, got)
        # the coefficients every oracle run agrees on
        allb = np.array([want["beta"]] + [p["beta"] for p in runs])
        scale = max(np.max(np.abs(want["beta"])), 1e-8)
        stable = np.all(np.abs(allb - want["beta"]) <= 1e-6 * scale, axis=0)
        assert r.return_flag in (R_SUCCESS, R_ILLCONDITIONED)
        assert np.all(np.isfinite(r.beta[stable]))
        assert np.max(np.abs(r.beta[stable] - want["beta"][stable])) <= 1e-6 * scale
        return
    if want["flag"] != R_SUCCESS or not np.all(np.isfinite(want["beta"])):
        return
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
