"""Profile-likelihood confidence bounds (ccd_b200/inference.py) against the
reference's CcdInterface::profileModel compiled from source, and against an
independent profile computed with the Newton solver.  The host logic -- the
sign-change bracket, Brent's zeroin, the warm-started refits with the profiled
coefficient fixed -- is driven by the oracle here (bit-exact with the
reference engine), so bounds and evaluation counts must agree with the
reference's; the zeroin tolerance (1e-3) bounds the agreement with the exact
profile."""
import numpy as np
import pytest

from ccd_b200 import inference, synthetic
from ccd_b200.data import GRADIENT, MODEL_CONDITIONAL_LOGISTIC, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_NORMAL
from oracle import checker

from .golden_io import load_known
from .newton import design, loglik_grad_hess, newton_mle

needs_ref = pytest.mark.skipif(not checker.reference_available(),
                               reason="reference engine not built (no reference sources here)")


class OracleProfileBackend:
    def __init__(self, engine, conv=GRADIENT, tol=1e-6, max_iter=1000):
        self.e, self.conv, self.tol, self.max_iter = engine, conv, tol, max_iter

    def beta(self):
        return self.e.beta()

    def step(self, j, delta):
        self.e.update_beta(j, delta)

    def refit(self, fixed):
        return self.e.fit(self.conv, self.tol, self.max_iter, fixed=fixed)["flag"]

    def loglik(self):
        return self.e.loglik()

    def restore(self, beta, fixed):
        self.e.set_beta(beta)


def test_zeroin_finds_roots_to_tolerance():
    f = lambda x: x ** 3 - 2.0 * x - 5.0  # root 2.0945514815423265
    r = inference.zeroin(f, 2.0, 3.0, f(2.0), f(3.0), tol=1e-12)
    assert abs(r - 2.0945514815423265) < 1e-11
    g = lambda x: np.cos(x) - x
    r = inference.zeroin(g, 0.0, 1.0, g(0.0), g(1.0), tol=1e-3)
    assert abs(r - 0.7390851332151607) < 1e-3


def test_bracket_doubles_the_step():
    seen = []

    def f(x):
        seen.append(x)
        return 1.0 - x
    x, fx = inference.bracket_sign_change(f, 0.5, 0.5, +1.0)
    assert fx <= 0 and seen == pytest.approx([0.55, 0.6, 0.7, 0.9, 1.3])


@needs_ref
@pytest.mark.parametrize("make,cols,kw", [
    (lambda: load_known("dobson_dense")[0], [0, 1, 2, 3, 4], {}),
    (lambda: synthetic.small(MODEL_LOGISTIC, seed=161, K=300, P=5, prior=PRIOR_NORMAL), [1, 3],
     dict(override_no_regularization=True, include_penalty=True)),
    (lambda: synthetic.small(MODEL_CONDITIONAL_LOGISTIC, seed=162, n_strata=50, K=300, P=4, prior=PRIOR_NORMAL),
     [0, 2], dict(override_no_regularization=True)),
    (lambda: synthetic.small(MODEL_POISSON, seed=163, K=200, P=4, offset=True, prior=PRIOR_NORMAL), [2],
     dict(override_no_regularization=True)),
])
def test_profile_matches_the_reference(make, cols, kw):
    d = make()
    ref = checker.ReferenceEngine(d)
    ref.fit(GRADIENT, 1e-6)
    lo, up, ev = ref.profile(cols, **kw)
    e = checker.RestatementEngine(d)
    e.fit(GRADIENT, 1e-6)
    glo, gup, gev = inference.profile_bounds(OracleProfileBackend(e), d, cols, **kw)
    np.testing.assert_allclose(glo, lo, rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(gup, up, rtol=1e-8, atol=1e-10)
    assert gev.tolist() == ev.tolist()


@needs_ref
def test_regularised_columns_are_refused_like_the_reference():
    d = synthetic.small(MODEL_LOGISTIC, seed=164, K=200, P=4, prior=PRIOR_NORMAL)
    ref = checker.ReferenceEngine(d)
    ref.fit(GRADIENT, 1e-6)
    with pytest.raises(RuntimeError, match="regularized"):
        ref.profile([2])
    e = checker.RestatementEngine(d)
    e.fit(GRADIENT, 1e-6)
    with pytest.raises(ValueError, match="regularized"):
        inference.profile_bounds(OracleProfileBackend(e), d, [2])


def test_dobson_profile_bounds_are_the_exact_profile():
    """test-smallPoisson.R compares confint with glm's profile intervals; here
    the exact profile: the Newton MLE with the coefficient fixed, where
    2 (LL(mode) - LL) = qchisq(0.95, 1), found by bisection."""
    d, _ = load_known("dobson_dense")
    e = checker.RestatementEngine(d)
    e.fit(GRADIENT, 1e-10, max_iter=10_000)
    lo, up, _ = inference.profile_bounds(OracleProfileBackend(e, tol=1e-10, max_iter=10_000), d, [0, 1, 2])
    X = design(d)
    b_hat, ll_hat, _ = newton_mle(d)

    def profile_ll(j, x):
        fixed = np.zeros(d.J, np.uint8)
        fixed[j] = 1
        dd = d
        beta = b_hat.copy()
        beta[j] = x
        free = fixed == 0
        for _ in range(100):  # Newton on the free coefficients
            _, g, H = loglik_grad_hess(dd, X, beta)
            step = np.linalg.solve(-H[np.ix_(free, free)], g[free])
            beta[free] += step
            if np.max(np.abs(step)) < 1e-13:
                break
        return loglik_grad_hess(dd, X, beta)[0]

    for i, j in enumerate([0, 1, 2]):
        for bound, sign in ((up[i], 1.0), (lo[i], -1.0)):
            a, b = b_hat[j], b_hat[j] + sign * 5.0
            for _ in range(80):  # bisection on ll_hat - LL(x) - 1.920729
                m = 0.5 * (a + b)
                if ll_hat - profile_ll(j, m) < inference.CHI2_95_HALF:
                    a = m
                else:
                    b = m
            assert abs(bound - 0.5 * (a + b)) < 2e-3


@needs_ref
@pytest.mark.parametrize("seed", range(40))
def test_profile_random_problems_match_the_reference(seed):
    """Seeded random problems (tests/test_oracle_fuzz.py's generator: every
    model, formats, mixed priors, an offset, weights with zeros): one or two
    columns profiled, with or without the penalty, around the mode of a plain
    fit; bounds, NaN where no sign change was found, and evaluation counts as
    the reference's profileModel."""
    from .test_oracle_fuzz import random_case
    d, w, _ = random_case(seed)
    rng = np.random.default_rng(10_000 + seed)
    first = 1 if d.offset_col0 else 0
    if d.J - first < 1:
        pytest.skip("no coefficient column")
    cols = sorted(rng.choice(np.arange(first, d.J), size=min(2, d.J - first), replace=False).tolist())
    kw = dict(override_no_regularization=True, include_penalty=bool(rng.integers(2)))
    ref = checker.ReferenceEngine(d)
    e = checker.RestatementEngine(d)
    if w is not None:
        ref.set_weights(w)
        e.set_weights(w)
    r = ref.fit(GRADIENT, 1e-6)
    if r["flag"] != 0 or not np.all(np.isfinite(r["beta"])):
        pytest.skip("the plain fit has no finite mode")
    lo, up, ev = ref.profile(cols, **kw)
    e.fit(GRADIENT, 1e-6)
    glo, gup, gev = inference.profile_bounds(OracleProfileBackend(e), d, cols, **kw)
    np.testing.assert_allclose(glo, lo, rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(gup, up, rtol=1e-8, atol=1e-10)
    assert gev.tolist() == ev.tolist()
