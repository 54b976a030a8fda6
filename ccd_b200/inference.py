"""Asymptotic standard errors, covariance and profile-likelihood confidence
bounds of a fitted model.

Mirrors the reference's R-level post-fit calls: ``getSEs`` (R/ModelFit.R:730-741)
and ``vcov.cyclopsFit`` (R/ModelFit.R:1005-1016) both take the Fisher
information of the chosen columns (``.cyclopsGetFisherInformation``, computed
here on the GPU by ``Fit.compute_fisher_information``) and invert it on the
host, as R's ``solve`` does.  The inversion is of an n x n matrix over the
requested columns; the O(nnz) work is the Fisher information itself.

Profile-likelihood bounds follow CcdInterface::profileModel
(CcdInterface.cpp:223-260, 262-525): for each column, first the upper then the
lower bound, each found by widening a step until the profile objective
LL(beta_j fixed, others refitted) + threshold - LL(mode) changes sign
(RZeroIn::bracketSignChange, utils/RZeroIn.h) and then Brent's zeroin inside
the bracket (tolerance 1e-3).  Every evaluation refits on the device, warm
started from the previous evaluation's coefficients, as the reference does.
"""
from __future__ import annotations

import dataclasses
import math
import warnings
from typing import Callable, Optional, Sequence

import numpy as np


def covariate_columns(fit) -> np.ndarray:
    """All coefficient columns of the fit: every column but the offset (which
    the reference holds outside the coefficients)."""
    first = 1 if fit.d.offset_col0 else 0
    return np.arange(first, fit.d.J, dtype=np.int32)


def vcov(fit, columns: Optional[Sequence[int]] = None) -> np.ndarray:
    """Inverse of the Fisher information over `columns` (default: every
    coefficient column), vcov.cyclopsFit."""
    cols = covariate_columns(fit) if columns is None else np.asarray(columns, dtype=np.int32)
    return np.linalg.inv(fit.compute_fisher_information(cols))


def standard_errors(fit, columns: Optional[Sequence[int]] = None) -> np.ndarray:
    """sqrt(diag(solve(Fisher information))) over `columns`, getSEs.  As the
    reference warns, the errors are only valid when every coefficient is
    included."""
    all_cols = covariate_columns(fit)
    cols = all_cols if columns is None else np.asarray(columns, dtype=np.int32)
    if len(cols) != len(all_cols):
        warnings.warn("Asymptotic standard errors are only valid if computed for all covariates "
                      "simultaneously")
    return np.sqrt(np.diag(np.linalg.inv(fit.compute_fisher_information(cols))))


# ---------------------------------------------------------------- profile likelihood
EPSILON = 2.220446049250313e-16  # DBL_EPSILON
CHI2_95_HALF = 1.920729  # qchisq(0.95, 1) / 2, the reference's default threshold


def zeroin(f: Callable[[float], float], ax: float, bx: float, fa: float, fb: float,
           tol: float = 1e-3, maxit: int = 1000) -> float:
    """Brent's root finder (zeroin: bisection combined with linear or inverse
    quadratic interpolation; Forsythe, Malcolm and Moler, Computer Methods for
    Mathematical Computations, 1977), started from the bracket [ax, bx] whose
    function values are known, as RZeroIn::getRoot runs it.  Accuracy
    4 * EPSILON * |x| + tol."""
    a, b, c = ax, bx, ax
    fc = fa
    if fa == 0.0:
        return a
    if fb == 0.0:
        return b
    for _ in range(maxit + 1):
        prev_step = b - a
        if abs(fc) < abs(fb):  # keep b the best estimate
            a, b, c = b, c, b
            fa, fb, fc = fb, fc, fb
        tol_act = 2.0 * EPSILON * abs(b) + tol / 2.0
        new_step = (c - b) / 2.0
        if abs(new_step) <= tol_act or fb == 0.0:
            return b
        if abs(prev_step) >= tol_act and abs(fa) > abs(fb):
            cb = c - b
            if a == c:  # two points: secant
                t1 = fb / fa
                p = cb * t1
                q = 1.0 - t1
            else:  # three points: inverse quadratic interpolation
                q = fa / fc
                t1 = fb / fc
                t2 = fb / fa
                p = t2 * (cb * q * (q - t1) - (b - a) * (t1 - 1.0))
                q = (q - 1.0) * (t1 - 1.0) * (t2 - 1.0)
            if p > 0.0:
                q = -q
            else:
                p = -p
            if p < (0.75 * cb * q - abs(tol_act * q) / 2.0) and p < abs(prev_step * q / 2.0):
                new_step = p / q
        if abs(new_step) < tol_act:  # at least the tolerance
            new_step = tol_act if new_step > 0.0 else -tol_act
        a, fa = b, fb
        b += new_step
        fb = f(b)
        if (fb > 0.0 and fc > 0.0) or (fb < 0.0 and fc < 0.0):
            c, fc = a, fa
    return b


def bracket_sign_change(f: Callable[[float], float], x0: float, f0: float, direction: float):
    """Step from x0 in `direction` by max(|x0|, 0.01) x 0.1, 0.2, 0.4, ... until
    f <= 0 (RZeroIn::bracketSignChange): (x, f(x)); f is NaN when 21 steps did
    not change the sign or f itself was NaN."""
    displacement = max(abs(x0), 0.01)
    multiplier = 0.1
    x1, f1 = x0, f0
    steps = 0
    while f1 > 0:
        x1 = x0 + direction * displacement * multiplier
        f1 = f(x1)
        if f1 != f1:
            return x1, f1
        if steps > 20:
            return x1, float("nan")
        steps += 1
        multiplier *= 2.0
    return x1, f1


def log_prior(beta, prior_type, prior_var) -> float:
    """Joint log density of the coefficients (priors/JointPrior.h:121-128;
    Laplace priors/CovariatePrior.h:220-224, Normal :404-408)."""
    total = 0.0
    for b, t, v in zip(beta, prior_type, prior_var):
        if t == 1:
            lam = math.sqrt(2.0 / v)
            total += math.log(0.5 * lam) - lam * abs(b)
        elif t == 2:
            total += -0.5 * math.log(2.0 * math.pi * v) - 0.5 * b * b / v
    return total


class NativeProfileBackend:
    """The calls a profile needs, on a native.Fit at its mode."""

    def __init__(self, fit, args=None):
        from . import native
        self.fit = fit
        self.args = args or native.ModeFindingArguments()

    def beta(self) -> np.ndarray:
        return self.fit.get_beta()

    def step(self, j: int, delta: float) -> None:
        self.fit.update_xbeta(j, delta)

    def refit(self, fixed: np.ndarray) -> int:
        return self.fit.find_mode(dataclasses.replace(self.args, fixed=fixed)).return_flag

    def loglik(self) -> float:
        return self.fit.get_log_likelihood()

    def restore(self, beta: np.ndarray, fixed: np.ndarray) -> None:
        self.fit.set_beta(beta)
        self.fit.set_fixed(fixed)


def profile_bounds(backend, d, columns: Sequence[int], threshold: float = CHI2_95_HALF,
                   include_penalty: bool = False, override_no_regularization: bool = False,
                   base_fixed: Optional[np.ndarray] = None):
    """Profile-likelihood bounds (lower, upper, evaluations per column) around
    the backend's current mode, as CcdInterface::profileModel computes them
    with one thread; NaN where no sign change was found.  A regularised column
    is refused unless `override_no_regularization` (its estimate is shrunk)."""
    cols = [int(j) for j in columns]
    for j in cols:
        if not override_no_regularization and int(d.prior_type[j]) != 0:
            raise ValueError(f"Variable {j + 1} is regularized.")
    base = np.zeros(d.J, np.uint8) if base_fixed is None else np.asarray(base_fixed, np.uint8).copy()
    if d.offset_col0:
        base[0] = 1
    x0s = backend.beta().copy()
    mode = backend.loglik()
    if include_penalty:
        mode += log_prior(x0s, d.prior_type, d.prior_var)
    lower, upper, evals = np.full(len(cols), np.nan), np.full(len(cols), np.nan), np.zeros(len(cols), int)
    for i, j in enumerate(cols):
        for direction in (1.0, -1.0):
            count = [0]

            def objective(x, j=j, count=count):
                count[0] += 1
                backend.step(j, x - backend.beta()[j])
                fixed = base.copy()
                fixed[j] = 1
                backend.refit(fixed)
                y = backend.loglik() + threshold - mode
                if include_penalty:
                    y += log_prior(backend.beta(), d.prior_type, d.prior_var)
                return y

            x0 = float(x0s[j])
            x1, f1 = bracket_sign_change(objective, x0, threshold, direction)
            if f1 != f1:
                pt = float("nan")
            elif x1 < x0:
                pt = zeroin(objective, x1, x0, f1, threshold)
            else:
                pt = zeroin(objective, x0, x1, threshold, f1)
            if direction > 0:
                upper[i] = pt
            else:
                lower[i] = pt
            evals[i] += count[0]
    backend.restore(x0s, base)
    return lower, upper, evals
