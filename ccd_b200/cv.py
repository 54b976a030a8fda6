"""Cross-validation drivers over the batched engine: grid search and the
default auto search, then the refit at the selected prior variance.

The reference runs one fit per (fold, variance) task on host threads
(drivers/AbstractCrossValidationDriver.cpp:131-240); here every fold of a
variance -- or, for the grid, every (fold, variance) pair -- is one
`ccdb_batch_find_mode` launch.  Per task the reference keeps the predictive
log-likelihood of the held-out fold when the fit succeeded and NaN otherwise
(:200-232), averages the non-NaN values (computePointEstimate, :250-261) and
measures their spread (computeStDev, :263-276).

* Grid search (drivers/GridSearchCrossValidationDriver.cpp): log-uniform grid
  (computeGridPoint, :37-47), value = point estimate / (foldToCompute / fold),
  first maximum wins (findMax, :234-244).
* Auto search (drivers/AutoSearchCrossValidationDriver.cpp:68-163): starting
  at the given variance or the normal-based default (ModelData.cpp:716-720),
  a `UniModalSearch(10, 0.01, log 1.5)` proposes the next variance from the
  (variance, mean, stdev) history (utils/HParSearch.cpp:66-115), at most 50
  steps.
* Refit (resetForOptimal, AbstractCrossValidationDriver.cpp:31-42): all rows
  weighted 1, the selected variance, cold start.

Instances start cold (the reference's resetCoefficients = TRUE); its default
warm start depends on which thread ran which task before, so it has no fixed
batched counterpart.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .data import DENSE, INTERCEPT, PRIOR_NONE, CyclopsData

SUCCESS = 0


def normal_based_default_var(d: CyclopsData) -> float:
    """Sum of squared entries over the variable columns / their number / rows
    (ModelData::getNormalBasedDefaultVar; the offset and intercept are not
    variable columns)."""
    total, n_var = 0.0, 0
    for j in range(d.J):
        if d.offset_col0 and j == 0:
            continue
        f = int(d.fmt[j])
        if f == INTERCEPT:
            continue
        n_var += 1
        vals = d.vals[d.val_start[j]:d.val_start[j + 1]]
        if f == DENSE:
            total += float(np.sum(vals * vals))
        elif vals.size:  # SPARSE
            total += float(np.sum(vals * vals))
        else:  # INDICATOR: each entry is 1
            total += float(d.col_start[j + 1] - d.col_start[j])
    return total / n_var / d.K


def point_estimate(values) -> float:
    """Mean of the non-NaN values, summed in order (computePointEstimate,
    AbstractCrossValidationDriver.cpp:250-261)."""
    total, count = 0.0, 0
    for x in values:
        x = float(x)
        if x == x:
            total += x
            count += 1
    return total / count if count else float("nan")


def st_dev(values, mean: float) -> float:
    """sqrt(mean of squares - mean^2) over the non-NaN values, summed in order
    (computeStDev, AbstractCrossValidationDriver.cpp:263-276)."""
    inner, count = 0.0, 0
    for x in values:
        x = float(x)
        if x == x:
            inner += x * x
            count += 1
    return math.sqrt(inner / count - mean * mean) if count else float("nan")


def quadratic_log_fit(history: dict):
    """Weighted least squares of y on (1, log x, log^2 x), weight 1/stdev
    (100 / the smallest positive stdev where a stdev is 0); QuadrLogFit,
    utils/HParSearch.cpp:13-52."""
    xs = sorted(history)
    pos = [history[x][1] for x in xs if history[x][1] > 0]
    zero_w = 100.0 / min(pos) if pos else 1.0
    X = np.array([[1.0, math.log(x), math.log(x) ** 2] for x in xs])
    W = np.array([1.0 / history[x][1] if history[x][1] > 0 else zero_w for x in xs])
    Y = np.array([history[x][0] for x in xs])
    XtW = X.T * W
    return np.linalg.solve(XtW @ X, XtW @ Y)


class UniModalSearch:
    """Next hyperparameter from the (x, mean, stdev) history
    (utils/HParSearch.h:25-69, HParSearch.cpp:66-115)."""

    def __init__(self, stdstep: float = 100.0, stop_by_y: float = 0.01, stop_by_x: float = math.log(1.5),
                 first_cut: float = 1.0):
        self.stdstep, self.stop_by_y, self.stop_by_x, self.first_cut = stdstep, stop_by_y, stop_by_x, first_cut
        self.history: dict = {}
        self.best: Optional[float] = None

    def tried(self, x: float, y: float, sd: float = 0.0) -> None:
        self.history[x] = (y, sd)
        if len(self.history) == 1 or y > self.history[self.best][0]:
            self.best = x

    def step(self):
        """(continue?, next x, expected y)."""
        h = self.history
        xs = sorted(h)
        if not xs:
            return True, 1.0, 0.0
        if len(xs) == 1:
            x = xs[0]
            return True, (x * self.stdstep if x < self.first_cut else x / self.stdstep), 0.0
        if len(xs) == 2:
            if h[xs[0]][0] > h[xs[-1]][0]:
                return True, xs[0] / self.stdstep, 0.0
            return True, xs[-1] * self.stdstep, 0.0
        b = self.best
        if xs[0] == b:  # maximum at the left end: move left
            cont = b > math.ulp(0.0)  # the smallest subnormal: 0 and NaN stop
            return (True, b / self.stdstep, 0.0) if cont else (False, b / self.stdstep, h[b][0])
        if xs[-1] == b:  # maximum at the right end: move right
            cont = b < math.inf
            return (True, b * self.stdstep, 0.0) if cont else (False, b * self.stdstep, h[b][0])
        c0, c1, c2 = quadratic_log_fit(h)  # bracketed
        log_argmax = -c1 / c2 / 2
        expected = -c1 * c1 / c2 / 4 + c0
        maxval = h[b][0]
        cont = True
        if maxval == 0:
            cont = False
        elif (expected - maxval) / abs(maxval) < self.stop_by_y:
            cont = False
        elif abs(log_argmax - math.log(b)) < self.stop_by_x:
            cont = False
        return cont, math.exp(log_argmax), expected


@dataclass
class CVResult:
    variance: float
    value: float
    tried: List[tuple] = field(default_factory=list)  # (variance, mean pred LL, stdev)
    fits: int = 0
    device_seconds: float = 0.0


def _fold_values(fit, variance: float, n_folds: int, row_fold, args):
    var = np.full(n_folds, float(variance))
    hold = np.arange(n_folds, dtype=np.int32)
    _, res, secs = fit.batch_find_mode(var, hold, row_fold, args)
    pred = [r["pred_loglik"] if r["flag"] == SUCCESS else float("nan") for r in res]
    return pred, secs


def auto_search(fit, d: CyclopsData, row_fold, n_folds: int, args=None, starting_variance: float = -1.0,
                max_steps: int = 50) -> CVResult:
    """The reference's default cross-validation (cvType "auto") for one
    hyperparameter: `fit` is a native.Fit over the data (FP64 or mixed)."""
    v = starting_variance if starting_variance > 0 else normal_based_default_var(d)
    search = UniModalSearch(10.0, 0.01, math.log(1.5))
    out = CVResult(v, float("nan"))
    for step in range(max_steps):
        pred, secs = _fold_values(fit, v, n_folds, row_fold, args)
        mean = point_estimate(pred)
        sd = st_dev(pred, mean)
        out.tried.append((v, mean, sd))
        out.fits += n_folds
        out.device_seconds += secs
        search.tried(v, mean, sd)
        cont, nxt, expected = search.step()
        v, out.value = nxt, expected
        if not cont:
            break
    out.variance = v
    return out


def grid_points(lower: float, upper: float, steps: int) -> np.ndarray:
    if steps == 1:
        return np.array([upper])
    size = (math.log(upper) - math.log(lower)) / (steps - 1)
    return np.array([math.exp(math.log(lower) + s * size) for s in range(steps)])


def grid_search(fit, row_fold, n_folds: int, lower: float = 0.01, upper: float = 20.0, steps: int = 10,
                args=None) -> CVResult:
    """Every (fold, variance) of the grid in one launch; the first maximum of
    the mean held-out predictive log-likelihood wins."""
    pts = grid_points(lower, upper, steps)
    var = np.repeat(pts, n_folds)
    hold = np.tile(np.arange(n_folds, dtype=np.int32), steps)
    _, res, secs = fit.batch_find_mode(var, hold, row_fold, args)
    out = CVResult(float(pts[0]), float("nan"), fits=len(var), device_seconds=secs)
    best = None
    for s, p in enumerate(pts):
        pred = [r["pred_loglik"] if r["flag"] == SUCCESS else float("nan")
                for r in res[s * n_folds:(s + 1) * n_folds]]
        mean = point_estimate(pred)
        out.tried.append((float(p), mean, st_dev(pred, mean)))
        if best is None or mean > best:
            best, out.variance, out.value = mean, float(p), mean
    return out


def refit_at(ctx, matrix, d: CyclopsData, variance: float, args=None):
    """resetForOptimal: all rows weighted 1, the selected variance on every
    regularised column, cold start; returns native.FitResult."""
    from . import native
    dv = CyclopsData(**{**d.__dict__})
    dv.prior_var = np.where(d.prior_type == PRIOR_NONE, d.prior_var, variance)
    f = native.Fit(ctx, matrix, dv)
    try:
        return f.find_mode(args)
    finally:
        f.close()
