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
  steps.  With several variance parameters (columns under different priors)
  the search tunes each in turn and repeats the round until the summed
  relative change of the proposals is below 1e-2.
* Refit (resetForOptimal, AbstractCrossValidationDriver.cpp:31-42): all rows
  weighted 1, the selected variances, cold start.

The hyperparameters are the joint prior's variance parameters
(JointPrior::getVariance, priors/JointPrior.h:48-70): one per distinct prior,
registered in column order, none for a flat column (variance_groups).  When
every regularised column shares one prior -- a single prior type with some
columns excluded, the usual set-up -- a variance is one launch of the batched
engine for logistic and Poisson models.  Otherwise each (fold, variances)
instance is a standalone device fit (native.Fit.fold_instances), which
needs an FP64 fit.  Every
column flat is refused as the R front end refuses it (createPrior,
R/ModelFit.R:600-602); the engine's own driver would index a variance
parameter that does not exist.

Instances start cold (the reference's resetCoefficients = TRUE); its default
warm start depends on which thread ran which task before, so it has no fixed
batched counterpart.
"""
from __future__ import annotations

import math
import sys
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .data import DENSE, INTERCEPT, MODEL_LOGISTIC, MODEL_POISSON, PRIOR_NONE, CyclopsData

SUCCESS = 0
FLAT_PRIOR = "Cannot perform cross validation with a flat prior"
CYCLE_TOLERANCE = 1e-2  # AutoSearchCrossValidationDriver.cpp:84
MAX_CYCLES = 100


def variance_groups(d: CyclopsData) -> List[np.ndarray]:
    """The columns under each variance parameter of the joint prior, in the
    order the parameters are registered: the prior of column 0, then each
    column's prior as MixtureJointPrior::changePrior adds it
    (priors/JointPrior.h:80-95), a parameter shared by every column of the
    same (prior type, variance).  Flat columns carry none (NoPrior,
    priors/CovariatePrior.h:160-172)."""
    keys: list = []
    groups: List[list] = []
    for j in range(d.J):
        t = int(d.prior_type[j])
        if t == PRIOR_NONE:
            continue
        key = (t, float(d.prior_var[j]))
        if key in keys:
            groups[keys.index(key)].append(j)
        else:
            keys.append(key)
            groups.append([j])
    return [np.asarray(g, dtype=np.int32) for g in groups]


def column_variances(d: CyclopsData, variances) -> np.ndarray:
    """Per-column prior variances with the leading variance parameters set
    (CyclicCoordinateDescent::setHyperprior(i, x) for each given i); a scalar
    sets the first, as setHyperprior(x)."""
    values = [float(variances)] if np.isscalar(variances) else [float(x) for x in variances]
    out = np.asarray(d.prior_var, dtype=np.float64).copy()
    for cols, x in zip(variance_groups(d), values):
        out[cols] = x
    return out


def _one_launch(fit, groups) -> bool:
    """Whether a variance's folds run as one batched launch: one variance
    parameter over every regularised column, on a model the batched engine
    takes."""
    return len(groups) == 1 and int(fit.d.model_type) in (MODEL_LOGISTIC, MODEL_POISSON)


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
    utils/HParSearch.cpp:22-64.

    Near the end of a search the history is nearly flat and this 3 x 3 system
    is badly conditioned, so the proposal depends on the rounding of each
    step.  The arithmetic is therefore done in the order the reference's
    build does it: its linear algebra library (Eigen 3.1.3, vendored with
    the reference, SSE2 doubles) forms X'W X by sequential sums over the
    history, X'W y by the column-major matrix-vector kernel (columns four at
    a time, in the order i, i+3, i+2, i+1, summed pairwise for the two rows
    of a vector register and one by one for the third row, then the leftover
    columns one by one), and solves by LU with complete pivoting (largest
    magnitude, first in column-major order), the column below the pivot
    multiplied by the pivot's reciprocal, then column-oriented forward and
    back substitution."""
    xs = sorted(history)
    n = len(xs)
    minsd = sys.float_info.max
    for x in xs:
        sd = history[x][1]
        if 0 < sd < minsd:
            minsd = sd
    zero_adjust = 100.0 / minsd if minsd < sys.float_info.max else 1.0
    X = []
    XTW = [[0.0] * n for _ in range(3)]
    Y = []
    for i, x in enumerate(xs):
        m, sd = history[x]
        weight = 1.0 / sd if sd > 0 else zero_adjust
        lx = math.log(x)
        row = [1.0, lx, math.log(x) * math.log(x)]
        X.append(row)
        for j in range(3):
            XTW[j][i] = row[j] * weight
        Y.append(m)
    # X'W X: sequential sums over the history
    A = [[0.0] * 3 for _ in range(3)]
    for r in range(3):
        for c in range(3):
            acc = 0.0
            for i in range(n):
                acc = acc + XTW[r][i] * X[i][c]
            A[r][c] = acc
    # X'W y: the matrix-vector kernel's order
    b = [0.0, 0.0, 0.0]
    bound = (n // 4) * 4
    for i in range(0, bound, 4):
        order = (i, i + 3, i + 2, i + 1)
        for r in (0, 1):
            t = [XTW[r][k] * Y[k] for k in order]
            b[r] = b[r] + ((t[0] + t[1]) + (t[2] + t[3]))
        for k in order:
            b[2] = XTW[2][k] * Y[k] + b[2]
    for k in range(bound, n):
        for r in range(3):
            b[r] = XTW[r][k] * Y[k] + b[r]
    # LU with complete pivoting
    lu = [row[:] for row in A]
    row_t, col_t = [0, 0, 0], [0, 0, 0]
    nonzero = 3
    for k in range(3):
        best, br, bc = -1.0, k, k
        for c in range(k, 3):
            for r in range(k, 3):
                v = abs(lu[r][c])
                if v > best:
                    best, br, bc = v, r, c
        if best == 0.0:
            nonzero = k
            for i in range(k, 3):
                row_t[i] = col_t[i] = i
            break
        row_t[k], col_t[k] = br, bc
        if br != k:
            lu[k], lu[br] = lu[br], lu[k]
        if bc != k:
            for r in range(3):
                lu[r][k], lu[r][bc] = lu[r][bc], lu[r][k]
        inv = 1.0 / lu[k][k]  # the column is scaled by the reciprocal, not divided
        for r in range(k + 1, 3):
            lu[r][k] = lu[r][k] * inv
        for c in range(k + 1, 3):
            for r in range(k + 1, 3):
                lu[r][c] = lu[r][c] - lu[r][k] * lu[k][c]
    if nonzero == 0:
        return 0.0, 0.0, 0.0
    c = b[:]
    for k in range(3):  # c = P b
        if row_t[k] != k:
            c[k], c[row_t[k]] = c[row_t[k]], c[k]
    for i in range(3):  # unit lower, column by column
        for t in range(i + 1, 3):
            c[t] = c[t] - c[i] * lu[t][i]
    for i in range(nonzero - 1, -1, -1):  # upper, from the last column
        c[i] = c[i] / lu[i][i]
        for t in range(0, i):
            c[t] = c[t] - c[i] * lu[t][i]
    q = list(range(3))  # x = Q c
    for k in range(3):
        if col_t[k] != k:
            q[k], q[col_t[k]] = q[col_t[k]], q[k]
    out = [0.0, 0.0, 0.0]
    for i in range(nonzero):
        out[q[i]] = c[i]
    return out[0], out[1], out[2]


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
    variances: List[float] = field(default_factory=list)  # every variance parameter selected
    rounds: int = 1  # auto search rounds over the variance parameters
    converged: bool = True  # False: max_cycles rounds ran without the rounds settling


def _fold_values(fit, groups, applied: np.ndarray, variance: float, n_folds: int, row_fold, args):
    """Held-out predictive log-likelihood of every fold (NaN where the fit
    failed) with the columns at `applied`; `variance` is the value of the
    single variance parameter when the folds run as one launch."""
    hold = np.arange(n_folds, dtype=np.int32)
    if _one_launch(fit, groups):
        _, res, secs = fit.batch_find_mode(np.full(n_folds, float(variance)), hold, row_fold, args)
    else:
        _, res, secs = fit.fold_instances(np.tile(applied, (n_folds, 1)), hold, row_fold, args)
    pred = [r["pred_loglik"] if r["flag"] == SUCCESS else float("nan") for r in res]
    return pred, secs


def auto_search(fit, d: CyclopsData, row_fold, n_folds: int, args=None, starting_variance: float = -1.0,
                max_steps: int = 50, max_cycles: int = MAX_CYCLES) -> CVResult:
    """The reference's default cross-validation (cvType "auto"): `fit` is a
    native.Fit over the data (FP64 or mixed).  Each variance parameter in turn
    runs a unimodal search of at most `max_steps` steps, all starting at the
    same variance; while a parameter is searched the others keep the values
    their fits last ran at (the prior's own before their first search), as
    setHyperprior(dim, x) leaves them.  With several parameters the rounds
    repeat until the summed relative change of the proposals is below 1e-2,
    at most `max_cycles` rounds.  The reference has no bound and does not
    return when the rounds never settle (a variance that shrinks by a
    constant factor each round; once it reaches 0 the change is NaN); here
    the result then says converged=False."""
    groups = variance_groups(d)
    if not groups:
        raise ValueError(FLAT_PRIOR)
    v = starting_variance if starting_variance > 0 else normal_based_default_var(d)
    current = [v] * len(groups)
    applied = np.asarray(d.prior_var, dtype=np.float64).copy()
    out = CVResult(v, float("nan"))
    out.converged = False
    for cycle in range(max_cycles):
        out.rounds = cycle + 1
        saved = list(current)
        for g, cols in enumerate(groups):
            search = UniModalSearch(10.0, 0.01, math.log(1.5))
            for step in range(max_steps):
                applied[cols] = current[g]
                pred, secs = _fold_values(fit, groups, applied, current[g], n_folds, row_fold, args)
                mean = point_estimate(pred)
                sd = st_dev(pred, mean)
                out.tried.append((current[g], mean, sd))
                out.fits += n_folds
                out.device_seconds += secs
                search.tried(current[g], mean, sd)
                cont, nxt, expected = search.step()
                current[g], out.value = nxt, expected
                if not cont:
                    break
        if len(groups) == 1 or sum(abs((c - s) / s) for c, s in zip(current, saved)) < CYCLE_TOLERANCE:
            out.converged = True
            break
    out.variance = current[0]
    out.variances = list(current)
    return out


def grid_points(lower: float, upper: float, steps: int) -> np.ndarray:
    if steps == 1:
        return np.array([upper])
    size = (math.log(upper) - math.log(lower)) / (steps - 1)
    return np.array([math.exp(math.log(lower) + s * size) for s in range(steps)])


def grid_search(fit, row_fold, n_folds: int, lower: float = 0.01, upper: float = 20.0, steps: int = 10,
                args=None) -> CVResult:
    """Every (fold, variance) of the grid at once; the first maximum of the
    mean held-out predictive log-likelihood wins.  The grid moves the first
    variance parameter only (setHyperprior(x)); the others keep the prior's
    values."""
    d = fit.d
    groups = variance_groups(d)
    if not groups:
        raise ValueError(FLAT_PRIOR)
    pts = grid_points(lower, upper, steps)
    hold = np.tile(np.arange(n_folds, dtype=np.int32), steps)
    if _one_launch(fit, groups):
        _, res, secs = fit.batch_find_mode(np.repeat(pts, n_folds), hold, row_fold, args)
    else:
        colvar = np.repeat(np.stack([column_variances(d, p) for p in pts]), n_folds, axis=0)
        _, res, secs = fit.fold_instances(colvar, hold, row_fold, args)
    out = CVResult(float(pts[0]), float("nan"), fits=len(hold), device_seconds=secs)
    best = None
    for s, p in enumerate(pts):
        pred = [r["pred_loglik"] if r["flag"] == SUCCESS else float("nan")
                for r in res[s * n_folds:(s + 1) * n_folds]]
        mean = point_estimate(pred)
        out.tried.append((float(p), mean, st_dev(pred, mean)))
        if best is None or mean > best:
            best, out.variance, out.value = mean, float(p), mean
    out.variances = [out.variance]
    return out


class ShardedFit:
    """The batched calls of a fit, spread over the ranks of a torch.distributed
    process group: one process per GPU, each with its own context, its own
    copy of the matrix in its GPU's memory and its own fit (`fit`), all over
    the same data.  Instance i of a call runs on rank i mod world (round
    robin, so every rank gets a share of each variance, the weak priors being
    the longest fits); after the local launch the ranks exchange their
    (instance, coefficients, result) lists once (all_gather_object, a host
    gather: no collective on the data path), so every rank returns the whole
    call's results in instance order and the drivers above run unchanged, in
    step, on every rank.  device_seconds is the slowest rank's.

    grid_search / auto_search take a ShardedFit wherever they take a fit."""

    def __init__(self, fit, group=None):
        import torch.distributed as dist
        self.fit = fit
        self.d = fit.d
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    @property
    def precision(self):
        return getattr(self.fit, "precision", 0)

    def _shard(self, n: int) -> np.ndarray:
        return np.arange(self.rank, n, self.world)

    def _gather(self, n: int, mine, beta, res, secs):
        import torch.distributed as dist
        parts = [None] * self.world
        dist.all_gather_object(parts, (np.asarray(mine).tolist(), np.asarray(beta), list(res), float(secs)),
                               group=self.group)
        out_b = np.zeros((n, self.d.J))
        out_r: list = [None] * n
        for idx, b, r, _ in parts:
            for q, i in enumerate(idx):
                out_b[i] = b[q]
                out_r[i] = r[q]
        return out_b, out_r, max(p[3] for p in parts)

    def batch_find_mode(self, variance, holdout=None, row_fold=None, args=None, group: int = 0,
                        cluster: int = 0):
        var = np.asarray(variance, dtype=np.float64)
        n = var.shape[0]
        mine = self._shard(n)
        if len(mine):
            hold = None if holdout is None else np.asarray(holdout)[mine]
            beta, res, secs = self.fit.batch_find_mode(var[mine], hold, row_fold, args, group=group,
                                                       cluster=cluster)
        else:
            beta, res, secs = np.zeros((0, self.d.J)), [], 0.0
        return self._gather(n, mine, beta, res, secs)

    def fold_instances(self, variances, holdout, row_fold, args=None):
        var = np.asarray(variances, dtype=np.float64)
        n = var.shape[0]
        mine = self._shard(n)
        if len(mine):
            beta, res, secs = self.fit.fold_instances(var[mine], np.asarray(holdout)[mine], row_fold, args)
        else:
            beta, res, secs = np.zeros((0, self.d.J)), [], 0.0
        return self._gather(n, mine, beta, res, secs)


def refit_at(ctx, matrix, d: CyclopsData, variance, args=None):
    """resetForOptimal: all rows weighted 1, the selected variance parameters
    (a scalar: the first; a sequence: one per parameter, CVResult.variances),
    cold start; returns native.FitResult."""
    from . import native
    dv = CyclopsData(**{**d.__dict__})
    dv.prior_var = column_variances(d, variance)
    f = native.Fit(ctx, matrix, dv)
    try:
        return f.find_mode(args)
    finally:
        f.close()
