"""Autotuning of launch shapes, keyed on the column-nnz histogram of the matrix.

Two launch parameters decide how fast the engine runs a given matrix, and
neither changes what is computed beyond the order of the per-column sums:

* the batched engine (ccdb_batch_find_mode, mixed precision): the lockstep
  group size G (instances stepped together by one CTA) and the CTAs per group
  C (a thread-block cluster that splits each column's rows);
* the plain cluster sweep (ccdb_find_mode): the CTAs of its cluster, set
  through ccdb_context_set_max_ctas (the largest power of two not above it).

The engine's own choice when nothing is passed is a fixed rule (the longest
column slice a CTA would stage, the instance count, the SM count).  The
tuners here measure instead: each candidate runs one sweep of the real
problem (max_iterations = 1) and the fastest by device time wins.  Results
are cached under a key made of the matrix's column-nnz histogram (log2 bins),
its shape and the call's size, so a second grid or fit over a matrix with the
same histogram reuses the choice without measuring.  A choice depends on
timing, so it can differ between machines and runs; a caller that needs the
same bits every time passes the returned values back explicitly
(group=, cluster=, set_max_ctas), which is what makes a run reproducible.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Iterable, Optional, Tuple

import numpy as np

from .data import DENSE, INTERCEPT, CyclopsData

_CACHE: Dict[tuple, tuple] = {}


def nnz_histogram(d: CyclopsData) -> np.ndarray:
    """Columns per log2 bin of their entry count: bin 0 holds empty columns,
    bin b >= 1 the columns with 2**(b-1) .. 2**b - 1 entries (dense-like
    columns count K entries)."""
    cnt = np.diff(np.asarray(d.col_start, dtype=np.int64))
    dense = np.isin(np.asarray(d.fmt), (DENSE, INTERCEPT))
    cnt = np.where(dense, d.K, cnt)
    bins = np.zeros(64, dtype=np.int64)
    nz = cnt > 0
    bins[0] = int(np.count_nonzero(~nz))
    if nz.any():
        b = np.floor(np.log2(cnt[nz])).astype(np.int64) + 1
        np.add.at(bins, b, 1)
    return bins


def histogram_key(d: CyclopsData) -> tuple:
    h = nnz_histogram(d)
    last = int(np.max(np.nonzero(h)[0])) + 1 if h.any() else 0
    return (int(d.K), int(d.J), tuple(int(x) for x in h[:last]))


def clear_cache() -> None:
    _CACHE.clear()


@dataclasses.dataclass
class BatchChoice:
    group: int
    cluster: int
    seconds: Dict[Tuple[int, int], float]  # one sweep per candidate (empty when cached)
    cached: bool = False


def batch_candidates() -> Iterable[Tuple[int, int]]:
    for g in (4, 2, 1):
        for c in (1, 2, 4, 8):
            yield g, c


def filling(candidates, n_instances: int, n_sm: int):
    """The candidates whose grid puts a CTA on every SM (groups x cluster >= SMs),
    or all of them when none does.  A grid's time is its slowest group's chain
    of sweeps (the least regularised instances take the most), and that chain
    is shorter when the group's instances spread over more CTAs; one measured
    sweep of the whole grid sees throughput, not that chain, and favours shapes
    that leave SMs idle."""
    cands = list(candidates)
    fill = [(g, c) for g, c in cands if ((n_instances + g - 1) // g) * c >= n_sm]
    return fill or cands


def tune_batch(fit, variance, holdout, row_fold, args=None, candidates=None) -> BatchChoice:
    """The (group, cluster) of the mixed-precision batched engine that runs one
    sweep of this grid fastest among the shapes that occupy every SM.  `fit` is a
    native.Fit (or anything with its batch_find_mode and ctx.sm_count); the grid
    is the one about to be fitted."""
    from . import native
    var = np.asarray(variance, dtype=np.float64)
    key = ("batch", histogram_key(fit.d), int(var.shape[0]), int(getattr(fit, "precision", 0)))
    if key in _CACHE:
        g, c = _CACHE[key]
        return BatchChoice(g, c, {}, cached=True)
    base = args or native.ModeFindingArguments()
    one = dataclasses.replace(base, max_iterations=1)
    seconds: Dict[Tuple[int, int], float] = {}
    n_sm = int(getattr(getattr(fit, "ctx", None), "sm_count", 0) or 0)
    cands = list(candidates or batch_candidates())
    if n_sm > 0:
        cands = filling(cands, int(var.shape[0]), n_sm)
    for g, c in cands:
        try:
            _, _, secs = fit.batch_find_mode(var, holdout, row_fold, one, group=g, cluster=c)
        except native.CcdbError:
            continue  # a shape this device or matrix cannot take
        seconds[(g, c)] = float(secs)
    if not seconds:
        raise RuntimeError("no candidate launch shape ran")
    best = min(seconds, key=lambda k: (seconds[k], k))
    _CACHE[key] = best
    return BatchChoice(best[0], best[1], seconds)


@dataclasses.dataclass
class SweepChoice:
    max_ctas: int
    seconds: Dict[int, float]
    cached: bool = False


def tune_sweep(ctx, fit, args=None, candidates=(16, 8, 4, 2)) -> SweepChoice:
    """The cluster size of the plain sweep that runs one sweep of this fit
    fastest; the context is left set to it (ccdb_context_set_max_ctas).  The
    fit's coefficients are reset to a cold start after each trial."""
    from . import native
    key = ("sweep", histogram_key(fit.d), int(fit.d.model_type))
    if key in _CACHE:
        (mc,) = _CACHE[key]
        ctx.set_max_ctas(mc)
        return SweepChoice(mc, {}, cached=True)
    base = args or native.ModeFindingArguments()
    one = dataclasses.replace(base, max_iterations=1, strategy=native.SWEEP_LEVELS)
    cold = np.zeros(fit.d.J)
    if fit.d.offset_col0:
        cold[0] = 1.0
    seconds: Dict[int, float] = {}
    for mc in candidates:
        ctx.set_max_ctas(mc)
        try:
            fit.find_mode(one, beta=cold.copy())  # the schedule for this size is built here
            r = fit.find_mode(one, beta=cold.copy())
        except native.CcdbError:
            continue
        seconds[mc] = float(r.kernel_seconds)
    if not seconds:
        raise RuntimeError("no candidate cluster size ran")
    best = min(seconds, key=lambda k: (seconds[k], -k))
    ctx.set_max_ctas(best)
    _CACHE[key] = (best,)
    return SweepChoice(best, seconds)
