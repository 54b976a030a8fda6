"""Seeded synthetic problems with the shapes of the benchmark workloads.

The reference publishes no dataset for this path, so every workload is
generated here from a seeded ``numpy.random.Generator`` (PCG64): the same seed
gives the same bytes on every machine, so the CPU checker and the GPU path see
identical inputs.

Workloads (sizes are parameters; defaults are the full benchmark sizes):

* ``logistic_l1``      -- L1 logistic, N=10,000 x P=1,000 Bernoulli(0.01)
  indicators + intercept, 50 true nonzeros, Laplace variance 0.1.
* ``poisson_offset``   -- Poisson with offset, N=1e6 x P=1e5, column nnz from
  a rank-Zipf(s=1.1) law capped at 50,000 and scaled to ~2e7 in total, 80 %
  indicator / 20 % sparse LogNormal(0,1) columns, offset log(t),
  t ~ U(0.1, 5), 200 true nonzeros, Normal prior variance 1.
* ``cox_breslow``      -- Breslow Cox, N=1e6 rows in 1,000 strata of
  Dirichlet(0.5) sizes, P=5e4 indicators at density 0.002, integer-day event
  times with ties, 30 % events, Laplace variance 0.05.
* ``logistic_cv``      -- shared X for a cross-validation grid, N=5e5 x P=2e4
  indicators at density 0.005, intercept -3.
* ``conditional_logistic`` -- matched sets of 1 case : 1..10 controls.
* ``small``            -- tiny problems of any model/format mix for tests.
"""
from __future__ import annotations

import numpy as np

from .data import (DENSE, INDICATOR, INTERCEPT, MODEL_CONDITIONAL_LOGISTIC,
                   MODEL_CONDITIONAL_POISSON, MODEL_COX,
                   MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NONE, PRIOR_NORMAL,
                   SPARSE, CyclopsData, build_columns, cox_sort_order, csc_from_coo)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _bernoulli_csc(rng, K: int, P: int, density: float):
    """Indicator CSC with each entry 1 w.p. ``density`` (per-column binomial
    count, rows uniform without replacement -- distributionally a Bernoulli
    matrix)."""
    counts = rng.binomial(K, density, size=P)
    return _columns_with_counts(rng, K, counts)


def _columns_with_counts(rng, K: int, counts: np.ndarray):
    """CSC with exactly counts[j] distinct uniform rows in column j."""
    counts = np.minimum(np.asarray(counts, np.int64), K)
    P = counts.size
    col = np.repeat(np.arange(P, dtype=np.int64), counts)
    key = col * K + rng.integers(0, K, size=col.size, dtype=np.int64)
    key.sort()
    key = key[np.concatenate([[True], key[1:] != key[:-1]])] if key.size else key
    have = np.bincount(key // K, minlength=P)
    # top up the columns that lost entries to duplicate draws, touching only them
    for _ in range(100):
        short = np.nonzero(have < counts)[0]
        if short.size == 0:
            break
        in_short = np.isin(key // K, short)
        sub = key[in_short]
        need = (counts - have)[short]
        extra = np.repeat(short, need) * K + rng.integers(0, K, size=int(need.sum()), dtype=np.int64)
        sub = np.concatenate([sub, extra])
        sub.sort()
        sub = sub[np.concatenate([[True], sub[1:] != sub[:-1]])]
        key = np.concatenate([key[~in_short], sub])
        key.sort()
        have = np.bincount(key // K, minlength=P)
    col_start = np.zeros(P + 1, np.int64)
    np.cumsum(have, out=col_start[1:])
    return col_start, (key % K).astype(np.int32)


def _xbeta(K: int, col_start, rows, vals_per_entry, beta) -> np.ndarray:
    xb = np.zeros(K)
    nz = np.nonzero(beta)[0]
    for j in nz:
        a, b = col_start[j], col_start[j + 1]
        v = 1.0 if vals_per_entry is None else vals_per_entry[a:b]
        np.add.at(xb, rows[a:b], beta[j] * v)
    return xb


def logistic_l1(seed: int = 1, K: int = 10_000, P: int = 1_000, density: float = 0.01,
                n_true: int = 50, intercept: float = -2.0, variance: float = 0.1) -> CyclopsData:
    rng = _rng(seed)
    cs, rows = _bernoulli_csc(rng, K, P, density)
    beta = np.zeros(P)
    pos = rng.choice(P, size=min(n_true, P), replace=False)
    beta[pos] = rng.normal(0.0, 0.5, size=pos.size)
    xb = intercept + _xbeta(K, cs, rows, None, beta)
    y = (rng.random(K) < 1.0 / (1.0 + np.exp(-xb))).astype(np.float64)
    cols = [(None, None)] + [(rows[cs[j]:cs[j + 1]], None) for j in range(P)]
    fmts = [INTERCEPT] + [INDICATOR] * P
    col_start, r, val_start, vals, fmt = build_columns(K, cols, fmts)
    pt = np.full(P + 1, PRIOR_LAPLACE, np.int32)
    pt[0] = PRIOR_NONE
    pv = np.full(P + 1, variance)
    return CyclopsData(MODEL_LOGISTIC, y, col_start, r, val_start, vals, fmt, pt, pv,
                       meta={"workload": "logistic_l1", "seed": seed})


def zipf_counts(P: int, total: float, cap: int, s: float = 1.1) -> np.ndarray:
    """Column sizes from a rank-Zipf law n_r = min(cap, A / r^s), with A chosen
    so the sizes sum to ``total``."""
    r = np.arange(1, P + 1, dtype=np.float64)
    lo, hi = 1.0, float(cap) * P ** s
    for _ in range(200):
        A = np.sqrt(lo * hi)
        tot = np.minimum(cap, np.maximum(1.0, np.round(A / r ** s))).sum()
        if tot < total:
            lo = A
        else:
            hi = A
    return np.minimum(cap, np.maximum(1, np.round(hi / r ** s))).astype(np.int64)


def poisson_offset(seed: int = 2, K: int = 1_000_000, P: int = 100_000, total_nnz: float = 2e7,
                   cap: int = 50_000, sparse_frac: float = 0.2, n_true: int = 200,
                   intercept: float = -3.0, variance: float = 1.0) -> CyclopsData:
    rng = _rng(seed)
    counts = zipf_counts(P, total_nnz, min(cap, K))
    counts = counts[rng.permutation(P)]
    cs, rows = _columns_with_counts(rng, K, counts)
    is_sparse = rng.random(P) < sparse_frac
    nnz = int(cs[-1])
    entry_vals = np.ones(nnz)
    ent_col = np.repeat(np.arange(P), np.diff(cs))
    sp_mask = is_sparse[ent_col]
    entry_vals[sp_mask] = rng.lognormal(0.0, 1.0, size=int(sp_mask.sum()))
    beta = np.zeros(P)
    pos = rng.choice(P, size=min(n_true, P), replace=False)
    beta[pos] = rng.normal(0.0, 0.3, size=pos.size)
    t = rng.uniform(0.1, 5.0, size=K)
    xb = intercept + _xbeta(K, cs, rows, entry_vals, beta)
    y = rng.poisson(t * np.exp(xb)).astype(np.float64)
    cols = [(None, np.log(t)), (None, None)]
    fmts = [DENSE, INTERCEPT]
    for j in range(P):
        a, b = cs[j], cs[j + 1]
        if is_sparse[j]:
            cols.append((rows[a:b], entry_vals[a:b]))
            fmts.append(SPARSE)
        else:
            cols.append((rows[a:b], None))
            fmts.append(INDICATOR)
    col_start, r, val_start, vals, fmt = build_columns(K, cols, fmts)
    pt = np.full(P + 2, PRIOR_NORMAL, np.int32)
    pt[:2] = PRIOR_NONE
    pv = np.full(P + 2, variance)
    return CyclopsData(MODEL_POISSON, y, col_start, r, val_start, vals, fmt, pt, pv,
                       offset_col0=True, meta={"workload": "poisson_offset", "seed": seed})


def cox_breslow(seed: int = 3, K: int = 1_000_000, n_strata: int = 1_000, P: int = 50_000,
                density: float = 0.002, n_true: int = 300, event_frac: float = 0.3,
                variance: float = 0.05) -> CyclopsData:
    rng = _rng(seed)
    props = rng.dirichlet(np.full(n_strata, 0.5))
    sizes = rng.multinomial(K, props)
    stratum = np.repeat(np.arange(n_strata, dtype=np.int64), sizes)
    cs, rows = _bernoulli_csc(rng, K, P, density)
    beta = np.zeros(P)
    pos = rng.choice(P, size=min(n_true, P), replace=False)
    beta[pos] = rng.normal(0.0, 0.4, size=pos.size)
    xb = _xbeta(K, cs, rows, None, beta)
    T = rng.exponential(1.0, size=K) / (0.01 * np.exp(xb))
    E = rng.exponential(1.0, size=K)
    lo, hi = 1e-8, 10.0  # censoring rate chosen by bisection for the event fraction
    for _ in range(80):
        rate = np.sqrt(lo * hi)
        frac = np.mean(T < E / rate)
        if frac > event_frac:
            lo = rate
        else:
            hi = rate
    C = E / np.sqrt(lo * hi)
    y = (T < C).astype(np.float64)
    time = np.floor(np.minimum(T, C))
    order = cox_sort_order(stratum, time, y)
    inv = np.empty(K, np.int64)
    inv[order] = np.arange(K)
    # relabel rows into the sorted order, keep each column ascending
    col = np.repeat(np.arange(P, dtype=np.int64), np.diff(cs))
    cs2, rows2 = csc_from_coo(K, P, col, inv[rows])
    cols = [(rows2[cs2[j]:cs2[j + 1]], None) for j in range(P)]
    col_start, r, val_start, vals, fmt = build_columns(K, cols, [INDICATOR] * P)
    pt = np.full(P, PRIOR_LAPLACE, np.int32)
    pv = np.full(P, variance)
    return CyclopsData(MODEL_COX, y[order], col_start, r, val_start, vals, fmt, pt, pv,
                       time=time[order], stratum=stratum[order],
                       meta={"workload": "cox_breslow", "seed": seed})


def logistic_cv(seed: int = 4, K: int = 500_000, P: int = 20_000, density: float = 0.005,
                n_true: int = 100, intercept: float = -3.0) -> CyclopsData:
    d = logistic_l1(seed=seed, K=K, P=P, density=density, n_true=n_true, intercept=intercept,
                    variance=1.0)
    d.meta = {"workload": "logistic_cv", "seed": seed}
    return d


def conditional_logistic(seed: int = 5, n_sets: int = 2_000, P: int = 500, density: float = 0.01,
                         n_true: int = 20, variance: float = 0.1) -> CyclopsData:
    rng = _rng(seed)
    controls = rng.integers(1, 11, size=n_sets)
    sizes = controls + 1
    K = int(sizes.sum())
    stratum = np.repeat(np.arange(n_sets, dtype=np.int64), sizes)
    cs, rows = _bernoulli_csc(rng, K, P, density)
    beta = np.zeros(P)
    pos = rng.choice(P, size=min(n_true, P), replace=False)
    beta[pos] = rng.normal(0.0, 0.5, size=pos.size)
    xb = _xbeta(K, cs, rows, None, beta)
    y = np.zeros(K)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    for s, (a, n) in enumerate(zip(starts, sizes)):
        p = np.exp(xb[a:a + n] - xb[a:a + n].max())
        y[a + rng.choice(n, p=p / p.sum())] = 1.0
    cols = [(rows[cs[j]:cs[j + 1]], None) for j in range(P)]
    col_start, r, val_start, vals, fmt = build_columns(K, cols, [INDICATOR] * P)
    pt = np.full(P, PRIOR_LAPLACE, np.int32)
    pv = np.full(P, variance)
    return CyclopsData(MODEL_CONDITIONAL_LOGISTIC, y, col_start, r, val_start, vals, fmt, pt, pv,
                       stratum=stratum, meta={"workload": "conditional_logistic", "seed": seed})


def small(model: int, seed: int = 0, K: int = 300, P: int = 12, density: float = 0.15,
          formats=("indicator", "sparse", "dense"), intercept: bool = True, offset: bool = False,
          prior: int = PRIOR_LAPLACE, variance: float = 1.0, n_strata: int = 20,
          tie_days: int = 20) -> CyclopsData:
    """A tiny problem mixing column formats, for parity tests."""
    rng = _rng(seed)
    names = {"indicator": INDICATOR, "sparse": SPARSE, "dense": DENSE}
    fm = [names[formats[j % len(formats)]] for j in range(P)]
    cols = []
    xb = np.zeros(K)
    beta_true = rng.normal(0.0, 0.6, size=P)
    for j in range(P):
        if fm[j] == DENSE:
            v = rng.normal(0.0, 1.0, size=K)
            cols.append((None, v))
            xb += beta_true[j] * v
        else:
            cnt = max(1, rng.binomial(K, density))
            r = np.sort(rng.choice(K, size=cnt, replace=False)).astype(np.int32)
            v = rng.lognormal(0.0, 0.5, size=cnt) if fm[j] == SPARSE else None
            cols.append((r, v))
            xb[r] += beta_true[j] * (1.0 if v is None else v)
    stratum = None
    time = None
    if model == MODEL_LOGISTIC:
        y = (rng.random(K) < 1 / (1 + np.exp(-(xb - 0.5)))).astype(np.float64)
    elif model == MODEL_POISSON:
        t = rng.uniform(0.5, 2.0, size=K)
        y = rng.poisson(t * np.exp(0.3 * xb)).astype(np.float64)
        time = np.log(t) if offset else None
    elif model == MODEL_CONDITIONAL_LOGISTIC:
        stratum = np.sort(rng.integers(0, n_strata, size=K)).astype(np.int64)
        y = np.zeros(K)
        for s in np.unique(stratum):
            idx = np.nonzero(stratum == s)[0]
            y[idx[rng.integers(0, idx.size)]] = 1.0
        intercept = False
    elif model == MODEL_CONDITIONAL_POISSON:
        stratum = np.sort(rng.integers(0, n_strata, size=K)).astype(np.int64)
        y = rng.poisson(np.exp(0.3 * xb)).astype(np.float64)
        intercept = False
    elif model == MODEL_COX:
        stratum = np.sort(rng.integers(0, n_strata, size=K)).astype(np.int64)
        T = rng.exponential(1.0, size=K) / (0.05 * np.exp(0.5 * xb))
        C = rng.exponential(1.0, size=K) / 0.03
        y = (T < C).astype(np.float64)
        time = np.floor(np.minimum(T, C) * tie_days / 20.0)
        order = cox_sort_order(stratum, time, y)
        inv = np.empty(K, np.int64)
        inv[order] = np.arange(K)
        new_cols = []
        for (r, v) in cols:
            if r is None:
                new_cols.append((None, v[order]))
            else:
                rr = inv[r]
                o = np.argsort(rr)
                new_cols.append((rr[o].astype(np.int32), None if v is None else v[o]))
        cols = new_cols
        y, time, stratum = y[order], time[order], stratum[order]
        intercept = False
    else:
        raise ValueError(model)
    if intercept:
        cols = [(None, None)] + cols
        fm = [INTERCEPT] + fm
    if offset:
        if time is None:
            raise ValueError("offset requires a Poisson model")
        cols = [(None, time)] + cols
        fm = [DENSE] + fm
        time = None
    col_start, r, val_start, vals, fmt = build_columns(K, cols, fm)
    J = len(fm)
    pt = np.full(J, prior, np.int32)
    pv = np.full(J, variance)
    for j in range(J):
        if fm[j] == INTERCEPT or (offset and j == 0):
            pt[j] = PRIOR_NONE
    d = CyclopsData(model, y, col_start, r, val_start, vals, fmt, pt, pv, time=time,
                    stratum=stratum, offset_col0=offset,
                    meta={"workload": "small", "seed": seed})
    d.validate()
    return d


def cv_folds(K: int, n_folds: int = 10, seed: int = 7) -> np.ndarray:
    """Row -> fold: a seeded permutation cut into contiguous intervals whose sizes
    follow CrossValidationSelector (drivers/CrossValidationSelector.cpp:31-45):
    K // n_folds rows each, one extra for the first K % n_folds folds."""
    rng = _rng(seed)
    perm = rng.permutation(K)
    sizes = np.full(n_folds, K // n_folds)
    sizes[:K % n_folds] += 1
    fold = np.empty(K, np.int32)
    start = 0
    for f, n in enumerate(sizes):
        fold[perm[start:start + n]] = f
        start += n
    return fold


def cv_grid(n_folds: int = 10, n_vars: int = 20, lower: float = 1e-4, upper: float = 1.0):
    """(holdout fold, variance) of every instance of a fold x variance grid.  Variances
    are log-uniform between lower and upper as GridSearchCrossValidationDriver::
    computeGridPoint places them (drivers/GridSearchCrossValidationDriver.cpp:38-50)."""
    if n_vars == 1:
        grid = np.array([upper])
    else:
        step = (np.log(upper) - np.log(lower)) / (n_vars - 1)
        grid = np.exp(np.log(lower) + step * np.arange(n_vars))
    hold = np.repeat(np.arange(n_folds, dtype=np.int32), n_vars)
    var = np.tile(grid, n_folds)
    return hold, var


def serving_stream(n_requests: int = 200, seed: int = 11, rate: float = 50.0,
                   K_range=(1e3, 1e5), J_range=(1e2, 1e4), density_range=(0.001, 0.02),
                   variance: float = 0.1):
    """A served stream of independent fits: Poisson(rate) arrivals; each request
    an independently seeded problem, 50 % logistic, 30 % conditional logistic
    (one case : 1-10 controls per matched set), 20 % Breslow Cox; K and J
    log-uniform over the given ranges, indicator density uniform, 10-200 true
    coefficients, Laplace prior of the given variance on every covariate.
    Returns [(arrival seconds, CyclopsData)] in arrival order."""
    rng = _rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    out = []
    for i in range(n_requests):
        u = rng.random()
        K = int(round(np.exp(rng.uniform(np.log(K_range[0]), np.log(K_range[1])))))
        J = int(round(np.exp(rng.uniform(np.log(J_range[0]), np.log(J_range[1])))))
        dens = float(rng.uniform(*density_range))
        n_true = int(rng.integers(10, 201))
        s = int(rng.integers(1, 2 ** 31 - 1))
        if u < 0.5:
            d = logistic_l1(seed=s, K=K, P=J, density=dens, n_true=n_true, intercept=-2.0, variance=variance)
        elif u < 0.8:
            d = conditional_logistic(seed=s, n_sets=max(1, int(round(K / 6.5))), P=J, density=dens,
                                     n_true=n_true, variance=variance)
        else:
            d = cox_breslow(seed=s, K=K, n_strata=max(1, K // 1000), P=J, density=dens, n_true=n_true,
                            variance=variance)
        d.meta = dict(d.meta, request=i)
        out.append((float(t[i]), d))
    return out
