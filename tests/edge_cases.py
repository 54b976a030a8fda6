"""Small problems at the edges of the engine's inputs, shared by the oracle
and GPU edge-case tests: strata of one row, strata without events, a stratum
whose rows all carry zero weight, empty and all-row columns, duplicated and
intercept-equal columns, ties everywhere, a count model with all-zero
outcomes, large covariate values."""
import numpy as np

from ccd_b200 import synthetic
from ccd_b200.data import (DENSE, INDICATOR, INTERCEPT, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX, MODEL_LOGISTIC,
                           MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL, CyclopsData, build_columns)


def _with_columns(d, extra_cols, extra_fmts, prior=PRIOR_NORMAL, var=1.0):
    """d with extra (rows, vals) columns appended."""
    cols = []
    for j in range(d.J):
        f = int(d.fmt[j])
        if f == INTERCEPT:
            cols.append((None, None))
        elif f == DENSE:
            cols.append((None, d.vals[d.val_start[j]:d.val_start[j] + d.K]))
        else:
            r = d.rows[d.col_start[j]:d.col_start[j + 1]]
            cols.append((r, None if f == INDICATOR else d.vals[d.val_start[j]:d.val_start[j] + len(r)]))
    cols += extra_cols
    fmts = list(d.fmt) + list(extra_fmts)
    cs, r, vs, v, fm = build_columns(d.K, cols, fmts)
    J = len(fmts)
    pt = np.concatenate([d.prior_type, np.full(len(extra_fmts), prior, np.int32)])
    pv = np.concatenate([d.prior_var, np.full(len(extra_fmts), var)])
    return CyclopsData(d.model_type, d.y, cs, r, vs, v, fm, pt, pv, time=d.time, stratum=d.stratum,
                       offset_col0=d.offset_col0)


def cases():
    """name -> (data, weights or None)."""
    out = {}
    # logistic: an empty column, a column on every row, a duplicate, a column equal to the intercept
    d = synthetic.small(MODEL_LOGISTIC, seed=180, K=200, P=6, prior=PRIOR_NORMAL)
    r1 = d.rows[d.col_start[1]:d.col_start[2]]
    d = _with_columns(d, [(np.array([], np.int32), None), (np.arange(d.K, dtype=np.int32), None), (r1, None)],
                      [INDICATOR, INDICATOR, INDICATOR])
    out["lr_empty_full_duplicate"] = (d, None)
    # logistic with large covariate values (exp over a wide range) under Laplace
    d = synthetic.small(MODEL_LOGISTIC, seed=181, K=200, P=5, formats=("dense",), prior=PRIOR_LAPLACE)
    d.vals = d.vals * 30.0
    out["lr_large_values"] = (d, None)
    # Poisson with all-zero outcomes on half the rows and a zero-weight block
    d = synthetic.small(MODEL_POISSON, seed=182, K=200, P=6, prior=PRIOR_NORMAL)
    d.y[: d.K // 2] = 0.0
    w = np.ones(d.K)
    w[10:40] = 0.0
    out["poisson_zeros_zero_weight_block"] = (d, w)
    # conditional logistic: strata of one row, strata without events
    rng = np.random.default_rng(183)
    sizes = np.array([1, 1, 3, 4, 1, 5, 2, 6, 1, 3] * 6)
    K = int(sizes.sum())
    stratum = np.repeat(np.arange(len(sizes), dtype=np.int64), sizes)
    y = np.zeros(K)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    for s, (a, n) in enumerate(zip(starts, sizes)):
        if s % 4 != 1:  # every fourth stratum has no event
            y[a + rng.integers(0, n)] = 1.0
    cols = [(np.sort(rng.choice(K, size=K // 3, replace=False)).astype(np.int32), None) for _ in range(4)]
    cols.append((None, rng.normal(size=K)))
    cs, r, vs, v, fm = build_columns(K, cols, [INDICATOR] * 4 + [DENSE])
    d = CyclopsData(MODEL_CONDITIONAL_LOGISTIC, y, cs, r, vs, v, fm, np.full(5, PRIOR_NORMAL, np.int32),
                    np.ones(5), stratum=stratum)
    out["clr_singletons_no_events"] = (d, None)
    # conditional logistic with zero weights on single rows inside strata
    w = (np.arange(K) % 5 != 3).astype(float)
    out["clr_row_zero_weights"] = (d, w)
    # Poisson with an offset, Laplace priors and fractional weights
    d = synthetic.small(MODEL_POISSON, seed=186, K=200, P=6, offset=True, prior=PRIOR_LAPLACE, variance=0.5)
    out["poisson_offset_laplace_fractional_weights"] = (d, 0.25 + (np.arange(d.K) % 4) * 0.5)
    # Cox: one stratum entirely censored, one with zero weights throughout, every time tied
    d = synthetic.small(MODEL_COX, seed=184, K=240, P=5, n_strata=4, tie_days=1, prior=PRIOR_NORMAL)
    s0 = d.stratum == d.stratum.min()
    d.y[s0] = 0.0
    w = np.ones(d.K)
    w[d.stratum == d.stratum.max()] = 0.0
    out["cox_censored_stratum_zero_weight_stratum"] = (d, w)
    d = synthetic.small(MODEL_COX, seed=185, K=150, P=4, n_strata=1, tie_days=1, prior=PRIOR_NORMAL)
    d.time[:] = 1.0  # one risk set: every event ties with every row
    out["cox_all_tied"] = (d, None)
    return out
