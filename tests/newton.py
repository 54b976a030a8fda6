"""An independent FP64 Newton solver for the unpenalised maximum-likelihood
fits of the reference's small R tests: the stand-in for glm (logistic,
Poisson), clogit (conditional logistic) and coxph (Breslow ties), which are
not available here.  Dense numpy, full Newton steps from beta = 0; the MLE is
unique, so it reproduces what those packages report."""
import numpy as np

from ccd_b200.data import DENSE, INDICATOR, INTERCEPT, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX, MODEL_LOGISTIC, MODEL_POISSON


def design(d) -> np.ndarray:
    X = np.zeros((d.K, d.J))
    for j in range(d.J):
        f = int(d.fmt[j])
        if f == INTERCEPT:
            X[:, j] = 1.0
        elif f == DENSE:
            X[:, j] = d.vals[d.val_start[j]:d.val_start[j] + d.K]
        else:
            r = d.rows[d.col_start[j]:d.col_start[j + 1]]
            X[r, j] = 1.0 if f == INDICATOR else d.vals[d.val_start[j]:d.val_start[j] + len(r)]
    return X


def _groups(d):
    """Row index sets of the conditional model's strata."""
    s = d.stratum
    return [np.nonzero(s == v)[0] for v in np.unique(s)]


def _cox_sets(d, wt):
    """(event row, risk set rows) of every event of nonzero weight: Breslow
    ties, each event's risk set is every row of its stratum with time >= its
    time."""
    out = []
    for idx in _groups(d):
        t = d.time[idx]
        for a in idx[(d.y[idx] == 1) & (wt[idx] != 0)]:
            out.append((a, idx[t >= d.time[a]]))
    return out


def loglik_grad_hess(d, X, beta, weights=None):
    """Weighted log-likelihood: each row's term times its weight (glm / coxph
    prior weights); for Cox the risk-set sums are weighted too."""
    wt = np.ones(d.K) if weights is None else np.asarray(weights, np.float64)
    xb = X @ beta
    if d.model_type == MODEL_LOGISTIC:
        p = 1.0 / (1.0 + np.exp(-xb))
        ll = float(np.sum(wt * (d.y * xb - np.log1p(np.exp(xb)))))
        return ll, X.T @ (wt * (d.y - p)), -(X.T * (wt * p * (1 - p))) @ X
    if d.model_type == MODEL_POISSON:
        mu = np.exp(xb)
        from math import lgamma
        ll = float(np.sum(wt * (d.y * xb - mu))) - sum(w * lgamma(v + 1.0) for w, v in zip(wt, d.y))
        return ll, X.T @ (wt * (d.y - mu)), -(X.T * (wt * mu)) @ X
    if d.model_type == MODEL_CONDITIONAL_LOGISTIC:
        if weights is not None:
            raise ValueError("weighted conditional logistic is not a known answer here")
        sets = [(idx, idx, float(np.sum(d.y[idx]))) for idx in _groups(d)]
        ll = float(np.sum(d.y * xb))
        g = X.T @ d.y
    elif d.model_type == MODEL_COX:
        sets = [(np.array([a]), r, wt[a]) for a, r in _cox_sets(d, wt)]
        ll = float(np.sum([n * xb[a[0]] for a, _, n in sets]))
        g = np.sum([n * X[a[0]] for a, _, n in sets], axis=0)
    else:
        raise ValueError(d.model_type)
    H = np.zeros((d.J, d.J))
    for _, r, n in sets:
        rw = wt[r] if d.model_type == MODEL_COX else np.ones(len(r))
        w = rw * np.exp(xb[r] - xb[r].max())
        p = w / w.sum()
        m = X[r].T @ p
        ll -= n * (np.log(w.sum()) + xb[r].max())
        g = g - n * m
        H -= n * ((X[r].T * p) @ X[r] - np.outer(m, m))
    return ll, g, H


def newton_mle(d, fixed=None, weights=None, iters=100):
    """beta maximising the unpenalised (weighted) log-likelihood (fixed columns
    at 0), the log-likelihood there, and the observed information of the free
    columns."""
    X = design(d)
    free = np.ones(d.J, bool) if fixed is None else (np.asarray(fixed) == 0)
    beta = np.zeros(d.J)
    for _ in range(iters):
        ll, g, H = loglik_grad_hess(d, X, beta, weights)
        step = np.linalg.solve(-H[np.ix_(free, free)], g[free])
        beta[free] += step
        if np.max(np.abs(step)) < 1e-14 * max(1.0, np.max(np.abs(beta))):
            break
    ll, g, H = loglik_grad_hess(d, X, beta, weights)
    return beta, ll, -H[np.ix_(free, free)]
