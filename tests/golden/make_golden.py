"""Generate the golden fixtures from the reference engine compiled from source.

    make -C oracle ref && python tests/golden/make_golden.py

Every case stores its inputs (the CompressedDataMatrix, outcomes, strata,
times, priors, weights) and what the reference Cyclops engine
(oracle/_ref/libccd_ref.so) returns for them: the gradient/Hessian of every
coordinate at the starting state, and CyclicCoordinateDescent::update's
coefficients, log-likelihood, iteration count and return flag.  At that mode
it also stores the calls on a fitted state: the Fisher information over every
coefficient column (unweighted cases; the reference refuses weighted ones),
the predictive estimates, and the predictive log-likelihood on a fixed
held-out row set.  Run only where the reference sources are present; the
fixtures are committed.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ccd_b200 import synthetic  # noqa: E402
from ccd_b200.data import (GRADIENT, LANGE, MITTAL, MODEL_CONDITIONAL_LOGISTIC, MODEL_COX,  # noqa: E402
                           MODEL_LOGISTIC, MODEL_POISSON, PRIOR_LAPLACE, PRIOR_NORMAL)
from oracle.checker import FisherRefused, ReferenceEngine  # noqa: E402

CASES = [
    ("lr_mixed_laplace", MODEL_LOGISTIC, dict(seed=21), GRADIENT, None),
    ("lr_mixed_normal_mittal", MODEL_LOGISTIC, dict(seed=22, prior=PRIOR_NORMAL), MITTAL, None),
    ("lr_indicator_lange_weighted", MODEL_LOGISTIC, dict(seed=23, formats=("indicator",), P=25), LANGE, "folds"),
    ("poisson_offset_normal", MODEL_POISSON, dict(seed=24, offset=True, prior=PRIOR_NORMAL), GRADIENT, None),
    ("poisson_sparse_dense_mittal", MODEL_POISSON, dict(seed=25, formats=("sparse", "dense")), MITTAL, None),
    ("clr_laplace", MODEL_CONDITIONAL_LOGISTIC, dict(seed=26, n_strata=40), GRADIENT, None),
    ("clr_normal_mittal", MODEL_CONDITIONAL_LOGISTIC, dict(seed=27, n_strata=25, prior=PRIOR_NORMAL), MITTAL, None),
    ("cox_strata_ties", MODEL_COX, dict(seed=28, n_strata=6, tie_days=3), GRADIENT, None),
    ("cox_one_stratum_normal", MODEL_COX, dict(seed=29, n_strata=1, prior=PRIOR_NORMAL), MITTAL, None),
    ("cox_weighted_lange", MODEL_COX, dict(seed=30, K=500, n_strata=8, tie_days=2), LANGE, "random"),
]


def weights_for(kind, K, seed):
    if kind is None:
        return None
    rng = np.random.default_rng(seed)
    if kind == "folds":
        return (rng.integers(0, 10, size=K) != 3).astype(float)
    return (rng.random(K) > 0.25).astype(float)


def heldout_for(K):
    """A fixed held-out row set: every fifth row."""
    return (np.arange(K) % 5 == 2).astype(float)


def digest(arrs) -> str:
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    index = {}
    for name, model, kw, conv, wkind in CASES:
        d = synthetic.small(model, **kw)
        w = weights_for(wkind, d.K, 99)
        e = ReferenceEngine(d)
        if w is not None:
            e.set_weights(w)
        gh = np.array([e.grad_hess(j) for j in range(d.J)])
        e.close()
        e = ReferenceEngine(d)
        if w is not None:
            e.set_weights(w)
        r = e.fit(conv, 1e-6)
        cols = np.arange(1 if d.offset_col0 else 0, d.J, dtype=np.int32)
        try:
            fisher = e.fisher_information(cols)
        except FisherRefused:
            fisher = None
        pred_est = e.predictive_estimates()
        held = heldout_for(d.K)
        pred_ll = e.predictive_loglik(held)
        e.close()
        arrays = dict(model_type=np.int32(d.model_type), y=d.y, col_start=d.col_start, rows=d.rows,
                      val_start=d.val_start, vals=d.vals, fmt=d.fmt, prior_type=d.prior_type,
                      prior_var=d.prior_var, offset_col0=np.int32(d.offset_col0),
                      conv=np.int32(conv), gh0=gh, beta=r["beta"], loglik=np.float64(r["loglik"]),
                      iterations=np.int32(r["iterations"]), flag=np.int32(r["flag"]),
                      pred_est=pred_est, heldout=held, pred_ll=np.float64(pred_ll))
        if fisher is not None:
            arrays["fisher_cols"] = cols
            arrays["fisher"] = fisher
        if d.time is not None:
            arrays["time"] = d.time
        if d.stratum is not None:
            arrays["stratum"] = d.stratum
        if w is not None:
            arrays["weights"] = w
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        index[name] = {"model": int(model), "conv": int(conv), "iterations": int(r["iterations"]),
                       "flag": int(r["flag"]), "loglik": r["loglik"]}
        print(name, index[name])
    # the 10,000 x 1,000 L1 logistic benchmark problem: inputs regenerated from the
    # seed (digest pinned), results from the reference
    d = synthetic.logistic_l1(seed=1)
    r = ReferenceEngine(d).fit(MITTAL, 1e-6)
    np.savez_compressed(os.path.join(HERE, "logistic_l1_10000x1000.npz"), beta=r["beta"],
                        loglik=np.float64(r["loglik"]), iterations=np.int32(r["iterations"]),
                        flag=np.int32(r["flag"]))
    index["logistic_l1_10000x1000"] = {
        "seed": 1, "input_sha256": digest([d.y, d.col_start, d.rows, d.fmt]),
        "iterations": int(r["iterations"]), "flag": int(r["flag"]), "loglik": r["loglik"]}
    with open(os.path.join(HERE, "index.json"), "w") as fh:
        json.dump(index, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
