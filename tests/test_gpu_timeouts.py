"""Bounded device-side waits that run out, on purpose, without faulting the GPU.

Every spin-wait of the engine's kernels gives up after a bound
(ccdb_fit_set_wait_limit), records where, and lets the kernel return; the host
turns that into CCDB_ERR_TIMEOUT and the context stays usable.  These tests set
the bound to one nanosecond, so that any wait not already satisfied on its
first look runs out, check the status, then restore the default bound and fit
the same problem correctly on the same context:

* the grid-wide level sweep (CCDB_SWEEP_GRID_LEVELS): its waits for a
  level's arrivals and for the grid barrier raise the launch's abort word and
  every CTA leaves;
* the persistent group sweep's grid form (Cox, CCDB_SWEEP_GRID_LEVELS): the
  same for its grid barriers;
* the mixed-precision batch engine on a cluster of two CTAs per group: a wait
  for the other CTA's column sums raises the abort word; every CTA of the
  cluster stops stepping, finishes the sweep's exchanges (nothing is left in
  flight towards a CTA that leaves), and after the sweep's closing cluster
  barrier all of them report the timeout together."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import MITTAL, MODEL_LOGISTIC

pytestmark = pytest.mark.gpu


def _rel(b, want):
    return np.max(np.abs(b - want)) / max(np.max(np.abs(want)), 1e-8)


def test_grid_sweep_wait_runs_out_then_recovers(gpu_ctx, oracle_engine):
    d = synthetic.small(MODEL_LOGISTIC, seed=80, K=3000, P=60)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    args = native.ModeFindingArguments(convergence_type=MITTAL, strategy=native.SWEEP_GRID_LEVELS)
    f.set_wait_limit(1)
    with pytest.raises(native.CcdbError) as ex:
        f.find_mode(args, beta=np.zeros(d.J))
    assert ex.value.code == native.ERR_TIMEOUT
    f.set_wait_limit(0)
    want = oracle_engine(d).fit(MITTAL, 1e-6)
    r = f.find_mode(args, beta=np.zeros(d.J))
    assert r.return_flag == want["flag"] == 0
    assert r.iterations == want["iterations"]
    assert _rel(r.beta, want["beta"]) <= 1e-6


def test_batch_cluster_exchange_wait_runs_out_then_recovers(gpu_ctx):
    d = synthetic.small(MODEL_LOGISTIC, seed=81, K=900, P=30)
    fold = synthetic.cv_folds(d.K, n_folds=4, seed=3)
    hold, var = synthetic.cv_grid(n_folds=4, n_vars=2, lower=0.05, upper=5.0)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d, precision=native.PRECISION_MIXED)
    b_want, r_want, _ = f.batch_find_mode(var, hold, fold, group=2, cluster=2)
    f.set_wait_limit(1)
    with pytest.raises(native.CcdbError) as ex:
        f.batch_find_mode(var, hold, fold, group=2, cluster=2)
    assert ex.value.code == native.ERR_TIMEOUT
    f.set_wait_limit(0)
    b, r, _ = f.batch_find_mode(var, hold, fold, group=2, cluster=2)
    assert np.array_equal(b, b_want)
    assert [x["iterations"] for x in r] == [x["iterations"] for x in r_want]
    assert all(x["flag"] == 0 for x in r)


def test_group_sweep_grid_wait_runs_out_then_recovers(gpu_ctx, oracle_engine):
    """The persistent group sweep's grid form (Cox): a grid barrier whose wait
    runs out raises the abort word and every CTA leaves; the cluster form has
    only hardware cluster barriers and no wait to bound."""
    from ccd_b200.data import MODEL_COX
    d = synthetic.small(MODEL_COX, seed=81, K=2000, P=30)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    args = native.ModeFindingArguments(convergence_type=MITTAL, strategy=native.SWEEP_GRID_LEVELS)
    f.set_wait_limit(1)
    with pytest.raises(native.CcdbError) as ex:
        f.find_mode(args, beta=np.zeros(d.J))
    assert ex.value.code == native.ERR_TIMEOUT
    f.set_wait_limit(0)
    want = oracle_engine(d).fit(MITTAL, 1e-6)
    r = f.find_mode(args, beta=np.zeros(d.J))
    assert r.return_flag == want["flag"] == 0
    assert r.iterations == want["iterations"]
    assert _rel(r.beta, want["beta"]) <= 1e-6
