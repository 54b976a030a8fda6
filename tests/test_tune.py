"""The launch-shape tuners (ccd_b200/tune.py) on CPU, over stand-in fits: the
column-nnz histogram key, the fastest candidate by measured device time, the
cache keyed on the histogram (a second matrix with the same histogram reuses
the choice without measuring), and candidates a device refuses skipped."""
import dataclasses

import numpy as np
import pytest

from ccd_b200 import native, synthetic, tune
from ccd_b200.data import MODEL_LOGISTIC


@pytest.fixture(autouse=True)
def fresh_cache():
    tune.clear_cache()
    yield
    tune.clear_cache()


def test_histogram_bins():
    d = synthetic.small(MODEL_LOGISTIC, seed=1, K=300, P=6, density=0.1, formats=("indicator",))
    h = tune.nnz_histogram(d)
    cnt = np.diff(d.col_start)
    cnt[0] = d.K  # the intercept counts every row
    assert h.sum() == d.J
    for c in cnt:
        b = 0 if c == 0 else int(np.floor(np.log2(c))) + 1
        assert h[b] >= 1
    assert tune.histogram_key(d)[:2] == (d.K, d.J)


class StandInBatch:
    def __init__(self, d, secs, refuse=()):
        self.d, self.secs, self.refuse, self.calls = d, secs, set(refuse), []
        self.precision = native.PRECISION_MIXED

    def batch_find_mode(self, var, hold, fold, args, group=0, cluster=0):
        self.calls.append((group, cluster, args.max_iterations))
        if (group, cluster) in self.refuse:
            raise native.CcdbError(native.ERR_UNSUPPORTED, "no")
        return None, [], self.secs[(group, cluster)]


def test_tune_batch_picks_the_fastest_and_caches_by_histogram():
    d = synthetic.small(MODEL_LOGISTIC, seed=2, K=400, P=8)
    secs = {(g, c): 1.0 + 0.1 * g + 0.01 * c for g, c in tune.batch_candidates()}
    secs[(2, 4)] = 0.5
    f = StandInBatch(d, secs, refuse={(4, 8)})
    var = np.full(10, 0.1)
    ch = tune.tune_batch(f, var, np.arange(10), np.zeros(d.K, int))
    assert (ch.group, ch.cluster) == (2, 4) and not ch.cached
    assert (4, 8) not in ch.seconds and len(ch.seconds) == 11
    assert all(mi == 1 for _, _, mi in f.calls)  # one sweep per trial
    # the same histogram and size: cached, no trial runs
    f2 = StandInBatch(dataclasses.replace(d), secs)
    ch2 = tune.tune_batch(f2, var, np.arange(10), np.zeros(d.K, int))
    assert ch2.cached and (ch2.group, ch2.cluster) == (2, 4) and f2.calls == []
    # another instance count measures again
    f3 = StandInBatch(d, secs)
    assert not tune.tune_batch(f3, np.full(12, 0.1), np.arange(12), np.zeros(d.K, int)).cached


class StandInCtx:
    def __init__(self):
        self.max_ctas = []

    def set_max_ctas(self, n):
        self.max_ctas.append(n)


class StandInFit:
    def __init__(self, d, ctx, t):
        self.d, self.ctx, self.t = d, ctx, t

    def find_mode(self, args, beta=None):
        assert args.max_iterations == 1 and args.strategy == native.SWEEP_LEVELS
        return native.FitResult(beta, 2, 1, 0.0, 0.0, self.d.J, 0.0, self.t[self.ctx.max_ctas[-1]])


def test_tune_sweep_sets_the_fastest_cluster_size():
    d = synthetic.small(MODEL_LOGISTIC, seed=3, K=500, P=10)
    ctx = StandInCtx()
    f = StandInFit(d, ctx, {16: 3e-3, 8: 2e-3, 4: 2.5e-3, 2: 4e-3})
    ch = tune.tune_sweep(ctx, f)
    assert ch.max_ctas == 8 and ctx.max_ctas[-1] == 8
    ctx2 = StandInCtx()
    ch2 = tune.tune_sweep(ctx2, StandInFit(d, ctx2, {}))
    assert ch2.cached and ctx2.max_ctas == [8]


def test_filling_keeps_shapes_that_occupy_every_sm():
    cands = list(tune.batch_candidates())
    # 200 instances on 148 SMs: 100 groups of 2 on one CTA each leave SMs idle
    kept = tune.filling(cands, 200, 148)
    assert (2, 1) not in kept and (4, 2) not in kept and (4, 1) not in kept
    assert (4, 4) in kept and (2, 2) in kept and (1, 1) in kept
    # nothing fills a tiny grid: every candidate stays
    assert tune.filling(cands, 2, 148) == cands


def test_tune_batch_ignores_shapes_that_leave_sms_idle():
    d = synthetic.small(MODEL_LOGISTIC, seed=3, K=400, P=8)
    secs = {(g, c): 1.0 for g, c in tune.batch_candidates()}
    secs[(2, 1)] = 0.1   # fastest single sweep, but 100 CTAs on 148 SMs
    secs[(4, 4)] = 0.5
    f = StandInBatch(d, secs)
    f.ctx = type("Ctx", (), {"sm_count": 148})()
    tune.clear_cache()
    ch = tune.tune_batch(f, np.full(200, 0.1), np.arange(200) % 10, np.zeros(d.K, int))
    assert (ch.group, ch.cluster) == (4, 4)
    assert (2, 1) not in ch.seconds
