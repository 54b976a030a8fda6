"""The cross-validation drivers sharded over ranks (cv.ShardedFit), on CPU:
two gloo ranks on 127.0.0.1 each drive a stand-in fit (no GPU) through the
grid search and the auto search; every rank must reach the result one
process reaches alone, see every instance exactly once between them, and
return the coefficients and results in instance order."""
import datetime
import math
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ccd_b200 import cv, synthetic
from ccd_b200.data import MODEL_LOGISTIC, MODEL_POISSON


class StandInFit:
    """Deterministic results from (variance, held-out fold) alone: the held-out
    log-likelihood peaks at variance 0.3; coefficients encode the instance."""

    def __init__(self, d, rank=0):
        self.d = d
        self.rank = rank
        self.seen = []

    def _one(self, v, h):
        pred = -(math.log(v) - math.log(0.3)) ** 2 - 0.01 * h
        flag = 1 if (h == 3 and v > 5.0) else 0  # a failed fit: NaN in the driver
        return {"flag": flag, "iterations": 3, "loglik": -1.0, "objective": 0.0, "pred_loglik": pred}

    def batch_find_mode(self, variance, holdout=None, row_fold=None, args=None, group=0, cluster=0):
        var = np.asarray(variance, dtype=np.float64)
        hold = np.zeros(len(var), int) if holdout is None else np.asarray(holdout)
        self.seen += [(float(v), int(h)) for v, h in zip(var, hold)]
        beta = np.outer(var * (1 + hold), np.ones(self.d.J))
        return beta, [self._one(v, h) for v, h in zip(var, hold)], 0.1 * len(var) * (1 + self.rank)

    def fold_instances(self, variances, holdout, row_fold, args=None):
        var = np.asarray(variances, dtype=np.float64)
        v = var[:, -1]
        return self.batch_find_mode(v, holdout, row_fold, args)


def _problems():
    d1 = synthetic.small(MODEL_LOGISTIC, seed=20, K=120, P=6)
    d2 = synthetic.small(MODEL_POISSON, seed=21, K=100, P=5, offset=True)
    d2.prior_var[-1] = 2.0  # two variance parameters: standalone instances
    return d1, d2


def _drive(fit, d):
    fold = np.arange(d.K) % 5
    g = cv.grid_search(fit, fold, 5, lower=0.01, upper=20.0, steps=7)
    a = cv.auto_search(fit, d, fold, 5, starting_variance=1.0)
    return g, a


def _summary(res):
    return (res.variance, res.value, [tuple(t) for t in res.tried], res.fits, list(res.variances))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = []
        for d in _problems():
            local = StandInFit(d, rank)
            sf = cv.ShardedFit(local)
            g, a = _drive(sf, d)
            seen = list(local.seen)
            beta, res, secs = sf.batch_find_mode(np.array([0.1, 0.2, 0.3, 0.4, 0.5]), np.arange(5), None)
            out.append((_summary(g), _summary(a), seen, beta, [r["pred_loglik"] for r in res], secs))
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array(out, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(180)
def test_sharded_drivers_match_one_process(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    outs = [np.load(tmp_path / f"r{r}.npy", allow_pickle=True) for r in range(world)]
    for p, d in enumerate(_problems()):
        alone = StandInFit(d)
        g, a = _drive(alone, d)
        want_g, want_a = _summary(g), _summary(a)
        for r in range(world):
            got_g, got_a, _, beta, pred, secs = outs[r][p]
            assert tuple(got_g) == tuple(want_g) or list(got_g) == list(want_g)
            assert list(got_a) == list(want_a)
            # instance order restored on every rank; the slowest rank's time
            np.testing.assert_array_equal(beta, np.outer(np.array([0.1, 0.2, 0.3, 0.4, 0.5]) * np.arange(1, 6),
                                                         np.ones(d.J)))
            assert pred == [alone._one(v, h)["pred_loglik"] for v, h in zip([0.1, 0.2, 0.3, 0.4, 0.5], range(5))]
            assert secs == pytest.approx(0.1 * 2 * world)  # rank 1's 2 instances x 0.1 x 2
        # between them the ranks fitted every instance of the drivers exactly once
        seen = sorted(outs[0][p][2] + outs[1][p][2])
        assert seen == sorted(alone.seen)
        assert len(outs[0][p][2]) and len(outs[1][p][2])
