"""Dependency levels of the fused sweep (host logic, no GPU): columns on one
level are disjoint, conflicting columns keep their visiting order, and every
column sits exactly one level above its latest conflicting predecessor."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import DENSE, INTERCEPT, MODEL_LOGISTIC, MODEL_POISSON


def rows_of(d, j):
    if d.fmt[j] in (DENSE, INTERCEPT):
        return np.arange(d.K)
    return d.rows[d.col_start[j]:d.col_start[j + 1]]


@pytest.mark.parametrize("make", [
    lambda: synthetic.small(MODEL_LOGISTIC, seed=1, K=200, P=40, density=0.05),
    lambda: synthetic.small(MODEL_POISSON, seed=2, K=150, P=30, offset=True, formats=("sparse", "dense", "indicator")),
    lambda: synthetic.logistic_l1(seed=3, K=2000, P=300),
])
def test_levels_reproduce_visiting_order(make):
    d = make()
    lv, n = native.sweep_levels(d)
    active = [j for j in range(d.J) if not (d.offset_col0 and j == 0)]
    assert lv.max() + 1 == n
    last = {}  # row -> level of the latest column touching it
    floor = -1
    for j in active:
        r = rows_of(d, j)
        want = max([floor] + [last.get(int(k), -1) for k in r]) + 1
        assert lv[j] == want, j
        for k in r:
            last[int(k)] = lv[j]
        if d.fmt[j] in (DENSE, INTERCEPT):
            floor = lv[j]
    # disjointness on each level
    for L in range(n):
        seen = set()
        for j in active:
            if lv[j] == L:
                s = set(map(int, rows_of(d, j)))
                assert not (s & seen)
                seen |= s
    if d.offset_col0:
        assert lv[0] == -1
