"""Host logic of the cross-validation drivers (no GPU): the uni-modal search
(utils/HParSearch.cpp) and the point estimates of AbstractCrossValidationDriver."""
import math

import numpy as np
import pytest

from ccd_b200 import cv, synthetic
from ccd_b200.data import MODEL_LOGISTIC


def test_quadratic_log_fit_recovers_a_quadratic():
    c = (-120.0, -3.0, -0.8)
    hist = {x: (c[0] + c[1] * math.log(x) + c[2] * math.log(x) ** 2, 0.5 + 0.1 * i)
            for i, x in enumerate([1e-3, 1e-2, 0.1, 1.0, 10.0])}
    got = cv.quadratic_log_fit(hist)
    assert np.allclose(got, c, rtol=1e-9, atol=1e-9)


def test_search_steps_follow_the_reference_rules():
    s = cv.UniModalSearch(10.0, 0.01, math.log(1.5))
    assert s.step() == (True, 1.0, 0.0)          # no point yet: start at 1
    s.tried(0.5, -10.0, 1.0)
    assert s.step()[1] == pytest.approx(5.0)     # one point below the first cut: x * step
    s.tried(5.0, -12.0, 1.0)
    assert s.step()[1] == pytest.approx(0.05)    # left point better: go left
    s.tried(0.05, -11.0, 1.0)                    # bracketed at 0.5: quadratic step
    cont, x, y = s.step()
    assert 0.05 < x < 5.0 and y >= -10.0


def test_maximum_at_the_edge_moves_outwards():
    s = cv.UniModalSearch(10.0)
    for x, y in [(1.0, -5.0), (10.0, -6.0), (100.0, -7.0)]:
        s.tried(x, y, 0.1)
    assert s.step()[1] == pytest.approx(0.1)


def test_point_estimate_ignores_nan():
    v = [1.0, float("nan"), 3.0]
    m = cv.point_estimate(v)
    assert m == 2.0 and cv.st_dev(v, m) == pytest.approx(1.0)


def test_default_variance_counts_indicator_entries():
    d = synthetic.small(MODEL_LOGISTIC, seed=3, K=200, P=6, formats=("indicator",))
    n_var = d.J - 1  # the intercept is not a variable column
    want = float(d.col_start[-1]) / n_var / d.K
    assert cv.normal_based_default_var(d) == pytest.approx(want)


def test_grid_points_are_log_uniform():
    g = cv.grid_points(0.01, 10.0, 4)
    assert np.allclose(np.diff(np.log(g)), math.log(10.0))
    assert cv.grid_points(0.01, 10.0, 1).tolist() == [10.0]
