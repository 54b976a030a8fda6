"""Malformed matrices are refused before any device work (host-side failure
injection, no GPU): every rule of the CompressedDataMatrix contract through
ccdb_matrix_validate, the check ccdb_matrix_create runs first."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import DENSE, INDICATOR, INTERCEPT, MODEL_LOGISTIC, SPARSE, CyclopsData, build_columns


def _data(cols, fmts, K=10):
    cs, r, vs, v, fm = build_columns(K, cols, fmts)
    J = len(fmts)
    return CyclopsData(MODEL_LOGISTIC, np.zeros(K), cs, r, vs, v, fm, np.zeros(J, np.int32), np.ones(J))


def _refused(d, match):
    with pytest.raises(native.CcdbError) as ei:
        native.validate_matrix(d)
    assert ei.value.code == native.ERR_INVALID and match in str(ei.value)


def test_valid_problems_pass():
    for d in (synthetic.small(MODEL_LOGISTIC, seed=170), synthetic.logistic_l1(seed=1, K=500, P=50),
              _data([(None, None), (np.array([], np.int32), None)], [INTERCEPT, INDICATOR])):
        native.validate_matrix(d)


def test_unsorted_duplicate_and_out_of_range_rows():
    _refused(_data([(np.array([3, 1], np.int32), None)], [INDICATOR]), "ascending")
    _refused(_data([(np.array([2, 2], np.int32), None)], [INDICATOR]), "ascending")
    _refused(_data([(np.array([1, 10], np.int32), None)], [INDICATOR]), "< K")
    _refused(_data([(np.array([-1, 2], np.int32), None)], [INDICATOR]), "ascending")


def test_format_contracts():
    d = _data([(np.array([1, 2], np.int32), np.array([0.5, 2.0]))], [SPARSE])
    d.fmt = np.array([INDICATOR], np.uint8)  # values on an indicator column
    _refused(d, "INDICATOR")
    d = _data([(None, np.ones(10))], [DENSE])
    d.val_start = np.array([0, 9], np.int64)  # short dense column
    d.vals = d.vals[:9]
    _refused(d, "DENSE")
    d = _data([(None, None)], [INTERCEPT])
    d.fmt = np.array([7], np.uint8)
    _refused(d, "unknown column format")


def test_offsets():
    d = _data([(np.array([1, 2], np.int32), None), (np.array([3], np.int32), None)], [INDICATOR, INDICATOR])
    d.col_start = np.array([0, 2, 1], np.int64)  # decreasing
    _refused(d, "non-decreasing")
    d = _data([(np.array([1], np.int32), None)], [INDICATOR])
    d.col_start = np.array([1, 2], np.int64)
    _refused(d, "bad offsets")


def _big(J=400, per=12_000, K=2_000_000, seed=5):
    """~4.8e6 indicator entries: enough that the row-id check runs on several
    host threads."""
    rng = np.random.default_rng(seed)
    cols = [(np.sort(rng.choice(K, size=per, replace=False)).astype(np.int32), None) for _ in range(J)]
    return _data(cols, [INDICATOR] * J, K=K)


def test_large_matrix_checks_in_column_order():
    d = _big()
    native.validate_matrix(d)
    cs = np.asarray(d.col_start)
    # a row-id error in the last column is found
    bad = _big()
    bad.rows = np.array(bad.rows)
    bad.rows[cs[-1] - 1] = bad.rows[cs[-1] - 2]
    _refused(bad, "ascending")
    # an out-of-range row early and a format error late: the earlier column is reported
    bad = _big()
    bad.rows = np.array(bad.rows)
    bad.rows[cs[3] - 1] = bad.K
    bad.fmt = np.array(bad.fmt)
    bad.fmt[-1] = 7
    _refused(bad, "< K")
    # a format error early and a row error late: the format error is reported
    bad = _big()
    bad.rows = np.array(bad.rows)
    bad.rows[cs[-1] - 1] = -5
    bad.fmt = np.array(bad.fmt)
    bad.fmt[2] = 7
    _refused(bad, "unknown column format")


def test_offsets_beyond_the_total_are_refused():
    """A column whose end offset passes the total would read past the row ids."""
    d = _data([(np.array([1, 2], np.int32), None), (np.array([3], np.int32), None)], [INDICATOR, INDICATOR])
    d.col_start = np.array([0, 100, 3], np.int64)
    _refused(d, "non-decreasing")
