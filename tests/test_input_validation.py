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
