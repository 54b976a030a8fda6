"""The row-major copy of the matrix (computeXBeta's row sums, the MM cycle)
built on the device, against a numpy construction of the same layout: per
row the columns in increasing order, dense-like columns at every row, the
values bit for bit; rows longer than the device sort takes are built on the
host with the same layout."""
import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import DENSE, INTERCEPT, MODEL_LOGISTIC, MODEL_POISSON, SPARSE

pytestmark = pytest.mark.gpu


def expected_row_major(d):
    K, J = d.K, d.J
    rs, cs, vs = [], [], []
    for j in range(J):
        f = int(d.fmt[j])
        if f in (DENSE, INTERCEPT):
            r = np.arange(K)
        else:
            r = np.asarray(d.rows[d.col_start[j]:d.col_start[j + 1]], np.int64)
        if f in (SPARSE, DENSE):
            v = np.asarray(d.vals[d.val_start[j]:d.val_start[j] + r.size], np.float64)
        else:
            v = np.ones(r.size)
        rs.append(r)
        cs.append(np.full(r.size, j, np.int64))
        vs.append(v)
    r, c, v = np.concatenate(rs), np.concatenate(cs), np.concatenate(vs)
    order = np.lexsort((c, r))
    row_ptr = np.concatenate([[0], np.cumsum(np.bincount(r, minlength=K))]).astype(np.int64)
    return row_ptr, c[order].astype(np.int32), v[order]


CASES = [
    # every format, an intercept
    ("mixed", lambda: synthetic.small(MODEL_POISSON, seed=31, K=3000, P=60, density=0.05, offset=True)),
    # the MM workload's shape, scaled down: matched sets, indicator columns
    ("clr", lambda: synthetic.conditional_logistic(seed=32, n_sets=4000, P=600)),
    # rows longer than the device sort takes (1,201 entries): the host build
    ("long rows", lambda: synthetic.small(MODEL_LOGISTIC, seed=33, K=400, P=1200, density=0.9,
                                          formats=("dense", "sparse"))),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_row_major_copy_matches_numpy(gpu_ctx, name, make):
    d = make()
    m = native.Matrix(gpu_ctx, d)
    try:
        row_ptr, col, val = m.row_major()
    finally:
        m.close()
    want_ptr, want_col, want_val = expected_row_major(d)
    assert np.array_equal(row_ptr, want_ptr)
    assert np.array_equal(col, want_col)
    assert np.array_equal(val, want_val)
