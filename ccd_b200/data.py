"""Host-side problem container for the coordinate-descent path.

``CyclopsData`` holds one regression problem in the reference's own layout:
an outcome vector, optional survival times and stratum ids, and a column-major
``CompressedDataMatrix`` whose columns each carry a FormatType (DENSE, SPARSE,
INDICATOR, INTERCEPT -- ``src/cyclops/CompressedDataMatrix.h:36-38``).  Column
order is the order the reference arrives at after ``ModelData::loadX`` and
``setOffsetCovariate`` (``src/cyclops/ModelData.cpp:246-370, 640-651``):
``[offset?, intercept?, covariates...]``; when an offset is present, column 0
is it and its coefficient is pinned to 1 (``CyclicCoordinateDescent.cpp:218-221``).

Rows of survival models must already be sorted by (stratum, -time, y), the
order ``R/DataManagement.R:166`` establishes before loading.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# src/cyclops/Types.h:134-147
MODEL_POISSON = 2
MODEL_LOGISTIC = 3
MODEL_CONDITIONAL_LOGISTIC = 4
MODEL_CONDITIONAL_POISSON = 6
MODEL_COX = 8
MODEL_NAMES = {
    "poisson": MODEL_POISSON,
    "logistic": MODEL_LOGISTIC,
    "clr": MODEL_CONDITIONAL_LOGISTIC,
    "conditional_logistic": MODEL_CONDITIONAL_LOGISTIC,
    "conditional_poisson": MODEL_CONDITIONAL_POISSON,
    "cox": MODEL_COX,
}

# src/cyclops/CompressedDataMatrix.h:36-38
DENSE, SPARSE, INDICATOR, INTERCEPT = 0, 1, 2, 3
# priors::PriorType, src/cyclops/Types.h:100-105
PRIOR_NONE, PRIOR_LAPLACE, PRIOR_NORMAL = 0, 1, 2
# ConvergenceType, src/cyclops/Types.h:108-114
GRADIENT, LANGE, MITTAL = 0, 1, 2
# UpdateReturnFlags, src/cyclops/Types.h:124-130
SUCCESS, FAIL, MAX_ITERATIONS, ILLCONDITIONED, MISSING_COVARIATES = 0, 1, 2, 3, 4


@dataclass
class CyclopsData:
    model_type: int
    y: np.ndarray
    col_start: np.ndarray  # int64[J+1] offsets into rows (SPARSE/INDICATOR)
    rows: np.ndarray  # int32 row ids, ascending within a column
    val_start: np.ndarray  # int64[J+1] offsets into vals (SPARSE: per entry, DENSE: K)
    vals: np.ndarray  # float64
    fmt: np.ndarray  # uint8[J]
    prior_type: np.ndarray  # int32[J]
    prior_var: np.ndarray  # float64[J]
    time: Optional[np.ndarray] = None
    stratum: Optional[np.ndarray] = None
    offset_col0: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def K(self) -> int:
        return int(self.y.shape[0])

    @property
    def J(self) -> int:
        return int(self.fmt.shape[0])

    @property
    def nnz(self) -> int:
        return int(self.col_start[-1])

    def validate(self) -> None:
        K, J = self.K, self.J
        assert self.col_start.shape == (J + 1,) and self.val_start.shape == (J + 1,)
        assert self.rows.dtype == np.int32 and self.col_start.dtype == np.int64
        for j in range(J):
            f = int(self.fmt[j])
            nr = self.col_start[j + 1] - self.col_start[j]
            nv = self.val_start[j + 1] - self.val_start[j]
            if f in (DENSE, INTERCEPT):
                assert nr == 0
                assert nv == (K if f == DENSE else 0)
            elif f == INDICATOR:
                assert nv == 0
            else:
                assert nv == nr
            r = self.rows[self.col_start[j]:self.col_start[j + 1]]
            if r.size:
                assert r[0] >= 0 and r[-1] < K and np.all(np.diff(r) > 0)
        if self.model_type == MODEL_COX:
            assert self.time is not None and self.stratum is not None

    def with_prior(self, prior_type: int, variance: float) -> "CyclopsData":
        """Copy with one prior on every covariate; intercept/offset keep none."""
        pt = np.full(self.J, prior_type, np.int32)
        pv = np.full(self.J, float(variance))
        for j in range(self.J):
            if self.fmt[j] == INTERCEPT or (self.offset_col0 and j == 0):
                pt[j] = PRIOR_NONE
        d = CyclopsData(**{**self.__dict__})
        d.prior_type, d.prior_var = pt, pv
        return d


def build_columns(K: int, columns, formats) -> tuple:
    """Assemble CSC arrays from per-column (rows, values) pairs.

    ``columns[j]`` is ``(rows int array, values float array or None)``;
    DENSE columns pass ``(None, values[K])``, INTERCEPT ``(None, None)``.
    """
    J = len(columns)
    col_start = np.zeros(J + 1, np.int64)
    val_start = np.zeros(J + 1, np.int64)
    rparts, vparts = [], []
    for j, ((r, v), f) in enumerate(zip(columns, formats)):
        nr = 0 if r is None else len(r)
        if f == DENSE:
            nv = K
        elif f == SPARSE:
            nv = nr
        else:
            nv = 0
        col_start[j + 1] = col_start[j] + nr
        val_start[j + 1] = val_start[j] + nv
        if nr:
            rparts.append(np.asarray(r, np.int32))
        if nv:
            vparts.append(np.asarray(v, np.float64))
    rows = np.concatenate(rparts) if rparts else np.zeros(0, np.int32)
    vals = np.concatenate(vparts) if vparts else np.zeros(0, np.float64)
    return col_start, rows, val_start, vals, np.asarray(formats, np.uint8)


def csc_from_coo(K: int, J: int, col: np.ndarray, row: np.ndarray) -> tuple:
    """Sorted, de-duplicated CSC (col_start, rows) from COO indices."""
    key = col.astype(np.int64) * K + row.astype(np.int64)
    key.sort()
    if key.size:
        keep = np.empty(key.size, bool)
        keep[0] = True
        np.not_equal(key[1:], key[:-1], out=keep[1:])
        key = key[keep]
    c = (key // K).astype(np.int64)
    r = (key % K).astype(np.int32)
    counts = np.bincount(c, minlength=J)
    col_start = np.zeros(J + 1, np.int64)
    np.cumsum(counts, out=col_start[1:])
    return col_start, r


def cox_sort_order(stratum: np.ndarray, time: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Row order (stratum, -time, y): ``order(pid, -time, y)`` in R/DataManagement.R:166."""
    return np.lexsort((y, -time, stratum))


def cox_groups(stratum: np.ndarray, time: np.ndarray, y: np.ndarray,
               weights: Optional[np.ndarray] = None):
    """Risk-set tie groups exactly as ``setPidForAccumulation`` forms them.

    Restates ``src/cyclops/engine/ModelSpecifics.hpp:1809-1868`` on rows already
    sorted by (stratum, -time, y).  Returns ``(group[K] int32, acc_reset int32,
    N)``: rows with zero weight get group ``N``; ``acc_reset`` lists the first
    group of every stratum after the first, followed by ``N``.  Integer work,
    bit-exact with the reference.
    """
    K = int(y.shape[0])
    keep = np.ones(K, bool) if weights is None else (np.asarray(weights) != 0.0)
    group = np.full(K, -1, np.int64)
    idx = np.nonzero(keep)[0]
    if idx.size == 0:
        return np.zeros(K, np.int32), np.array([0], np.int32), 0
    s = stratum[idx]
    t = time[idx]
    yy = y[idx]
    new_stratum = np.zeros(idx.size, bool)
    new_stratum[1:] = s[1:] != s[:-1]
    tie = np.zeros(idx.size, bool)
    tie[1:] = (yy[:-1] == 1.0) & (t[1:] == t[:-1]) & (yy[1:] == yy[:-1])
    inc = np.ones(idx.size, np.int64)
    inc[0] = 0
    inc[1:] = np.where(new_stratum[1:] | ~tie[1:], 1, 0)
    g = np.cumsum(inc)
    N = int(g[-1]) + 1
    group[idx] = g
    group[group < 0] = N
    acc_reset = np.concatenate([g[new_stratum], [N]]).astype(np.int32)
    return group.astype(np.int32), acc_reset, N
