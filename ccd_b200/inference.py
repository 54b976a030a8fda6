"""Asymptotic standard errors and covariance of a fitted model.

Mirrors the reference's R-level post-fit calls: ``getSEs`` (R/ModelFit.R:730-741)
and ``vcov.cyclopsFit`` (R/ModelFit.R:1005-1016) both take the Fisher
information of the chosen columns (``.cyclopsGetFisherInformation``, computed
here on the GPU by ``Fit.compute_fisher_information``) and invert it on the
host, as R's ``solve`` does.  The inversion is of an n x n matrix over the
requested columns; the O(nnz) work is the Fisher information itself.
"""
from __future__ import annotations

import warnings
from typing import Optional, Sequence

import numpy as np


def covariate_columns(fit) -> np.ndarray:
    """All coefficient columns of the fit: every column but the offset (which
    the reference holds outside the coefficients)."""
    first = 1 if fit.d.offset_col0 else 0
    return np.arange(first, fit.d.J, dtype=np.int32)


def vcov(fit, columns: Optional[Sequence[int]] = None) -> np.ndarray:
    """Inverse of the Fisher information over `columns` (default: every
    coefficient column), vcov.cyclopsFit."""
    cols = covariate_columns(fit) if columns is None else np.asarray(columns, dtype=np.int32)
    return np.linalg.inv(fit.compute_fisher_information(cols))


def standard_errors(fit, columns: Optional[Sequence[int]] = None) -> np.ndarray:
    """sqrt(diag(solve(Fisher information))) over `columns`, getSEs.  As the
    reference warns, the errors are only valid when every coefficient is
    included."""
    all_cols = covariate_columns(fit)
    cols = all_cols if columns is None else np.asarray(columns, dtype=np.int32)
    if len(cols) != len(all_cols):
        warnings.warn("Asymptotic standard errors are only valid if computed for all covariates "
                      "simultaneously")
    return np.sqrt(np.diag(np.linalg.inv(fit.compute_fisher_information(cols))))
