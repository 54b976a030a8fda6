"""ctypes binding of libccdb.so (the C ABI in include/ccdb.h).

The objects mirror the reference's operator API: ``Fit`` exposes the
``AbstractModelSpecifics`` calls (``compute_gradient_and_hessian``,
``update_xbeta``, ``get_log_likelihood`` ...) and ``find_mode`` is
``CyclicCoordinateDescent::update``.  There is no CPU fallback: if the CUDA
library is missing or no GPU is present, constructing a ``Context`` raises.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import weakref
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .data import DENSE, INTERCEPT, CyclopsData, GRADIENT

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libccdb.so")

OK = 0
ERR_INVALID, ERR_CUDA, ERR_UNSUPPORTED, ERR_BUDGET, ERR_TIMEOUT = -1, -2, -3, -4, -5
ALGORITHM_CCD, ALGORITHM_MM = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
SWEEP_AUTO, SWEEP_LEVELS, SWEEP_SPECULATIVE, SWEEP_GRID_LEVELS, SWEEP_RESIDENT = 0, 1, 2, 3, 4


class CcdbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ccdb error {code}: {msg}")
        self.code = code


class _FitDesc(C.Structure):
    _fields_ = [("model_type", C.c_int32), ("precision", C.c_int32), ("y", C.c_void_p),
                ("time", C.c_void_p), ("stratum", C.c_void_p), ("offset_col0", C.c_int32)]


class _ModeArgs(C.Structure):
    _fields_ = [("prior_type", C.c_void_p), ("prior_var", C.c_void_p),
                ("convergence_type", C.c_int32), ("tolerance", C.c_double),
                ("max_iterations", C.c_int32), ("initial_bound", C.c_double),
                ("max_bound_count", C.c_int32), ("per_coordinate", C.c_int32),
                ("strategy", C.c_int32), ("algorithm", C.c_int32), ("use_kkt_swindle", C.c_int32),
                ("fixed", C.c_void_p)]


class _BatchDesc(C.Structure):
    _fields_ = [("n_instances", C.c_int32), ("row_fold", C.c_void_p), ("holdout", C.c_void_p),
                ("variance", C.c_void_p), ("group", C.c_int32), ("cluster", C.c_int32)]


class _BatchResult(C.Structure):
    _fields_ = [("return_flag", C.c_int32), ("iterations", C.c_int32),
                ("log_likelihood", C.c_double), ("objective", C.c_double),
                ("predictive_loglik", C.c_double), ("steps", C.c_int64), ("updates", C.c_int64),
                ("update_entries", C.c_int64), ("gradient_entries", C.c_int64)]


class _FitResult(C.Structure):
    _fields_ = [("return_flag", C.c_int32), ("iterations", C.c_int32),
                ("log_likelihood", C.c_double), ("objective", C.c_double),
                ("coordinate_updates", C.c_int64), ("device_seconds", C.c_double),
                ("kernel_seconds", C.c_double), ("kernel_launches", C.c_int64),
                ("attempts", C.c_int32), ("sweeps_total", C.c_int32), ("nonzero_steps", C.c_int64)]


@dataclass
class ModeFindingArguments:
    """CcdInterface.h:70-94 defaults."""
    convergence_type: int = GRADIENT
    tolerance: float = 1e-6
    max_iterations: int = 1000
    initial_bound: float = 2.0
    max_bound_count: int = 5
    per_coordinate: bool = False
    strategy: int = 0  # SWEEP_AUTO / SWEEP_LEVELS / SWEEP_SPECULATIVE
    algorithm: int = 0  # ALGORITHM_CCD / ALGORITHM_MM (AlgorithmType)
    kkt_swindle: bool = False  # ModeFindingArguments::useKktSwindle
    fixed: Optional[np.ndarray] = None  # J flags (setFixedBeta), None keeps the fit's set


@dataclass
class FitResult:
    beta: np.ndarray
    return_flag: int
    iterations: int
    log_likelihood: float
    objective: float
    coordinate_updates: int
    device_seconds: float
    kernel_seconds: float = 0.0
    kernel_launches: int = 0
    attempts: int = 1       # findMode runs (the ILLCONDITIONED retry adds some)
    sweeps_total: int = 0   # cycles over all of them
    nonzero_steps: int = -1  # steps that moved a coefficient (-1: not counted)


_lib = None

_P = C.c_void_p


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ccd_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.ccdb_last_error.restype = C.c_char_p
        L.ccdb_context_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(_P)]
        L.ccdb_context_destroy.argtypes = [_P]
        L.ccdb_context_memory.argtypes = [_P, C.POINTER(C.c_size_t)]
        L.ccdb_context_sm_count.argtypes = [_P, C.POINTER(C.c_int32)]
        L.ccdb_context_set_max_ctas.argtypes = [_P, C.c_int32]
        L.ccdb_context_set_blocking_wait.argtypes = [_P, C.c_int32]
        L.ccdb_matrix_create.argtypes = [_P, C.c_int64, C.c_int32, _P, _P, _P, _P, _P, C.POINTER(_P)]
        L.ccdb_matrix_destroy.argtypes = [_P]
        L.ccdb_matrix_row_major.argtypes = [_P, _P, _P, _P]
        L.ccdb_fit_create.argtypes = [_P, _P, C.POINTER(_FitDesc), C.POINTER(_P)]
        L.ccdb_fit_destroy.argtypes = [_P]
        L.ccdb_set_weights.argtypes = [_P, _P]
        L.ccdb_set_beta.argtypes = [_P, _P]
        L.ccdb_compute_xbeta.argtypes = [_P, _P]
        L.ccdb_compute_gradient_hessian.argtypes = [_P, C.c_int32, _P, _P]
        L.ccdb_update_xbeta.argtypes = [_P, C.c_int32, C.c_double]
        L.ccdb_compute_remaining_statistics.argtypes = [_P]
        L.ccdb_get_log_likelihood.argtypes = [_P, _P]
        L.ccdb_get_xbeta.argtypes = [_P, _P]
        L.ccdb_get_beta.argtypes = [_P, _P]
        L.ccdb_get_gradient_objective.argtypes = [_P, _P]
        L.ccdb_find_mode.argtypes = [_P, C.POINTER(_ModeArgs), _P, C.POINTER(_FitResult)]
        L.ccdb_fit_model.argtypes = [_P, C.c_int64, C.c_int32, _P, _P, _P, _P, _P, C.POINTER(_FitDesc),
                                     _P, C.POINTER(_ModeArgs), _P, C.POINTER(_FitResult)]
        L.ccdb_batch_find_mode.argtypes = [_P, C.POINTER(_BatchDesc), C.POINTER(_ModeArgs), _P, _P, _P]
        L.ccdb_column_gradient_hessian_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_int64, _P, _P, _P,
                                                           C.c_double, _P, _P]
        L.ccdb_sweep_levels.argtypes = [C.c_int64, C.c_int32, _P, _P, _P, _P, _P, _P]
        L.ccdb_fisher_information.argtypes = [_P, _P, C.c_int32, _P]
        L.ccdb_get_predictive_log_likelihood.argtypes = [_P, _P, _P]
        L.ccdb_get_predictive_estimates.argtypes = [_P, _P, _P]
        L.ccdb_compute_mm_gradient_hessian.argtypes = [_P, _P, _P, _P]
        L.ccdb_get_last_call_seconds.argtypes = [_P, _P]
        L.ccdb_set_fixed.argtypes = [_P, _P]
        L.ccdb_fit_set_wait_limit.argtypes = [_P, C.c_int64]
        L.ccdb_matrix_validate.argtypes = [C.c_int64, C.c_int32, _P, _P, _P, _P, _P]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != OK:
        raise CcdbError(rc, lib().ccdb_last_error().decode(errors="replace"))


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


class Context:
    """One GPU; ``hbm_budget`` bytes bound every allocation made through it."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = _P()
        _check(lib().ccdb_context_create(device, hbm_budget, C.byref(h)))
        self.h = h
        self.device = device
        # matrices and fits made on this context: closed before it, whatever
        # order the interpreter releases the Python objects in
        self._children = weakref.WeakSet()

    @property
    def sm_count(self) -> int:
        v = C.c_int32()
        _check(lib().ccdb_context_sm_count(self.h, C.byref(v)))
        return v.value

    def set_blocking_wait(self, on: bool = True) -> None:
        """Host waits sleep until the device signals instead of spinning
        (ccdb_context_set_blocking_wait); for many concurrent contexts."""
        _check(lib().ccdb_context_set_blocking_wait(self.h, int(bool(on))))

    def set_max_ctas(self, max_ctas: int) -> None:
        """Persistent sweep grids of this context's fits use at most max_ctas CTAs."""
        _check(lib().ccdb_context_set_max_ctas(self.h, int(max_ctas)))

    def memory_in_use(self) -> int:
        v = C.c_size_t()
        _check(lib().ccdb_context_memory(self.h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            kids = list(getattr(self, "_children", ()))
            for c in sorted(kids, key=lambda c: isinstance(c, Matrix)):  # fits, then matrices
                c.close()
            lib().ccdb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Matrix:
    """Device-resident CompressedDataMatrix, shared by fits."""

    def __init__(self, ctx: Context, d: CyclopsData):
        self.ctx = ctx
        self.K, self.J = d.K, d.J
        dense_like = np.isin(np.asarray(d.fmt), (DENSE, INTERCEPT))
        self.entries = int(np.sum(np.where(dense_like, d.K, np.diff(np.asarray(d.col_start)))))
        arrs = [_c(d.col_start, np.int64), _c(d.rows, np.int32), _c(d.val_start, np.int64),
                _c(d.vals, np.float64), _c(d.fmt, np.uint8)]
        h = _P()
        _check(lib().ccdb_matrix_create(ctx.h, d.K, d.J, *[_p(a) for a in arrs], C.byref(h)))
        self.h = h
        ctx._children.add(self)

    def row_major(self):
        """The row-major copy (row offsets, columns, values) the engine builds on
        the device for computeXBeta and the MM cycle."""
        total = int(self.entries)
        row_ptr = np.zeros(self.K + 1, np.int64)
        col = np.zeros(max(total, 1), np.int32)
        val = np.zeros(max(total, 1), np.float64)
        _check(lib().ccdb_matrix_row_major(self.h, _p(row_ptr), _p(col), _p(val)))
        return row_ptr, col[:total], val[:total]

    def close(self):
        if getattr(self, "h", None):
            lib().ccdb_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _desc(d: CyclopsData, precision: int, keep: list) -> _FitDesc:
    y = _c(d.y, np.float64)
    t = _c(d.time, np.float64)
    s = _c(d.stratum, np.int64)
    keep += [y, t, s]
    return _FitDesc(d.model_type, precision, _p(y), _p(t), _p(s), int(d.offset_col0))


def _mode_args(d: CyclopsData, a: ModeFindingArguments, keep: list) -> _ModeArgs:
    pt = _c(d.prior_type, np.int32)
    pv = _c(d.prior_var, np.float64)
    fx = None if a.fixed is None else np.ascontiguousarray(a.fixed, dtype=np.uint8)
    keep += [pt, pv, fx]
    return _ModeArgs(_p(pt), _p(pv), a.convergence_type, a.tolerance, a.max_iterations,
                     a.initial_bound, a.max_bound_count, int(a.per_coordinate), int(a.strategy),
                     int(a.algorithm), int(a.kkt_swindle), _p(fx))


class Fit:
    """Per-fit device state: the B200 counterpart of ModelSpecifics<Model,Real>
    driven by CyclicCoordinateDescent."""

    def __init__(self, ctx: Context, matrix: Matrix, d: CyclopsData,
                 precision: int = PRECISION_FP64):
        self.ctx, self.matrix, self.d = ctx, matrix, d
        keep = []
        desc = _desc(d, precision, keep)
        h = _P()
        _check(lib().ccdb_fit_create(ctx.h, matrix.h, C.byref(desc), C.byref(h)))
        self.h = h
        ctx._children.add(self)

    def close(self):
        if getattr(self, "h", None):
            lib().ccdb_fit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- AbstractModelSpecifics-level calls
    def set_weights(self, w: Optional[np.ndarray]) -> None:
        w = _c(w, np.float64)
        _check(lib().ccdb_set_weights(self.h, _p(w)))

    def set_beta(self, beta: np.ndarray) -> None:
        b = _c(beta, np.float64)
        _check(lib().ccdb_set_beta(self.h, _p(b)))

    def compute_xbeta(self, beta: np.ndarray) -> None:
        """xBeta from beta as the MM cycle forms it (ModelSpecifics::computeXBeta:
        with INDICATOR and no DENSE columns every non-zero entry counts 1)."""
        b = _c(beta, np.float64)
        _check(lib().ccdb_compute_xbeta(self.h, _p(b)))

    def compute_gradient_and_hessian(self, j: int):
        g, h = C.c_double(), C.c_double()
        _check(lib().ccdb_compute_gradient_hessian(self.h, j, C.byref(g), C.byref(h)))
        return g.value, h.value

    def update_xbeta(self, j: int, delta: float) -> None:
        _check(lib().ccdb_update_xbeta(self.h, j, delta))

    def compute_remaining_statistics(self) -> None:
        _check(lib().ccdb_compute_remaining_statistics(self.h))

    def get_log_likelihood(self) -> float:
        v = C.c_double()
        _check(lib().ccdb_get_log_likelihood(self.h, C.byref(v)))
        return v.value

    def get_xbeta(self) -> np.ndarray:
        out = np.zeros(self.d.K)
        _check(lib().ccdb_get_xbeta(self.h, _p(out)))
        return out

    def get_gradient_objective(self) -> float:
        v = C.c_double()
        _check(lib().ccdb_get_gradient_objective(self.h, C.byref(v)))
        return v.value

    def get_beta(self) -> np.ndarray:
        out = np.zeros(self.d.J)
        _check(lib().ccdb_get_beta(self.h, _p(out)))
        return out

    # --- calls on a fitted state
    def compute_fisher_information(self, indices) -> np.ndarray:
        """CyclicCoordinateDescent::computeFisherInformation(indices)
        (CyclicCoordinateDescent.cpp:1288-1299): the n x n Fisher information
        over the columns `indices` on the current state.  Weighted fits raise
        CcdbError(ERR_UNSUPPORTED), as the reference refuses them."""
        idx = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1)
        out = np.zeros((len(idx), len(idx)))
        _check(lib().ccdb_fisher_information(self.h, _p(idx), len(idx), _p(out)))
        return out

    def compute_mm_gradient_and_hessian(self, fixed: Optional[np.ndarray] = None):
        """ModelSpecifics::computeMMGradientAndHessian: the MM algorithm's
        gradient and Hessian bound of every column on the current state."""
        fx = _c(fixed, np.uint8)
        g, h = np.zeros(self.d.J), np.zeros(self.d.J)
        _check(lib().ccdb_compute_mm_gradient_hessian(self.h, _p(fx), _p(g), _p(h)))
        return g, h

    def set_fixed(self, fixed: np.ndarray) -> None:
        """setFixedBeta for every column (the offset stays fixed)."""
        fx = _c(fixed, np.uint8)
        _check(lib().ccdb_set_fixed(self.h, _p(fx)))

    def set_wait_limit(self, nanoseconds: int) -> None:
        """Bound on every single device-side wait of later launches (0: the
        defaults, 20 s for the grid sweep, 2 s for the batch exchange)."""
        _check(lib().ccdb_fit_set_wait_limit(self.h, int(nanoseconds)))

    def last_call_seconds(self) -> float:
        """Device time of the kernels of the last compute_fisher_information."""
        v = C.c_double()
        _check(lib().ccdb_get_last_call_seconds(self.h, C.byref(v)))
        return v.value

    def get_predictive_log_likelihood(self, weights: np.ndarray) -> float:
        """getNewPredictiveLogLikelihood (CyclicCoordinateDescent.cpp:319-355)
        of the current beta on held-out row weights."""
        w = _c(weights, np.float64)
        v = C.c_double()
        _check(lib().ccdb_get_predictive_log_likelihood(self.h, _p(w), C.byref(v)))
        return v.value

    def get_predictive_estimates(self, weights: Optional[np.ndarray] = None,
                                 y: Optional[np.ndarray] = None) -> np.ndarray:
        """getPredictiveEstimates (ModelSpecifics.hpp:692-705): the model's
        prediction of every row; with weights, rows of weight zero keep y."""
        out = np.zeros(self.d.K) if y is None else np.array(y, dtype=np.float64)
        w = _c(weights, np.float64)
        _check(lib().ccdb_get_predictive_estimates(self.h, _p(w), _p(out)))
        return out

    # --- the cross-validation grid: many instances in one launch
    def batch_find_mode(self, variance, holdout=None, row_fold=None,
                        args: Optional[ModeFindingArguments] = None, group: int = 0, cluster: int = 0):
        """Fit len(variance) instances (fold held out, prior variance) together.
        ``group``: lockstep group size of a mixed-precision fit, ``cluster``: its CTAs
        per group (0: the engine's choice).
        Returns (beta[n, J], list of per-instance dicts, device seconds)."""
        args = args or ModeFindingArguments()
        keep = []
        ma = _mode_args(self.d, args, keep)
        var = _c(variance, np.float64)
        n = var.shape[0]
        hold = None if holdout is None else _c(holdout, np.int32)
        fold = None if row_fold is None else _c(row_fold, np.int32)
        bd = _BatchDesc(n, _p(fold), _p(hold), _p(var), int(group), int(cluster))
        beta = np.zeros((n, self.d.J))
        res = (_BatchResult * n)()
        secs = C.c_double()
        _check(lib().ccdb_batch_find_mode(self.h, C.byref(bd), C.byref(ma), _p(beta),
                                          C.cast(res, C.c_void_p), C.byref(secs)))
        out = [{"flag": r.return_flag, "iterations": r.iterations, "loglik": r.log_likelihood,
                "objective": r.objective, "pred_loglik": r.predictive_loglik, "steps": r.steps,
                "updates": r.updates, "update_entries": r.update_entries,
                "gradient_entries": r.gradient_entries} for r in res]
        return beta, out, secs.value

    def fold_instances(self, variances, holdout, row_fold, args: Optional[ModeFindingArguments] = None):
        """Cross-validation instances as standalone fits on this handle, for
        any model: instance i weights the rows 1 off fold holdout[i] and 0 on
        it (CrossValidationSelector::getWeights), runs its columns at the J
        prior variances variances[i], starts cold, and reports the held-out
        fold's predictive log-likelihood when it succeeded
        (AbstractCrossValidationDriver.cpp:180-232).  Serves what one batched
        launch does not: several variance parameters, and the conditional
        and Cox models.  Needs an FP64 handle (the mixed-precision engine
        runs batched launches only; ccdb_find_mode refuses it).  The handle
        is left unweighted.  Returns (beta[n, J], list of per-instance
        dicts, device seconds)."""
        args = args or ModeFindingArguments()
        var = np.ascontiguousarray(variances, dtype=np.float64)
        if var.ndim != 2 or var.shape[1] != self.d.J:
            raise ValueError("variances must be n x J")
        hold = np.asarray(holdout, dtype=np.int64)
        fold = np.asarray(row_fold)
        start = np.zeros(self.d.J)
        if self.d.offset_col0:
            start[0] = 1.0
        beta = np.zeros((var.shape[0], self.d.J))
        out, secs = [], 0.0
        try:
            for i in range(var.shape[0]):
                w = (fold != hold[i]).astype(np.float64)
                self.set_weights(w)
                keep = []
                ma = _mode_args(dataclasses.replace(self.d, prior_var=var[i]), args, keep)
                b = start.copy()
                res = _FitResult()
                _check(lib().ccdb_find_mode(self.h, C.byref(ma), _p(b), C.byref(res)))
                pred = (self.get_predictive_log_likelihood(1.0 - w) if res.return_flag == 0
                        else float("nan"))
                beta[i] = b
                secs += res.device_seconds
                out.append({"flag": res.return_flag, "iterations": res.iterations,
                            "loglik": res.log_likelihood, "objective": res.objective, "pred_loglik": pred})
        finally:
            self.set_weights(None)
        return beta, out, secs

    # --- CyclicCoordinateDescent::update
    def find_mode(self, args: Optional[ModeFindingArguments] = None,
                  beta: Optional[np.ndarray] = None) -> FitResult:
        args = args or ModeFindingArguments()
        keep = []
        ma = _mode_args(self.d, args, keep)
        b = None if beta is None else np.ascontiguousarray(beta, np.float64).copy()
        res = _FitResult()
        _check(lib().ccdb_find_mode(self.h, C.byref(ma), _p(b), C.byref(res)))
        out = b if b is not None else self.get_beta()
        return FitResult(out, res.return_flag, res.iterations, res.log_likelihood, res.objective,
                         res.coordinate_updates, res.device_seconds, res.kernel_seconds,
                         res.kernel_launches, res.attempts, res.sweeps_total, res.nonzero_steps)


def fit_model(ctx: Context, d: CyclopsData, args: Optional[ModeFindingArguments] = None,
              weights: Optional[np.ndarray] = None, precision: int = PRECISION_FP64) -> FitResult:
    """One call from host buffers: upload, find the mode, return beta
    (the fitCyclopsModel-style entry point, ccdb_fit_model)."""
    args = args or ModeFindingArguments()
    keep = []
    desc = _desc(d, precision, keep)
    ma = _mode_args(d, args, keep)
    arrs = [_c(d.col_start, np.int64), _c(d.rows, np.int32), _c(d.val_start, np.int64),
            _c(d.vals, np.float64), _c(d.fmt, np.uint8)]
    w = _c(weights, np.float64)
    beta = np.zeros(d.J)
    res = _FitResult()
    _check(lib().ccdb_fit_model(ctx.h, d.K, d.J, *[_p(a) for a in arrs], C.byref(desc), _p(w),
                                C.byref(ma), _p(beta), C.byref(res)))
    return FitResult(beta, res.return_flag, res.iterations, res.log_likelihood, res.objective,
                     res.coordinate_updates, res.device_seconds, res.kernel_seconds,
                     res.kernel_launches, res.attempts, res.sweeps_total, res.nonzero_steps)


def validate_matrix(d: CyclopsData) -> None:
    """The checks a matrix upload applies (host only); raises CcdbError."""
    arrs = [_c(d.col_start, np.int64), _c(d.rows, np.int32), _c(d.val_start, np.int64),
            _c(d.vals, np.float64), _c(d.fmt, np.uint8)]
    _check(lib().ccdb_matrix_validate(d.K, d.J, *[_p(a) for a in arrs]))


def sweep_levels(d: CyclopsData, fixed: Optional[np.ndarray] = None):
    """Dependency level of every column in a fused sweep (host-only)."""
    fx = np.zeros(d.J, np.uint8) if fixed is None else np.ascontiguousarray(fixed, np.uint8)
    if fixed is None and d.offset_col0:
        fx[0] = 1
    out = np.zeros(d.J, np.int32)
    n = C.c_int32()
    cs, rows, fmt = _c(d.col_start, np.int64), _c(d.rows, np.int32), _c(d.fmt, np.uint8)
    _check(lib().ccdb_sweep_levels(d.K, d.J, _p(cs), _p(rows), _p(fmt), _p(fx), _p(out), C.byref(n)))
    return out, n.value
