"""ORACLE / TEST INFRASTRUCTURE ONLY -- ctypes access to the two CPU checkers.

* ``ReferenceEngine``   -- the reference Cyclops engine compiled from source
  (``oracle/_ref/libccd_ref.so``, built by ``make -C oracle ref`` where the
  reference sources are present).
* ``RestatementEngine`` -- the plain-C FP64 restatement (``oracle/_build/
  libccd_oracle.so``, ``make -C oracle port``; builds anywhere gcc exists).

Both expose the same calls (``fit``, ``grad_hess``, ``update_beta``,
``loglik``, ``xbeta`` ...) on a ``CyclopsData`` problem.  Only tests/,
``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` import this
module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libccd_ref.so")
REF_B200_LIB = os.path.join(HERE, "_ref", "libccd_ref_b200.so")
PORT_LIB = os.path.join(HERE, "_build", "libccd_oracle.so")

_P = C.c_void_p
_D = C.POINTER(C.c_double)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def build(target: str = "all") -> None:
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


class _Engine:
    prefix = ""
    libpath = ""
    create_name = None
    _lib_cache: dict = {}

    @classmethod
    def lib(cls):
        if cls.libpath not in _Engine._lib_cache:
            if not os.path.exists(cls.libpath):
                if cls is RestatementEngine:
                    build("port")
                else:
                    raise FileNotFoundError(cls.libpath)
            lib = C.CDLL(cls.libpath)
            p = cls.prefix
            cname = cls.create_name or (p + "create")
            getattr(lib, cname).restype = _P
            getattr(lib, cname).argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int] + [_P] * 8 + [
                C.c_int, _P, _P, C.c_char_p, C.c_int]
            getattr(lib, p + "destroy").argtypes = [_P]
            getattr(lib, p + "fit").argtypes = [_P, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int,
                                                C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_char_p, C.c_int]
            getattr(lib, p + "grad_hess").argtypes = [_P, C.c_int, _P, _P]
            getattr(lib, p + "update_beta").argtypes = [_P, C.c_int, C.c_double]
            for name in ("set_weights", "set_beta", "loglik", "log_prior", "get_beta", "get_xbeta"):
                getattr(lib, p + name).argtypes = [_P, _P]
            getattr(lib, p + "predictive_loglik").argtypes = [_P, _P, _P]
            getattr(lib, p + "num_patients").argtypes = [_P]
            if p == "ref_":
                lib.ref_fisher_information.argtypes = [_P, _P, C.c_int, _P, C.c_char_p, C.c_int]
                lib.ref_asymptotic_variance.argtypes = [_P, C.c_int, C.c_int, _P, C.c_char_p, C.c_int]
            else:
                lib.orc_fisher_information.argtypes = [_P, _P, C.c_int, _P]
            getattr(lib, p + "predictive_estimates").argtypes = [_P, _P, _P]
            _Engine._lib_cache[cls.libpath] = lib
        lib = _Engine._lib_cache[cls.libpath]
        # engines sharing a library may use different constructors
        cname = cls.create_name or (cls.prefix + "create")
        fn = getattr(lib, cname)
        if fn.restype is not _P:
            fn.restype = _P
            fn.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int] + [_P] * 8 + [C.c_int, _P, _P, C.c_char_p, C.c_int]
        return lib

    def __init__(self, d, fp32: bool = False):
        self.d = d
        self._keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        lib = self.lib()
        err = C.create_string_buffer(512)
        self.h = getattr(lib, self.create_name or (self.prefix + "create"))(
            d.model_type, int(fp32), d.K, d.J, _ptr(arr(d.y, np.float64)),
            _ptr(arr(d.time, np.float64)), _ptr(arr(d.stratum, np.int64)),
            _ptr(arr(d.col_start, np.int64)), _ptr(arr(d.rows, np.int32)),
            _ptr(arr(d.val_start, np.int64)), _ptr(arr(d.vals, np.float64)),
            _ptr(arr(d.fmt, np.uint8)), int(d.offset_col0), _ptr(arr(d.prior_type, np.int32)),
            _ptr(arr(d.prior_var, np.float64)), err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())

    def _f(self, name):
        return getattr(self.lib(), self.prefix + name)

    def close(self):
        if getattr(self, "h", None):
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_weights(self, w: Optional[np.ndarray]):
        if w is not None:
            w = np.ascontiguousarray(w, np.float64)
            self._w = w
        self._f("set_weights")(self.h, _ptr(w))

    def set_beta(self, beta: np.ndarray):
        beta = np.ascontiguousarray(beta, np.float64)
        self._f("set_beta")(self.h, _ptr(beta))

    def fit(self, conv_type: int = 0, tol: float = 1e-6, max_iter: int = 1000,
            initial_bound: float = 2.0, max_bound_count: int = 5, algorithm: int = 0,
            kkt_swindle: bool = False, fixed: Optional[np.ndarray] = None):
        """CyclicCoordinateDescent::update; algorithm 0 = CCD, 1 = MM."""
        beta = np.zeros(self.d.J)
        ll = C.c_double()
        it = C.c_int()
        fl = C.c_int()
        err = C.create_string_buffer(512)
        fx = None if fixed is None else np.ascontiguousarray(fixed, np.uint8)
        rc = self._f("fit")(self.h, conv_type, tol, max_iter, initial_bound, max_bound_count,
                            algorithm, int(kkt_swindle), _ptr(fx), _ptr(beta), C.byref(ll), C.byref(it),
                            C.byref(fl), err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return {"beta": beta, "loglik": ll.value, "iterations": it.value, "flag": fl.value}

    def grad_hess(self, j: int):
        g, h = C.c_double(), C.c_double()
        self._f("grad_hess")(self.h, j, C.byref(g), C.byref(h))
        return g.value, h.value

    def update_beta(self, j: int, delta: float):
        self._f("update_beta")(self.h, j, delta)

    def loglik(self) -> float:
        v = C.c_double()
        self._f("loglik")(self.h, C.byref(v))
        return v.value

    def log_prior(self) -> float:
        v = C.c_double()
        self._f("log_prior")(self.h, C.byref(v))
        return v.value

    def beta(self) -> np.ndarray:
        b = np.zeros(self.d.J)
        self._f("get_beta")(self.h, _ptr(b))
        return b

    def xbeta(self) -> np.ndarray:
        x = np.zeros(self.d.K)
        self._f("get_xbeta")(self.h, _ptr(x))
        return x

    def predictive_loglik(self, w: np.ndarray) -> float:
        w = np.ascontiguousarray(w, np.float64)
        v = C.c_double()
        self._f("predictive_loglik")(self.h, _ptr(w), C.byref(v))
        return v.value


    def fisher_information(self, indices) -> np.ndarray:
        """Fisher information over the columns `indices` (n x n).  Raises
        FisherRefused where the engine refuses (weighted fits)."""
        idx = np.ascontiguousarray(indices, np.int32)
        out = np.zeros((len(idx), len(idx)))
        if self.prefix == "ref_":
            err = C.create_string_buffer(512)
            rc = self._f("fisher_information")(self.h, _ptr(idx), len(idx), _ptr(out), err, 512)
            msg = err.value.decode()
        else:
            rc = self._f("fisher_information")(self.h, _ptr(idx), len(idx), _ptr(out))
            msg = "Weights are not yet implemented in Fisher Information calculations"
        if rc == -2:
            raise FisherRefused(msg)
        if rc != 0:
            raise RuntimeError(msg)
        return out

    def predictive_estimates(self, w: Optional[np.ndarray] = None, y: Optional[np.ndarray] = None):
        y = np.zeros(self.d.K) if y is None else np.array(y, dtype=np.float64)
        if w is not None:
            w = np.ascontiguousarray(w, np.float64)
        self._f("predictive_estimates")(self.h, _ptr(w), _ptr(y))
        return y


class FisherRefused(RuntimeError):
    """The engine refuses a Fisher information request (a weighted fit)."""


class ReferenceEngine(_Engine):
    prefix = "ref_"
    libpath = REF_LIB


    @classmethod
    def quadr_log_fit(cls, history: dict):
        """The auto search's quadratic fit (utils/HParSearch.cpp:22-64) of a
        {x: (mean, stdev)} history: (c0, c1, c2)."""
        fn = cls.lib().ref_quadr_log_fit
        fn.argtypes = [C.c_int, _P, _P, _P, _P]
        xs = np.array(sorted(history), dtype=np.float64)
        m = np.array([history[x][0] for x in xs], dtype=np.float64)
        sd = np.array([history[x][1] for x in xs], dtype=np.float64)
        out = np.zeros(3)
        fn(len(xs), _ptr(xs), _ptr(m), _ptr(sd), _ptr(out))
        return float(out[0]), float(out[1]), float(out[2])

    def asymptotic_variance(self, i: int, j: int) -> float:
        v = C.c_double()
        err = C.create_string_buffer(512)
        rc = self._f("asymptotic_variance")(self.h, i, j, C.byref(v), err, 512)
        if rc != 0:
            raise (FisherRefused if rc == -2 else RuntimeError)(err.value.decode())
        return v.value


    def cross_validate(self, auto_search: bool = True, fold: int = 10, grid_steps: int = 10,
                       lower: float = 0.01, upper: float = 20.0, starting_variance: float = -1.0,
                       seed: int = 123, conv_type: int = 0, tol: float = 1e-6, max_iter: int = 1000,
                       threads: int = 1, fold_to_compute: int = 0):
        """CcdInterface::runCrossValidation with one thread and cold starts:
        the reference selector's fold map, the grid (grid search), the drivers'
        log, the selected variance and the refit there."""
        lib = self.lib()
        fn = lib.ref_cross_validate
        fn.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_long,
                       C.c_int, C.c_double, C.c_int, _P, _P, _P, C.c_int, _P, _P, _P, _P, C.c_char_p,
                       C.c_int, _P, C.c_int, _P, C.c_int, C.c_int, C.c_char_p, C.c_int]
        row_fold = np.zeros(self.d.K, np.int32)
        pts, vals = np.zeros(max(grid_steps, 1)), np.zeros(max(grid_steps, 1))
        n = C.c_int()
        var, ll = C.c_double(), C.c_double()
        beta = np.zeros(self.d.J)
        log = C.create_string_buffer(1 << 24)
        err = C.create_string_buffer(512)
        hyper = np.zeros(64)
        nh = C.c_int()
        rc = fn(self.h, int(auto_search), fold, grid_steps, lower, upper, starting_variance, seed, conv_type,
                tol, max_iter, _ptr(row_fold), _ptr(pts), _ptr(vals), len(pts), C.byref(n), C.byref(var),
                _ptr(beta), C.byref(ll), log, 1 << 24, _ptr(hyper), len(hyper), C.byref(nh), int(threads),
                int(fold_to_compute), err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return {"row_fold": row_fold, "points": pts[:n.value], "values": vals[:n.value], "variance": var.value,
                "variances": hyper[:min(nh.value, len(hyper))].copy(), "beta": beta, "loglik": ll.value,
                "log": log.value.decode()}


    def profile(self, cols, threshold: float = 1.920729, include_penalty: bool = False,
                override_no_regularization: bool = False, conv_type: int = 0, tol: float = 1e-6,
                max_iter: int = 1000):
        """CcdInterface::profileModel around the current mode: (lower, upper,
        objective evaluations) per column."""
        fn = self.lib().ref_profile
        fn.argtypes = [_P, _P, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                       _P, _P, _P, C.c_char_p, C.c_int]
        cols = np.ascontiguousarray(cols, np.int32)
        lo, up = np.zeros(len(cols)), np.zeros(len(cols))
        ev = np.zeros(len(cols), np.int32)
        err = C.create_string_buffer(512)
        rc = fn(self.h, _ptr(cols), len(cols), threshold, int(include_penalty), int(override_no_regularization),
                conv_type, tol, max_iter, _ptr(lo), _ptr(up), _ptr(ev), err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return lo, up, ev


class ReferenceOnB200Engine(ReferenceEngine):
    """The reference's own CyclicCoordinateDescent driving the B200 engine
    through ccd_b200/integration/B200ModelSpecifics.h (the drop-in)."""
    prefix = "ref_"
    libpath = REF_B200_LIB
    create_name = "ref_create_b200"


class ReferenceOnB200FusedEngine(ReferenceEngine):
    """The reference's solver as B200CyclicCoordinateDescent
    (ccd_b200/integration/B200CyclicCoordinateDescent.h): each findMode of
    update() is one ccdb_find_mode call on the device."""
    prefix = "ref_"
    libpath = REF_B200_LIB
    create_name = "ref_create_b200_fused"

    def device_calls(self) -> int:
        fn = self.lib().ref_device_calls
        fn.argtypes = [_P]
        fn.restype = C.c_int64
        return int(fn(self.h))


class RestatementEngine(_Engine):
    prefix = "orc_"
    libpath = PORT_LIB

    def fit_attempts(self):
        """Cycles of each findMode attempt of the last fit (the ILLCONDITIONED
        retry of CyclicCoordinateDescent::update runs several)."""
        fn = self.lib().orc_fit_attempts
        fn.argtypes = [_P, _P, C.c_int]
        buf = np.zeros(16, np.int32)
        n = fn(self.h, _ptr(buf), 16)
        return [int(x) for x in buf[:min(n, 16)]]

    @classmethod
    def set_exp_perturbation(cls, one_in: int, salt: int = 0):
        """Move exp by one ulp on 2 in `one_in` arguments (0: off), for every
        restatement engine of the process (see orc_set_exp_perturbation)."""
        fn = cls.lib().orc_set_exp_perturbation
        fn.argtypes = [C.c_uint, C.c_uint]
        fn(int(one_in), int(salt))


def best_engine():
    """The compiled reference when present, else the restatement."""
    return ReferenceEngine if reference_available() else RestatementEngine
