"""The C ABI library loads and exports every function include/ccdb.h declares
(no GPU needed); calls that need a device fail with a status, not a crash."""
import ctypes as C
import os
import re

import pytest

from ccd_b200 import native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ccdb.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(ccdb_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_operator_api():
    names = declared_functions()
    for must in ("ccdb_compute_gradient_hessian", "ccdb_update_xbeta", "ccdb_find_mode",
                 "ccdb_fit_model", "ccdb_matrix_create", "ccdb_set_weights",
                 # the rest of the AbstractModelSpecifics operator API and setFixedBeta
                 "ccdb_fisher_information", "ccdb_compute_mm_gradient_hessian",
                 "ccdb_get_predictive_log_likelihood", "ccdb_get_predictive_estimates", "ccdb_set_fixed",
                 "ccdb_compute_xbeta"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_context_without_gpu_returns_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = native.lib().ccdb_context_create(0, 0, C.byref(h))
    assert rc < 0
    assert native.lib().ccdb_last_error()


def test_invalid_matrix_is_rejected_before_any_device_work():
    # NULL context: argument validation fails first
    h = C.c_void_p()
    rc = native.lib().ccdb_matrix_create(None, 10, 1, None, None, None, None, None, C.byref(h))
    assert rc == native.ERR_INVALID
