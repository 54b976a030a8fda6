import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle_engine():
    """The CPU checker: the reference engine compiled from source when it is
    present, otherwise the plain-C restatement (built from oracle/ on demand)."""
    from oracle import checker
    return checker.best_engine()


@pytest.fixture(scope="session")
def gpu_ctx():
    from ccd_b200 import native
    ctx = native.Context(0)
    yield ctx
    ctx.close()
