import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference checkout whose golden files the CPU tests read (absent on
# machines without it: those tests skip).
REFERENCE = os.environ.get("SPECFEMPP_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def native_lib():
    """The product library, built in-tree when missing."""
    from specfempp_b200 import _capi, build
    if not os.path.exists(_capi.LIB_PATH):
        build.build()
    return _capi.load()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import bridge
    return bridge.load()


@pytest.fixture(scope="session")
def reference_tests_dir():
    d = os.path.join(REFERENCE, "tests", "unit-tests")
    if not os.path.isdir(d):
        pytest.skip("reference tree not mounted")
    return d


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
