"""The C-ABI library loads and exports every entry point include/specfem_b200.h
declares (no GPU needed)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "specfem_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"SFB_API\s+[^;(]*?\b(sfb_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "sfb_run_forward" in syms and "sfb_domain_update_wavefields" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol(native_lib):
    from specfempp_b200 import _capi
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares a signature for every entry point
    assert sorted(_capi.SIGNATURES) == declared_symbols()


def test_errors_are_reported_not_thrown(native_lib):
    import pytest
    from specfempp_b200 import Simulation, SfbError
    with pytest.raises(SfbError) as e:
        Simulation.from_yaml("/nonexistent/specfem_config.yaml")
    assert e.value.code == -3  # SFB_E_IO
    assert "open" in str(e.value)


def test_fp64_verification_build_exports_the_same_abi(native_lib):
    """The FP64 verification build exports every entry point except the
    FP32-only allocation-free one, and reports its arithmetic width."""
    from specfempp_b200 import _capi
    lib = ctypes.CDLL(_capi.LIB64_PATH)
    missing = [s for s in declared_symbols() if s not in _capi.FP32_ONLY and not hasattr(lib, s)]
    assert not missing, missing
    assert _capi.load(64).sfb_real_bytes() == 8
    assert _capi.load(32).sfb_real_bytes() == 4
