"""The C-ABI library loads and exports every entry point include/specfem_b200.h
declares (no GPU needed)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "specfem_b200.h")
HEADER3 = os.path.join(ROOT, "include", "specfem_b200_3d.h")


def declared_symbols(header=HEADER, prefix="sfb_"):
    text = open(header).read()
    return sorted(set(re.findall(r"SFB_API\s+[^;(]*?\b(%s\w+)\s*\(" % prefix, text)))


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


def test_library_exports_every_3d_entry_point(native_lib):
    """include/specfem_b200_3d.h: every declared entry point is exported by
    the product library and bound in specfempp_b200.hex3d."""
    from specfempp_b200 import _capi, hex3d
    syms = declared_symbols(HEADER3, "sfb3_")
    assert "sfb3_run_combined" in syms and len(syms) >= 12
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(hex3d.SIGNATURES3) == syms


def test_3d_descriptor_matches_the_header():
    """The ctypes mirror of sfb3_desc / sfb3_info / sfb3_source lists the
    header's fields in order."""
    from specfempp_b200 import hex3d
    text = open(HEADER3).read()
    for cls, name in ((hex3d.sfb3_desc, "sfb3_desc"), (hex3d.sfb3_info, "sfb3_info"),
                      (hex3d.sfb3_source, "sfb3_source")):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = re.findall(r"\**\s*(\w+)\s*(?=[,;])", body)
        assert [f[0] for f in cls._fields_] == fields, (name, fields)


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
