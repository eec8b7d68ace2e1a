"""The C++ adapter (include/specfem_b200.hpp) and the time-loop driver
written against it (tests/cpp/time_marching_b200.cpp) compile against the
library, and the driver builds a context from a reference-format parameter
file without a device; the reference's Python entry points (specfempp_core)
behave as the reference's do before and after initialisation."""
import os
import subprocess

import pytest

from conftest import ROOT

DRIVER_SRC = os.path.join(ROOT, "tests", "cpp", "time_marching_b200.cpp")


def build_driver(out_dir):
    from specfempp_b200 import _capi
    exe = os.path.join(out_dir, "time_marching_b200")
    lib = os.path.dirname(_capi.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-o", exe, DRIVER_SRC, "-L" + lib, "-lspecfem_b200",
           "-Wl,-rpath," + lib]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_driver_compiles_and_reads_parameter_file(native_lib, tmp_path):
    import workflow_util as WU
    exe = build_driver(str(tmp_path))
    cfg = WU.write_forward(str(tmp_path), 100, 5e-4)
    r = subprocess.run([exe, "info", cfg], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["nspec", str(WU.NX * WU.NZ), "nstep", "100", "dofs", "10530"]
    r = subprocess.run([exe, "info", "/nonexistent.yaml"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "open" in r.stderr


def test_specfempp_core_entry_points(native_lib):
    import specfempp_core as core
    from specfempp_b200 import SfbError
    core._finalize()
    assert core._execute("parameters: {}", "") is False  # before _initialize, as the reference
    assert core._initialize(["prog"]) is True
    assert core._initialize(["prog"]) is False
    with pytest.raises(SfbError):
        core._execute("parameters:\n  header:\n    title: x\n", "")
    assert os.path.exists(core._default_file_path)
    assert core._finalize() is True
    assert core._finalize() is False
    assert core.WaveformMisfit is not None
