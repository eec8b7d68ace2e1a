"""The reference's time loops written in C++ against include/specfem_b200.hpp
(tests/cpp/time_marching_b200.cpp, with the reference's DOF and element
accounting after every step) on the GPU, and the reference's Python entry
point specfempp_core._execute with YAML text:

  * forward: the C++ loop's seismograms against the library's fused run of
    the same parameter file (relative L2 <= 1e-5, two FP32 runs);
  * combined: the C++ loop, reading the forward wavefield a forward run
    wrote and External adjoint sources (waveform residuals) from files,
    writes kernels that agree with the fused combined run's (sfb_execute)
    within the gradient bar 1e-3;
  * specfempp_core._execute(text) writes the same seismogram files as
    sfb_execute(file), bit for bit in the deterministic mode.
"""
import os
import subprocess

import numpy as np
import pytest

from test_cpp_adapter import build_driver
from workflow_util import NX, NZ, STATIONS, read_kernel, write_combined, write_forward

pytestmark = pytest.mark.gpu

NSTEP, DT = 300, 5e-4


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def traces(folder):
    names = ["AA.S%04d.S2.BX%s.semd" % (k + 1, c) for k in range(len(STATIONS)) for c in "XZ"]
    return np.stack([np.loadtxt(os.path.join(folder, n))[:, 1] for n in names])


def test_cpp_forward_and_combined_loops(tmp_path):
    from specfempp_b200 import adjoint_sources as AS
    from specfempp_b200.__main__ import run
    root = str(tmp_path)
    exe = build_driver(root)
    cfg = write_forward(root, NSTEP, DT)
    run(cfg)  # fused forward through sfb_execute: seismograms + forward wavefield
    cpp_seis = os.path.join(root, "cpp_seismograms")
    os.makedirs(cpp_seis)
    r = subprocess.run([exe, "forward", cfg, cpp_seis], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    e = rel_l2(traces(cpp_seis), traces(os.path.join(root, "seismograms")))
    print("C++ reference-order forward loop vs fused run: %.2e" % e)
    assert e <= 1e-5

    seis = os.path.join(root, "seismograms")
    names = ["AA.S%04d.S2" % (k + 1) for k in range(len(STATIONS))]
    adj = os.path.join(root, "adjoint_sources")
    os.makedirs(adj)
    # waveform-residual adjoint sources (the synthetics against zero data):
    # well conditioned, so the two loops' kernels differ only by FP32
    # rounding (cross-correlation traveltime sources divide by the
    # traces' norms and make the kernels cancel to a few digits)
    for name in names:
        for comp in ("BXX", "BXZ"):
            t, v = AS.read_trace(os.path.join(seis, "%s.%s.semd" % (name, comp)))
            AS.write_trace(os.path.join(adj, "%s.%s.adj" % (name, comp)), t[0], (t[-1] - t[0]) / (len(t) - 1), v)
    ccfg = write_combined(root, NSTEP, DT, adj, names)
    run(ccfg)  # fused combined run writes kernels/
    cpp_k = os.path.join(root, "cpp_kernels")
    cpp_b = os.path.join(root, "cpp_backward")
    os.makedirs(cpp_k)
    os.makedirs(cpp_b)
    r = subprocess.run([exe, "combined", ccfg, root, cpp_k, cpp_b], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    for name in ("rho", "mu", "kappa"):
        a = read_kernel(cpp_k, "elastic_psv_isotropic", name, NX * NZ, 5)
        b = read_kernel(os.path.join(root, "kernels"), "elastic_psv_isotropic", name, NX * NZ, 5)
        e = rel_l2(a, b)
        print("C++ reference-order combined loop vs fused combined run, kernel %s: %.2e" % (name, e))
        assert np.abs(b).max() > 0 and e <= 1e-3


def test_specfempp_core_execute_text(tmp_path, monkeypatch):
    import specfempp_core as core
    from specfempp_b200.__main__ import run
    monkeypatch.setenv("SFB_DETERMINISTIC", "1")
    a = tmp_path / "a"
    b = tmp_path / "b"
    a.mkdir()
    b.mkdir()
    cfg_a = write_forward(str(a), 200, DT)
    run(cfg_a)
    cfg_b = write_forward(str(b), 200, DT)
    core._initialize(["test"])
    try:
        assert core._execute(open(cfg_b).read(), open(core._default_file_path).read()) is True
    finally:
        core._finalize()
    ta, tb = traces(os.path.join(str(a), "seismograms")), traces(os.path.join(str(b), "seismograms"))
    assert np.abs(ta).max() > 0
    assert np.array_equal(ta, tb)
