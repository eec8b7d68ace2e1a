"""Parameter-file path on the host (no GPU): the structured database.bin
writer reproduces the structured mesher's assembly, and combined-mode
sources files with adjoint sources and External time functions parse with
the reference's checks (src/io/sources.cpp:92-160,
src/source_time_function/external.cpp)."""
import ctypes as C
import os

import numpy as np
import pytest

from specfempp_b200 import SfbError, Simulation
from workflow_util import STATIONS, structured, write_combined, write_forward

NSTEP, DT = 200, 5e-4


def arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy()


def test_database_writer_matches_structured_mesher(tmp_path, native_lib):
    cfg = write_forward(str(tmp_path), NSTEP, DT)
    a = Simulation.from_yaml(cfg)
    b = Simulation.structured(structured(NSTEP, DT))
    va, vb = a.problem_view(), b.problem_view()
    assert va.nspec == vb.nspec and list(va.nglob) == list(vb.nglob)
    nloc = va.nspec * va.ngll * va.ngll
    for name in ("xix", "xiz", "gammax", "gammaz", "jacobian", "kappa", "mu", "rho"):
        np.testing.assert_array_equal(arr(getattr(va, name), nloc, np.float32), arr(getattr(vb, name), nloc, np.float32))
    np.testing.assert_array_equal(arr(va.iglob, nloc, np.int32), arr(vb.iglob, nloc, np.int32))
    np.testing.assert_array_equal(arr(va.bnd, nloc, np.uint8), arr(vb.bnd, nloc, np.uint8))
    np.testing.assert_array_equal(arr(va.rec_ispec, va.nreceivers, np.int32), arr(vb.rec_ispec, vb.nreceivers, np.int32))
    assert abs(va.t0 - vb.t0) < 1e-12


def write_adj(folder, names, nstep, dt, t0, dt_file=None):
    os.makedirs(folder, exist_ok=True)
    rng = np.random.default_rng(0)
    for name in names:
        for comp in ("BXX", "BXZ"):
            v = rng.standard_normal(nstep)
            t = t0 + (dt_file or dt) * np.arange(nstep)
            np.savetxt(os.path.join(folder, "%s.%s.adj" % (name, comp)), np.c_[t, v])


def test_combined_sources_file_parses(tmp_path, native_lib):
    root = str(tmp_path)
    write_forward(root, NSTEP, DT)
    t0 = Simulation.from_yaml(os.path.join(root, "forward_config.yaml")).info().t0
    names = ["AA.S%04d.S2" % (k + 1) for k in range(len(STATIONS))]
    write_adj(os.path.join(root, "adj"), names, NSTEP, DT, t0)
    sim = Simulation.from_yaml(write_combined(root, NSTEP, DT, os.path.join(root, "adj"), names))
    info = sim.info()
    assert info.simulation == 1 and info.nsources == 1 and info.nadjoint_sources == len(STATIONS)
    # adjoint sources come from the file: the per-station setter refuses
    with pytest.raises(SfbError):
        sim.set_adjoint_sources(np.zeros((NSTEP, len(STATIONS), 2), np.float32))


def test_external_time_step_mismatch_is_rejected(tmp_path, native_lib):
    root = str(tmp_path)
    write_forward(root, NSTEP, DT)
    t0 = Simulation.from_yaml(os.path.join(root, "forward_config.yaml")).info().t0
    names = ["AA.S%04d.S2" % (k + 1) for k in range(len(STATIONS))]
    write_adj(os.path.join(root, "adj"), names, NSTEP, DT, t0, dt_file=2 * DT)
    with pytest.raises(SfbError, match="time step"):
        Simulation.from_yaml(write_combined(root, NSTEP, DT, os.path.join(root, "adj"), names))


def test_adjoint_source_in_forward_mode_is_rejected(tmp_path, native_lib):
    root = str(tmp_path)
    write_forward(root, NSTEP, DT)
    t0 = Simulation.from_yaml(os.path.join(root, "forward_config.yaml")).info().t0
    names = ["AA.S0001.S2"]
    write_adj(os.path.join(root, "adj"), names, NSTEP, DT, t0)
    cfg = write_combined(root, NSTEP, DT, os.path.join(root, "adj"), names)
    text = open(cfg).read()
    text = text.replace("      combined:", "      forward:").replace("        reader:\n          wavefield:", "        writer:\n          wavefield:")
    text = text.replace("""        writer:
          kernels:
            format: ascii""", """          seismogram:
            format: ascii""")
    with open(cfg, "w") as f:
        f.write(text)
    with pytest.raises(SfbError, match="Adjoint sources found"):
        Simulation.from_yaml(cfg)


def test_user_defined_source_in_a_sources_file(tmp_path, native_lib):
    """A `user-defined` entry (src/io/sources.cpp:88-91): the source array is
    the Lagrange weight of the location in every component."""
    cfg = write_forward(str(tmp_path), NSTEP, DT)
    src = os.path.join(str(tmp_path), "forward_sources.yaml")
    with open(src, "w") as f:
        f.write("number-of-sources: 1\nsources:\n  - user-defined:\n      x : 413.0\n      z : 287.0\n"
                "      Ricker:\n        factor: 1e10\n        tshift: 0.0\n        f0: 10.0\n")
    sim = Simulation.from_yaml(cfg)
    view = sim.problem_view()
    n = view.ngll
    assert view.nsources == 1
    a = np.ctypeslib.as_array(view.src_array, shape=(1, 2, n, n))
    np.testing.assert_allclose(a.sum(axis=(2, 3)), [[1.0, 1.0]], rtol=1e-6)
    np.testing.assert_array_equal(a[0, 0], a[0, 1])
    stf = np.ctypeslib.as_array(view.src_stf, shape=(1, NSTEP, 2))
    np.testing.assert_array_equal(stf[0, :, 0], stf[0, :, 1])
    assert np.abs(stf).max() > 0
