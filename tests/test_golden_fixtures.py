"""The committed golden Newmark fixtures (tests/golden/newmark, made by
tests/golden/make_newmark_fixtures.py from the reference's
tests/unit-tests/displacement_tests/Newmark/serial/*): they reproduce the
reference's files where the reference is present, and the CPU oracle meets
the reference's metric (newmark_tests.cpp:304-346, 1e-3) on them with no
reference checkout, as the GPU tests use them."""
import gzip
import os

import numpy as np
import pytest

from conftest import REFERENCE
from golden_util import CASES, FIXTURES, fixture_case, station_errors


@pytest.mark.parametrize("case", CASES)
def test_fixture_matches_reference_files(case):
    src = os.path.join(REFERENCE, "tests", "unit-tests", "displacement_tests", "Newmark", "serial", case)
    if not os.path.isdir(src):
        pytest.skip("reference tree not mounted")
    with gzip.open(os.path.join(FIXTURES, case, "database.bin.gz"), "rb") as f:
        assert f.read() == open(os.path.join(src, "database.bin"), "rb").read()
    traces = np.load(os.path.join(FIXTURES, case, "traces.npz"))
    assert sorted(traces.files) == sorted(os.listdir(os.path.join(src, "traces")))
    for name in traces.files[:5]:
        ref = np.loadtxt(os.path.join(src, "traces", name))
        np.testing.assert_allclose(traces[name], ref, rtol=1e-6, atol=1e-30)


@pytest.mark.parametrize("case", CASES)
def test_oracle_meets_golden_metric_on_fixture(case, tmp_path, native_lib, oracle_lib):
    from oracle import bridge
    from specfempp_b200 import Simulation
    cfg, traces, stations = fixture_case(case, str(tmp_path))
    sim = Simulation.from_yaml(cfg)
    info = sim.info()
    out = bridge.forward(sim, 32, threads=4)
    v = sim.problem_view()
    types = [v.seismogram_types[k] for k in range(info.nseismogram_types)]
    errs = station_errors(case, traces, stations, types, out["seismograms"], sim.seismogram_times())
    assert np.all(errs <= 1e-3), (case, errs.max())
