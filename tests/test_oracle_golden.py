"""The CPU oracle reproduces the reference's golden Newmark traces
(tests/unit-tests/displacement_tests/Newmark/serial/*) within the reference's
own tolerance (1e-3, newmark_tests.cpp:325-334), starting from the reference
test's YAML file and database.bin parsed by the product's host setup."""
import os

import numpy as np
import pytest

from golden_util import CASES, station_errors

from conftest import REFERENCE

DEFAULT_YAML = os.path.join(REFERENCE, "parameter_files", "defaults", "default.yaml")


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_golden_traces(case, reference_tests_dir, native_lib, oracle_lib):
    from oracle import bridge
    from specfempp_b200 import Simulation
    d = os.path.join(reference_tests_dir, "displacement_tests", "Newmark", "serial", case)
    sim = Simulation.from_yaml(os.path.join(d, "specfem_config.yaml"), DEFAULT_YAML)
    info = sim.info()
    out = bridge.forward(sim, 32, threads=4)
    stations = [tuple(l.split()[:2][::-1]) for l in open(os.path.join(d, "STATIONS")) if l.strip()]
    v = sim.problem_view()
    types = [v.seismogram_types[k] for k in range(info.nseismogram_types)]
    errs = station_errors(case, lambda n: np.loadtxt(os.path.join(d, "traces", n)), stations, types,
                          out["seismograms"], sim.seismogram_times())
    assert np.all(errs <= 1e-3), (case, errs.max())
