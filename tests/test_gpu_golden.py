"""The device path on the reference's own golden Newmark cases
(tests/unit-tests/displacement_tests/Newmark/serial/*, committed as
fixtures under tests/golden/newmark): meshes from the reference's Fortran
mesher with 9-node elements, its edge orders, composite Stacey / Dirichlet
boundaries and the acoustic-elastic interface of AcousticElasticCoupledDomain,
built through Simulation.from_yaml from the reference's parameter files.

Three bars per case, through the C ABI:
  * the reference's own metric against its golden traces
    (newmark_tests.cpp:304-346: per station, sum|u - u_ref| / sum|u_ref|
    over components and types, 1e-3);
  * the product's FP32 seismograms within 1e-5 relative L2 of the FP32
    oracle, or of the FP64 oracle within 1e-5 + 2x the FP32 oracle's own
    distance from it (the FP32 rounding level of the problem);
  * the FP64 verification build within 1e-10 of the FP64 oracle.
"""
import numpy as np
import pytest

from golden_util import CASES, fixture_case, station_errors
from specfempp_b200 import Simulation

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("case", CASES)
def test_golden_case_on_gpu(case, tmp_path):
    from oracle import bridge
    cfg, traces, stations = fixture_case(case, str(tmp_path))
    sim = Simulation.from_yaml(cfg)
    sim.run_forward()
    info = sim.info()
    gpu = sim.seismograms()
    v = sim.problem_view()
    types = [v.seismogram_types[k] for k in range(info.nseismogram_types)]
    errs = station_errors(case, traces, stations, types, gpu, sim.seismogram_times())
    o32 = bridge.forward(sim, 32, threads=8)["seismograms"]
    o64 = bridge.forward(sim, 64, threads=8, exact=True)["seismograms"]
    e32, e64, eref = rel_l2(gpu, o32), rel_l2(gpu, o64), rel_l2(o32, o64)
    print("%s: golden metric worst station %.2e; rel-L2 vs FP32 oracle %.2e, vs FP64 %.2e "
          "(FP32 oracle vs FP64 %.2e)" % (case, errs.max(), e32, e64, eref))
    assert np.all(errs <= 1e-3), (case, errs.max())
    assert e32 <= 1e-5 or e64 <= 1e-5 + 2.0 * eref, (case, e32, e64, eref)

    sim64 = Simulation.from_yaml(cfg, precision=64)
    sim64.run_forward()
    g64 = sim64.seismograms()
    e = rel_l2(g64, o64)
    errs64 = station_errors(case, traces, stations, types, g64, sim64.seismogram_times())
    print("%s: FP64 build rel-L2 vs FP64 oracle %.2e; golden metric worst station %.2e" % (case, e, errs64.max()))
    assert e <= 1e-10, (case, e)
    assert np.all(errs64 <= 1e-3)
