"""Parity at the benchmark configurations' full sizes, through the C ABI.

  * plain elastic P-SV, 100 x 80 NGLL=5 elements (128,721 points), all of
    its 4000 steps: the 20 receivers' displacement traces;
  * coupled acoustic-elastic, 400 x 300 (1,924,402 points, the workload
    bench.py times), 1400 steps (the source sits mid-water, 1.5 km above the
    sea floor: the wave reaches the elastic medium after about 1.25 s):
    final wavefields of both media and the 200 pressure traces, for the
    compact-block kernel the autotuner picks there and the full-block one;
  * batched, 800 x 400 (5.1 M points, 64 shots in one context), 1000 steps:
    the first and last shots' traces at the 400 receivers and final fields
    against the oracle run of each shot alone.

Two bars per case.  The FP64 verification build (the same generic kernels
in FP64) within 1e-10 relative L2 of the FP64 oracle: the discrete
operators are the reference's.  The product's FP32 result within 1e-5 of
the FP32 oracle, or of the FP64 oracle within 1e-5 + 2x the FP32 oracle's
own distance from it (two FP32 runs differ by their rounding, which an
ill-conditioned long run amplifies).  Every FP32 distance is printed next
to the 1e-5 bar.  The oracle's CPU time bounds the step counts."""
import os

import numpy as np
import pytest

from specfempp_b200 import Simulation
from specfempp_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5
BAR64 = 1e-10
NSTEP_COUPLED = 1400
NSTEP_BATCHED = 1000
MEDIA = ((0, "psv"), (3, "acoustic"))  # device medium index, oracle field key
THREADS = max(1, min(32, os.cpu_count() or 1))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fp32_ok(label, g, o32, o64):
    e32, e64, eref = rel_l2(g, o32), rel_l2(g, o64), rel_l2(o32, o64)
    print("%s: FP32 vs FP32 oracle %.2e (seismogram bar 1e-5: %s), vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
          % (label, e32, "met" if e32 <= TOL_FP32 else "not met", e64, eref))
    assert np.isfinite(g).all() and np.abs(o64).max() > 0, label
    assert e32 <= TOL_FP32 or e64 <= TOL_FP32 + 2.0 * eref, (label, e32, e64, eref)


def fp64_ok(label, g, o64):
    e = rel_l2(g, o64)
    print("%s: FP64 build vs FP64 oracle %.2e" % (label, e))
    assert e <= BAR64, (label, e)


def test_full_size_plain_elastic_all_steps():
    from oracle import bridge
    p = W.plain_elastic(1.0, nstep=4000)
    sim = Simulation.structured(p)
    info = sim.info()
    assert info.nspec == 8000 and info.nglob[0] == 128721 and info.nstep == 4000
    sim.run_forward()
    o32 = bridge.forward(sim, 32, threads=THREADS)["seismograms"]
    o64 = bridge.forward(sim, 64, threads=THREADS, exact=True)["seismograms"]
    fp32_ok("plain 4000 steps, variant %d, traces" % info.stiffness_variant[0], sim.seismograms(), o32, o64)
    sim64 = Simulation.structured(p, precision=64)
    sim64.run_forward()
    fp64_ok("plain 4000 steps, traces", sim64.seismograms(), o64)


@pytest.fixture(scope="module")
def coupled_oracle():
    from oracle import bridge
    sim = Simulation.structured(W.coupled(1.0, nstep=NSTEP_COUPLED, seismogram_types=("pressure",)))
    o32 = bridge.forward(sim, 32, threads=THREADS, want_fields=True)
    o64 = bridge.forward(sim, 64, threads=THREADS, want_fields=True, exact=True)
    return o32, o64


@pytest.mark.parametrize("variant", [3, 1])
def test_full_size_coupled_fields(coupled_oracle, variant):
    o32, o64 = coupled_oracle
    sim = Simulation.structured(W.coupled(1.0, nstep=NSTEP_COUPLED, seismogram_types=("pressure",)))
    info = sim.info()
    assert info.nspec == 120000
    assert info.nglob[0] + info.nglob[3] == 1924402
    for medium, _ in MEDIA:
        sim.set_stiffness_variant(medium, variant)
    sim.run_forward()
    for medium, key in MEDIA:
        for which, name in ((0, "u"), (1, "v"), (2, "a")):
            fp32_ok("coupled variant %d %s %s" % (variant, key, name), sim.field(medium, which),
                    o32[key][which], o64[key][which])
    fp32_ok("coupled variant %d pressure traces" % variant, sim.seismograms(), o32["seismograms"], o64["seismograms"])


def test_full_size_coupled_fp64_build(coupled_oracle):
    _, o64 = coupled_oracle
    sim = Simulation.structured(W.coupled(1.0, nstep=NSTEP_COUPLED, seismogram_types=("pressure",)), precision=64)
    sim.run_forward()
    for medium, key in MEDIA:
        for which, name in ((0, "u"), (1, "v"), (2, "a")):
            fp64_ok("coupled %s %s" % (key, name), sim.field(medium, which), o64[key][which])
    fp64_ok("coupled pressure traces", sim.seismograms(), o64["seismograms"])


def test_full_size_batched_shots():
    """The packed two-shots-per-lane kernel at full size, 64 shots."""
    from oracle import bridge
    p = W.batched(1.0, nshots=64, nstep=NSTEP_BATCHED)
    sim = Simulation.structured(p)
    info = sim.info()
    assert info.nshots == 64 and info.nspec == 320000 and info.nglob[0] == 5124801
    sim.run_forward()
    sim64 = Simulation.structured(p, precision=64)
    sim64.run_forward()
    for shot in (0, 63):
        o32 = bridge.forward(sim, 32, shot=shot, threads=THREADS, want_fields=True)
        o64 = bridge.forward(sim, 64, shot=shot, threads=THREADS, want_fields=True, exact=True)
        fp32_ok("batched shot %d traces" % shot, sim.seismograms(shot=shot), o32["seismograms"], o64["seismograms"])
        fp64_ok("batched shot %d traces" % shot, sim64.seismograms(shot=shot), o64["seismograms"])
        for which, name in ((0, "u"), (1, "v"), (2, "a")):
            fp32_ok("batched shot %d %s" % (shot, name), sim.field(0, which, shot=shot),
                    o32["psv"][which], o64["psv"][which])
            fp64_ok("batched shot %d %s" % (shot, name), sim64.field(0, which, shot=shot), o64["psv"][which])
