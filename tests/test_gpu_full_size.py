"""Parity at the benchmark's full sizes.  The coupled acoustic-elastic forward
on 400 x 300 NGLL=5 elements (1,924,402 points, the workload bench.py times),
1400 steps (the source sits mid-water, 1.5 km above the sea floor: the wave
reaches the elastic medium after about 1.25 s), final wavefields of both
media and the receivers' pressure traces against the FP32 and FP64 oracle on
identical inputs, for the compact-block kernel the autotuner picks there and
for the full-block kernel; and the batched 64-shot workload (800 x 400), two
of its shots against the oracle run of each alone.  Same bar as
test_gpu_forward.py:
    e(gpu, fp32) <= 1e-5  or  e(gpu, fp64) <= 1e-5 + 2 * e(fp32, fp64).
The oracle's CPU time is the limit on the step count (about 40 s per
precision on 16 host threads)."""
import os

import numpy as np
import pytest

from specfempp_b200 import Simulation
from specfempp_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5
NSTEP = 1400
MEDIA = ((0, "psv"), (3, "acoustic"))  # device medium index, oracle field key


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def oracle_fields():
    from oracle import bridge
    sim = Simulation.structured(W.coupled(1.0, nstep=NSTEP, seismogram_types=("pressure",)))
    threads = max(1, min(32, os.cpu_count() or 1))
    o32 = bridge.forward(sim, 32, threads=threads, want_fields=True)
    o64 = bridge.forward(sim, 64, threads=threads, want_fields=True)
    return o32, o64


@pytest.mark.parametrize("variant", [3, 1])
def test_full_size_coupled_fields(oracle_fields, variant):
    o32, o64 = oracle_fields
    sim = Simulation.structured(W.coupled(1.0, nstep=NSTEP, seismogram_types=("pressure",)))
    info = sim.info()
    assert info.nglob[0] + info.nglob[3] == 1924402 or info.nspec == 120000
    for medium, _ in MEDIA:
        sim.set_stiffness_variant(medium, variant)
    sim.run_forward()
    for medium, key in MEDIA:
        for which, name in ((0, "u"), (1, "v"), (2, "a")):
            g = sim.field(medium, which)
            assert np.isfinite(g).all()
            assert np.abs(o64[key][which]).max() > 0, (key, name)
            e32, e64 = rel_l2(g, o32[key][which]), rel_l2(g, o64[key][which])
            eref = rel_l2(o32[key][which], o64[key][which])
            print("variant %d %s %s: vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
                  % (variant, key, name, e32, e64, eref))
            assert e32 <= TOL_FP32 or e64 <= TOL_FP32 + 2.0 * eref, (variant, key, name, e32, e64, eref)
    seis = sim.seismograms()
    s32, s64 = o32["seismograms"], o64["seismograms"]
    assert np.isfinite(seis).all() and np.abs(s64).max() > 0
    e32, e64, eref = rel_l2(seis, s32), rel_l2(seis, s64), rel_l2(s32, s64)
    print("variant %d pressure traces: vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
          % (variant, e32, e64, eref))
    assert e32 <= TOL_FP32 or e64 <= TOL_FP32 + 2.0 * eref, (variant, "traces", e32, e64, eref)


def test_full_size_batched_shots():
    """The batched workload at full size (800 x 400 NGLL=5 elements, 5.1 M
    points, 64 shots in one context, the packed two-shots-per-lane kernel):
    the first and the last shot's final P-SV fields after 300 steps against
    the oracle run of that shot alone."""
    from oracle import bridge
    nstep = 300
    sim = Simulation.structured(W.batched(1.0, nshots=64, nstep=nstep))
    assert sim.info().nshots == 64
    sim.run_forward()
    threads = max(1, min(32, os.cpu_count() or 1))
    for shot in (0, 63):
        o32 = bridge.forward(sim, 32, shot=shot, threads=threads, want_fields=True)["psv"]
        o64 = bridge.forward(sim, 64, shot=shot, threads=threads, want_fields=True)["psv"]
        for which, name in ((0, "u"), (1, "v"), (2, "a")):
            g = sim.field(0, which, shot=shot)
            assert np.isfinite(g).all() and np.abs(o64[which]).max() > 0, (shot, name)
            e32, e64, eref = rel_l2(g, o32[which]), rel_l2(g, o64[which]), rel_l2(o32[which], o64[which])
            print("batched shot %d %s: vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
                  % (shot, name, e32, e64, eref))
            assert e32 <= TOL_FP32 or e64 <= TOL_FP32 + 2.0 * eref, (shot, name, e32, e64, eref)
