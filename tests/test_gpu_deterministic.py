"""The deterministic assembly mode (sfb_set_deterministic): element colours,
one stiffness launch per colour, fixed-order sums for sources, coupling,
seismograms and the mass matrix.

  * two runs of the same problem give bit-identical seismograms, fields and
    Frechet kernels: single shot (row kernel), batched (packed kernel),
    coupled, the combined loop with the Frechet-fused backward launch;
  * the FP64 build in this mode meets the FP64 oracle at 1e-10, on a
    structured mesh and on one of the reference's own meshes (9-node
    elements, more colours), so the colour split and the owner-computes
    sums compute the same operator;
  * the FP32 results meet the usual parity bar against the oracle.
Every case goes through the C ABI.
"""
import numpy as np
import pytest

from adjoint_util import anomaly, base_model, observed, problem
from golden_util import fixture_case
from specfempp_b200 import Simulation
from specfempp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def det_sim(p, precision=32):
    sim = Simulation.structured(p, precision=precision)
    sim.set_deterministic(True)
    return sim


def outputs(sim):
    info = sim.info()
    out = []
    for s in range(info.nshots):
        out.append(sim.seismograms(shot=s))
        for m in (0, 1, 3):
            if info.nglob[m]:
                for which in range(3):
                    out.append(sim.field(m, which, shot=s))
    return out


def assert_identical(a, b, label):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        assert np.array_equal(x, y), (label, float(np.max(np.abs(x.astype(np.float64) - y))))


@pytest.mark.parametrize("case", ["plain", "coupled", "batched"])
def test_forward_runs_are_bit_identical(case):
    if case == "plain":
        p = W.plain_elastic(scale=0.2, nstep=300, seismogram_types=("displacement", "velocity", "pressure"))
    elif case == "coupled":
        p = W.coupled(scale=0.06, nstep=300, seismogram_types=("pressure", "displacement"))
    else:
        p = W.batched(scale=0.04, nshots=4, nstep=250, seismogram_types=("displacement", "velocity"))
    runs = []
    for _ in range(2):
        sim = det_sim(p)
        sim.run_forward()
        runs.append(outputs(sim))
    assert_identical(runs[0], runs[1], case)
    # parity against the oracle as in the atomic mode
    from oracle import bridge
    sim = det_sim(p)
    sim.run_forward()
    for s in range(min(2, p.nshots)):
        g = sim.seismograms(shot=s)
        o32 = bridge.forward(sim, 32, shot=s, threads=8)["seismograms"]
        o64 = bridge.forward(sim, 64, shot=s, threads=8, exact=True)["seismograms"]
        e32, e64, eref = rel_l2(g, o32), rel_l2(g, o64), rel_l2(o32, o64)
        print("%s deterministic shot %d: vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
              % (case, s, e32, e64, eref))
        assert e32 <= 1e-5 or e64 <= 1e-5 + 2.0 * eref


@pytest.mark.parametrize("nshots", [1, 2])
def test_combined_kernels_are_bit_identical(nshots):
    absorb = (True, True, False, True)
    p, model, XZ = base_model(nshots=nshots, nstep=300)
    obs = observed(anomaly(model, XZ, p), 300, absorb, nshots=nshots)
    ks = []
    for _ in range(2):
        sim = det_sim(problem(model, 300, absorb, nshots))
        sim.run_forward()
        for s in range(nshots):
            sim.set_adjoint_sources((sim.seismograms(shot=s)[:, 0].astype(np.float64) - obs[s]).astype(np.float32),
                                    shot=s)
        sim.run_combined()
        ks.append([sim.kernels(q) for q in range(3)] + [sim.seismograms(wavefield=2, shot=s) for s in range(nshots)])
    assert_identical(ks[0], ks[1], "combined S=%d" % nshots)


def test_fp64_deterministic_mode_meets_oracle():
    from oracle import bridge
    for p in (W.coupled(scale=0.06, nstep=300, seismogram_types=("pressure", "displacement")),
              W.batched(scale=0.04, nshots=2, nstep=250)):
        sim = det_sim(p, precision=64)
        sim.run_forward()
        for s in range(p.nshots):
            ref = bridge.forward(sim, 64, shot=s, threads=8, exact=True)["seismograms"]
            e = rel_l2(sim.seismograms(shot=s), ref)
            print("FP64 deterministic shot %d: vs FP64 oracle %.2e" % (s, e))
            assert e <= 1e-10


def test_fp64_deterministic_mode_on_a_reference_mesh(tmp_path):
    """AcousticElasticCoupledDomain: the reference's 9-node mesh with its
    fluid-solid interface, in the deterministic mode."""
    from oracle import bridge
    cfg, _, _ = fixture_case("AcousticElasticCoupledDomain", str(tmp_path))
    sim = Simulation.from_yaml(cfg, precision=64)
    sim.set_deterministic(True)
    sim.run_forward()
    ref = bridge.forward(sim, 64, threads=8, exact=True)["seismograms"]
    e = rel_l2(sim.seismograms(), ref)
    print("reference coupled mesh, FP64 deterministic: vs FP64 oracle %.2e" % e)
    assert e <= 1e-10
    runs = []
    for _ in range(2):
        s32 = Simulation.from_yaml(cfg)
        s32.set_deterministic(True)
        s32.run_forward()
        runs.append(outputs(s32))
    assert_identical(runs[0], runs[1], "reference coupled mesh")


def test_mode_is_chosen_before_device_use():
    from specfempp_b200 import SfbError
    sim = Simulation.structured(W.plain_elastic(scale=0.1, nstep=10))
    sim.run_forward(1)
    with pytest.raises(SfbError):
        sim.set_deterministic(True)
