"""Runs driven by moment-tensor sources on the GPU, through the C ABI:
single shot (explosion and a double couple) and a batched run with one
random double couple per shot (seeded strike angles), against the FP32 /
FP64 oracle; the FP64 build against the FP64 oracle at 1e-10."""
import numpy as np
import pytest

from specfempp_b200 import ForceSource, Material, Simulation, Station, StructuredProblem

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def double_couple(theta):
    """In-plane double couple with fault strike angle theta (radians)."""
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    return float(s), float(-s), float(c)


def problem(nshots, tensors):
    srcs = [ForceSource(x=700.0 + 400.0 * k, z=850.0, f0=12.0, factor=1e10, kind="moment_tensor",
                        mxx=mt[0], mzz=mt[1], mxz=mt[2], shot=k) for k, mt in enumerate(tensors)]
    return StructuredProblem(nx=40, nz=32, x0=0.0, x1=2000.0, z0=0.0, z1=1600.0,
                             materials=[Material(2700.0, 3000.0, 1732.0)], absorb=(True, True, False, True),
                             dt=2.5e-4, nstep=500, nshots=nshots, sources=srcs,
                             stations=[Station(x=100.0 + 90.0 * k, z=1500.0) for k in range(20)],
                             seismogram_types=("displacement", "velocity", "pressure"))


@pytest.mark.parametrize("label,tensors", [("explosion", [(1.0, 1.0, 0.0)]),
                                           ("double couple", [double_couple(0.3)]),
                                           ("batched double couples",
                                            [double_couple(t) for t in np.random.default_rng(5).uniform(0, np.pi, 4)])])
def test_moment_tensor_runs_match_oracle(label, tensors):
    from oracle import bridge
    p = problem(len(tensors), tensors)
    sim = Simulation.structured(p)
    sim.run_forward()
    sim64 = Simulation.structured(p, precision=64)
    sim64.run_forward()
    for s in range(len(tensors)):
        g = sim.seismograms(shot=s)
        o32 = bridge.forward(sim, 32, shot=s, threads=8)["seismograms"]
        o64 = bridge.forward(sim, 64, shot=s, threads=8, exact=True)["seismograms"]
        e32, e64, eref = rel_l2(g, o32), rel_l2(g, o64), rel_l2(o32, o64)
        e = rel_l2(sim64.seismograms(shot=s), o64)
        print("%s shot %d: FP32 vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e); FP64 build %.2e"
              % (label, s, e32, e64, eref, e))
        assert np.abs(o64).max() > 0
        assert e32 <= 1e-5 or e64 <= 1e-5 + 2.0 * eref
        assert e <= 1e-10
