"""Edge cases of the forward path on the GPU against the oracle: seismogram
decimation, no receivers, a single time step, a one-element mesh, a mesh
smaller than one element chunk of the row kernel, and an odd shot count.
Displacement fields are compared where there are no seismograms."""
import numpy as np
import pytest

from specfempp_b200 import Simulation, StructuredProblem, Material, ForceSource, Station

pytestmark = pytest.mark.gpu

SOLID = Material(2700.0, 3000.0, 1732.0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def problem(nx=12, nz=10, nstep=200, stations=None, nsbs=1, nshots=1, absorb=(True, True, False, True)):
    dx, dz = 50.0, 50.0
    if stations is None:
        stations = [Station(x=dx * (1.5 + 2 * k), z=dz * (nz - 1.5)) for k in range(max(1, nx // 3))]
    return StructuredProblem(nx=nx, nz=nz, x0=0.0, x1=nx * dx, z0=0.0, z1=nz * dz, materials=[SOLID],
                             absorb=absorb, dt=2.5e-4, nstep=nstep, nshots=nshots,
                             sources=[ForceSource(x=nx * dx * (0.3 + 0.4 * s / max(1, nshots - 1)), z=nz * dz * 0.4,
                                                  f0=12.0, factor=1e10, shot=s) for s in range(nshots)],
                             stations=stations, seismogram_types=("displacement", "velocity"),
                             nstep_between_samples=nsbs)


def fields_match(sim, shot=0, tol=1e-5, which=0):
    """which: 0 displacement, 1 velocity, 2 acceleration."""
    from oracle import bridge
    gpu = sim.field(0, which, shot=shot)
    o32 = bridge.forward(sim, 32, shot=shot, threads=8, want_fields=True)["psv"][which]
    o64 = bridge.forward(sim, 64, shot=shot, threads=8, want_fields=True)["psv"][which]
    e32, e64, ref = rel_l2(gpu, o32), rel_l2(gpu, o64), rel_l2(o32, o64)
    print("field %d: rel-L2 vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)" % (which, e32, e64, ref))
    assert np.abs(o64).max() > 0
    assert e32 <= tol or e64 <= tol + 2.0 * ref


def seismograms_match(sim, shot=0, tol=1e-5):
    from oracle import bridge
    gpu = sim.seismograms(shot=shot)
    o32 = bridge.forward(sim, 32, shot=shot, threads=8)["seismograms"]
    o64 = bridge.forward(sim, 64, shot=shot, threads=8)["seismograms"]
    e32, e64, ref = rel_l2(gpu, o32), rel_l2(gpu, o64), rel_l2(o32, o64)
    print("seismograms %s: rel-L2 vs FP32 oracle %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
          % (gpu.shape, e32, e64, ref))
    assert np.abs(o64).max() > 0
    assert e32 <= tol or e64 <= tol + 2.0 * ref


def test_seismogram_decimation():
    """nstep_between_samples = 3: samples at steps 0, 3, 6, ... (the fused
    update's taps and the oracle's cadence)."""
    sim = Simulation.structured(problem(nsbs=3, nstep=240))
    sim.run_forward()
    info = sim.info()
    assert info.max_sig_step == 80
    seismograms_match(sim)


def test_no_receivers():
    sim = Simulation.structured(problem(stations=[]))
    sim.run_forward()
    assert sim.info().nreceivers == 0
    assert sim.seismograms().size == 0
    fields_match(sim)


def test_single_step():
    """One step: the displacement is still zero; velocity and acceleration
    carry the first force."""
    sim = Simulation.structured(problem(nstep=1))
    sim.run_forward()
    assert not np.abs(sim.field(0, 0)).any()
    fields_match(sim, which=1)
    fields_match(sim, which=2)


@pytest.mark.parametrize("nx,nz", [(1, 1), (3, 2)])
def test_meshes_smaller_than_a_chunk(nx, nz):
    """One element, and six elements: fewer than one 16- or 32-element chunk
    of the row kernel; every element is a boundary element."""
    p = problem(nx=nx, nz=nz, nstep=150, stations=[Station(x=25.0 * nx, z=30.0 * nz)])
    p.sources = [ForceSource(x=20.0 * nx, z=20.0 * nz, f0=40.0, factor=1e10)]
    p.dt = 1e-4
    sim = Simulation.structured(p)
    sim.run_forward()
    seismograms_match(sim)
    fields_match(sim)


def test_odd_shot_count():
    """S = 3: the one-shot-per-lane batched kernel; every shot against its own
    oracle run."""
    sim = Simulation.structured(problem(nshots=3, nstep=200))
    sim.run_forward()
    assert sim.info().stiffness_variant[0] == 3
    for s in range(3):
        seismograms_match(sim, shot=s)


def test_contexts_of_different_ngll_interleaved():
    """Two live contexts of different NGLL (5 and 8) in one process, their
    steps interleaved: each keeps its own GLL tables (one constant-memory
    bank per NGLL), so both still match the oracle."""
    from dataclasses import replace
    a = Simulation.structured(problem(nstep=200))
    b = Simulation.structured(replace(problem(nstep=200), ngll=8))
    a.run_forward(60)        # set up with NGLL 5 ...
    b.run_forward(60)        # ... then NGLL 8 ...
    a.run_forward(140)       # ... then NGLL 5 again
    b.run_forward(140)
    seismograms_match(a)
    seismograms_match(b)
