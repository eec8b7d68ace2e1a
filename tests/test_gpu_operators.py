"""Operator-level parity of every FP32 stiffness kernel variant against the
FP64 verification build, from identical random states.

The FP32-only kernels (bulk-copy fed row kernels with 32- and 16-element
chunks, the compact block of affine elements, the packed f32x2 two-shot
kernel and its Frechet-fused form) have no FP64 instantiation.  Over a few
steps from a random state the rounding of an FP32 run stays at its
single-operation level (~1e-7), so each variant's fields after three fused
steps (stiffness with Stacey, free surface, sources, coupling and the
in-launch update of element-private points, then the fused update and its
seismogram taps) and its Frechet kernels after a three-step combined run
are compared with the FP64 build's (itself held to the FP64 oracle at
1e-10 in test_gpu_fp64.py) at 1e-6 relative L2 (measured: 0.9-2.3e-7);
a wrong index or coefficient shows at 1e-2 or worse.  Every case goes through the C ABI.
"""
import numpy as np
import pytest

from specfempp_b200 import ForceSource, Material, Simulation, Station, StructuredProblem
from specfempp_b200 import workloads as W

pytestmark = pytest.mark.gpu

BAR = 1e-6
NSTEP = 3


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def media(sim):
    info = sim.info()
    return [(m, 2 if m == 0 else 1) for m in (0, 1, 3) if info.nglob[m] > 0]


def random_state(sim, seed=7):
    """u, v, a of every medium and shot, smooth enough that the step stays
    stable: seeded values of unit size."""
    rng = np.random.default_rng(seed)
    info = sim.info()
    state = {}
    for s in range(info.nshots):
        for m, nc in media(sim):
            for which, scale in ((0, 1e-3), (1, 1e-2), (2, 1.0)):
                state[(s, m, which)] = (scale * rng.standard_normal((nc, info.nglob[m]))).astype(np.float32)
    return state


def load_state(sim, state):
    for (s, m, which), a in state.items():
        sim.set_field(m, which, a, shot=s)


def run_steps(p, precision, variant=None, state=None):
    sim = Simulation.structured(p, precision=precision)
    if variant is not None:
        for m in (0, 1, 3):
            sim.set_stiffness_variant(m, variant)
    load_state(sim, state)
    sim.run_forward(NSTEP)
    return sim


def compare(sim32, sim64, label):
    info = sim32.info()
    worst = 0.0
    for s in range(info.nshots):
        for m, _ in media(sim32):
            for which in range(3):
                e = rel_l2(sim32.field(m, which, shot=s), sim64.field(m, which, shot=s))
                worst = max(worst, e)
                assert e <= BAR, (label, s, m, which, e)
        e = rel_l2(sim32.seismograms(shot=s)[:NSTEP], sim64.seismograms(shot=s)[:NSTEP])
        worst = max(worst, e)
        assert e <= BAR, (label, s, "seismograms", e)
    print("%s: worst rel-L2 of the FP32 kernels vs the FP64 build after %d steps: %.2e" % (label, NSTEP, worst))
    return worst


def small(p, types=("displacement", "velocity", "acceleration", "pressure")):
    p.nstep = NSTEP
    p.seismogram_types = types
    return p


CASES = {
    "psv": lambda: small(W.plain_elastic(scale=0.2, nstep=NSTEP)),
    "coupled": lambda: small(W.coupled(scale=0.06, nstep=NSTEP), ("pressure", "displacement")),
    "sh": lambda: small(W.plain_elastic(scale=0.2, nstep=NSTEP), ("displacement", "velocity")),
    "acoustic": lambda: StructuredProblem(nx=20, nz=16, x0=0, x1=1000, z0=0, z1=800,
                                          materials=[Material(1020.0, 1500.0, 0.0)],
                                          absorb=(True, True, False, True), dt=5e-4, nstep=NSTEP,
                                          sources=[ForceSource(x=480, z=410, f0=6.0, factor=1e10)],
                                          stations=[Station(x=100 + 80 * k, z=700) for k in range(10)],
                                          seismogram_types=("pressure", "displacement")),
}


def make(case, nshots=1):
    p = CASES[case]()
    if case == "sh":
        p.elastic_sh = True
    if nshots > 1:
        p.nshots = nshots
        xs = np.linspace(p.x0 + 0.2 * (p.x1 - p.x0), p.x0 + 0.8 * (p.x1 - p.x0), nshots)
        src = p.sources[0]
        p.sources = [ForceSource(x=float(x), z=src.z, f0=src.f0, factor=src.factor, shot=s)
                     for s, x in enumerate(xs)]
    return p


@pytest.mark.parametrize("case", ["psv", "coupled", "sh", "acoustic"])
@pytest.mark.parametrize("variant", [1, 2, 3])
def test_single_shot_variants_match_fp64_build(case, variant):
    """Row kernel with 32- and 16-element chunks, compact-block kernel."""
    p = make(case)
    probe = Simulation.structured(p)
    state = random_state(probe)
    sim32 = run_steps(p, 32, variant, state)
    sim64 = run_steps(p, 64, None, state)
    info = sim32.info()
    for m in (0, 1, 3):
        if info.nelements[m]:
            assert info.stiffness_variant[m] == variant
    compare(sim32, sim64, "%s single-shot variant %d" % (case, variant))


@pytest.mark.parametrize("case", ["psv", "sh", "acoustic"])
@pytest.mark.parametrize("variant", [1, 2, 3])
def test_batched_variants_match_fp64_build(case, variant):
    """Packed f32x2 two-shot kernel (geometry constants of affine elements),
    scalar two-shot kernel, one shot per lane."""
    p = make(case, nshots=4)
    probe = Simulation.structured(p)
    state = random_state(probe)
    sim32 = run_steps(p, 32, variant, state)
    sim64 = run_steps(p, 64, None, state)
    compare(sim32, sim64, "%s batched variant %d" % (case, variant))


@pytest.mark.parametrize("nshots", [1, 2])
def test_gll7_kernels_match_fp64_build(nshots):
    for case in ("psv", "sh", "acoustic"):
        p = make(case, nshots)
        p.ngll = 8
        p.nx, p.nz = 10, 8
        p.x0, p.z0 = 0.0, 0.0
        p.x1, p.z1 = 10 * 80.0, 8 * 75.0
        p.dt = 2.5e-4
        for k, s in enumerate(p.sources):
            s.x, s.z = 300.0 + 200.0 * k, 300.0
        p.stations = [Station(x=100.0 + 150.0 * k, z=500.0) for k in range(4)]
        probe = Simulation.structured(p)
        state = random_state(probe)
        compare(run_steps(p, 32, None, state), run_steps(p, 64, None, state), "GLL7 %s S=%d" % (case, nshots))


def test_non_affine_mesh_kernels_match_fp64_build(tmp_path):
    """General bilinear elements (control nodes moved by a topography-like
    map): the full static block in the row kernels and per-point geometry
    in the packed kernel."""
    import math
    import workflow_util as WU
    cfg = WU.write_forward(str(tmp_path), NSTEP, 2.5e-4,
                           deform=lambda x, z: (x, z + 25.0 * math.sin(2.0 * math.pi * x / WU.LX) * z / WU.LZ))
    for variant in (1, 2, 3):
        sim32 = Simulation.from_yaml(cfg)
        sim32.set_stiffness_variant(0, variant)
        state = random_state(sim32)
        load_state(sim32, state)
        sim32.run_forward(NSTEP)
        sim64 = Simulation.from_yaml(cfg, precision=64)
        load_state(sim64, state)
        sim64.run_forward(NSTEP)
        compare(sim32, sim64, "non-affine variant %d" % variant)


@pytest.mark.parametrize("nshots", [1, 2, 3, 4])
def test_frechet_kernels_match_fp64_build(nshots):
    """A three-step forward from a random state, then the combined run with
    seeded adjoint sources: the Frechet kernels of the FP32 path (for even S
    fused into the packed backward stiffness launch, which also finishes the
    element-private points of both wavefields) against the FP64 build's."""
    p = make("psv", nshots)
    p.absorb = (True, True, False, True)
    p.save_boundary_values = True
    p.seismogram_types = ("displacement",)
    probe = Simulation.structured(p)
    state = random_state(probe)
    info = probe.info()
    rng = np.random.default_rng(3)
    adj = [(1e-3 * rng.standard_normal((NSTEP, info.nreceivers, 2))).astype(np.float32) for _ in range(nshots)]
    out = []
    for precision in (32, 64):
        sim = Simulation.structured(p, precision=precision)
        load_state(sim, state)
        sim.run_forward(NSTEP)
        for s in range(nshots):
            sim.set_adjoint_sources(adj[s], shot=s)
        sim.run_combined()
        out.append(np.stack([sim.kernels(q) for q in range(3)], axis=-1))
    for c, name in enumerate(("rho", "mu", "kappa")):
        e = rel_l2(out[0][..., c], out[1][..., c])
        print("S=%d kernel %s: FP32 path vs FP64 build %.2e" % (nshots, name, e))
        assert np.abs(out[1][..., c]).max() > 0
        assert e <= BAR, (name, e)
