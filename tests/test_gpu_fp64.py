"""GPU parity at FP64 rounding level: the FP64 verification build of the
device path against the FP64 oracle, on identical inputs.

The FP32 parity tests cannot tell a kernel defect from rounding: an FP32
run of an ill-conditioned problem is one realisation of its rounding error
(up to 1e-4 from FP64 at NGLL 8).  Here the same kernel sources -- the
scalar shot-parallel stiffness (single shot and batched, NGLL 5 and 8, with
Stacey, free surface, sources, coupling and the in-launch update of
element-private points), the fused update with its seismogram taps, the
unfused Newmark pieces, sources, coupling and receiver kernels, the Frechet
kernels, the mass matrix, Kahan sums and snapshot restores -- are compiled
with FP64 arithmetic (libspecfem_b200_fp64.so) and compared with the
oracle's FP64 run of the same discrete problem (FP32 inputs and FP32
constants, as the reference's type_real) with every output kept in FP64.
A wrong index, coefficient or step order shows at 1e-8 or worse; the bar is
1e-10 relative L2.  FP32-only kernels (the bulk-copy fed row kernels, the
compact block and the packed f32x2 kernels) are checked against these FP32
kernels operator by operator in test_gpu_operators.py.
Every case goes through the C ABI.
"""
import numpy as np
import pytest

from adjoint_util import anomaly, base_model, observed, problem
from specfempp_b200 import ForceSource, Material, Simulation, Station, StructuredProblem
from specfempp_b200 import workloads as W

pytestmark = pytest.mark.gpu

BAR = 1e-10


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def exact(sim, shot=0, fields=False, stacey=False):
    from oracle import bridge
    return bridge.forward(sim, 64, shot=shot, threads=8, want_fields=fields, want_stacey=stacey, exact=True)


def check_forward(p, label, shots=(0,), graph=True, compensated=False, unfused=False, fields=True):
    sim = Simulation.structured(p, precision=64)
    if compensated:
        sim.set_newmark_compensation(True)
    if unfused:
        sim.run_forward_unfused()
    else:
        sim.run_forward(graph=graph)
    worst = 0.0
    for s in shots:
        ref = exact(sim, s, fields=fields)
        gpu = sim.seismograms(shot=s)
        assert gpu.dtype == np.float64 and np.isfinite(gpu).all()
        assert np.abs(ref["seismograms"]).max() > 0
        e = rel_l2(gpu, ref["seismograms"])
        print("%s shot %d: FP64 seismograms rel-L2 vs FP64 oracle %.2e" % (label, s, e))
        assert e <= BAR, (label, s, e)
        worst = max(worst, e)
        if not fields:
            continue
        info = sim.info()
        for name, m in (("psv", 0), ("sh", 1), ("acoustic", 3)):
            if info.nglob[m] == 0:
                continue
            for which in range(4):
                g = sim.field(m, which, shot=s)
                e = rel_l2(g, ref[name][which])
                assert e <= BAR, (label, s, name, which, e)
                worst = max(worst, e)
    return sim, worst


def small_elastic(sh=False, nstep=400, types=("displacement", "velocity", "acceleration", "pressure")):
    p = W.plain_elastic(scale=0.2, nstep=nstep, seismogram_types=types)
    p.elastic_sh = sh
    return p


def acoustic_problem(nshots=1, nstep=300):
    return StructuredProblem(nx=20, nz=16, x0=0, x1=1000, z0=0, z1=800,
                             materials=[Material(1020.0, 1500.0, 0.0)],
                             absorb=(True, True, False, True), dt=5e-4, nstep=nstep, nshots=nshots,
                             sources=[ForceSource(x=380 + 200 * s, z=410, f0=6.0, factor=1e10, shot=s)
                                      for s in range(nshots)],
                             stations=[Station(x=100 + 80 * k, z=700) for k in range(10)],
                             seismogram_types=("displacement", "velocity", "acceleration", "pressure"))


def test_fp64_library_is_fp64():
    from specfempp_b200 import _capi
    assert _capi.load(64).sfb_real_bytes() == 8


def test_fp64_elastic_psv_stacey_free_surface():
    sim, _ = check_forward(small_elastic(), "P-SV")
    assert sim.info().private_points > 0  # in-launch update of element-private points ran


def test_fp64_elastic_psv_eager_launches():
    check_forward(small_elastic(nstep=120), "P-SV eager", graph=False)


def test_fp64_elastic_sh():
    check_forward(small_elastic(sh=True, types=("displacement", "velocity", "acceleration")), "SH")


def test_fp64_acoustic_free_surface_and_stacey():
    check_forward(acoustic_problem(), "acoustic")


def test_fp64_coupled_acoustic_elastic():
    check_forward(W.coupled(scale=0.06, nstep=300, seismogram_types=("pressure", "displacement", "velocity")),
                  "coupled")


def test_fp64_batched_shots():
    check_forward(W.batched(scale=0.04, nshots=4, nstep=250,
                            seismogram_types=("displacement", "velocity", "acceleration")),
                  "batched", shots=range(4))


def test_fp64_batched_sh_and_acoustic():
    p = small_elastic(sh=True, nstep=250, types=("displacement", "velocity"))
    p.nshots = 2
    p.sources = [ForceSource(x=1000.0 + 1000.0 * s, z=1500.0, f0=10.0, factor=1e10, shot=s) for s in range(2)]
    check_forward(p, "SH batched", shots=range(2))
    check_forward(acoustic_problem(nshots=2), "acoustic batched", shots=range(2))


def test_fp64_kahan_compensated():
    p = small_elastic(nstep=600, types=("displacement", "velocity"))
    p.dt = 1e-4
    check_forward(p, "P-SV compensated", compensated=True)
    check_forward(W.batched(scale=0.04, nshots=2, nstep=250), "batched compensated", shots=range(2),
                  compensated=True)


def test_fp64_unfused_reference_granularity_path():
    """Predictor, coupling, sources, stiffness, divide, corrector and the
    receiver kernel as separate launches (sfb_run_forward_unfused)."""
    check_forward(small_elastic(nstep=150), "P-SV unfused", unfused=True)
    check_forward(W.coupled(scale=0.06, nstep=150, seismogram_types=("pressure", "displacement")),
                  "coupled unfused", unfused=True)


@pytest.mark.parametrize("nshots", [1, 2])
def test_fp64_gll7(nshots):
    for label, sh, vs, types in (("P-SV", False, 1732.0, ("displacement", "velocity")),
                                 ("SH", True, 1732.0, ("displacement",)),
                                 ("acoustic", False, 0.0, ("pressure",))):
        p = small_elastic(sh=sh, nstep=250, types=types)
        p.ngll = 8
        p.nx, p.nz = 10, 8
        p.x1, p.z1 = 10 * 80.0, 8 * 75.0
        p.materials = [Material(2700.0 if vs else 1020.0, 3000.0 if vs else 1500.0, vs)]
        p.dt = 2.5e-4
        p.nshots = nshots
        p.sources = [ForceSource(x=300.0 + 200.0 * s, z=300.0, f0=10.0 if vs else 6.0, factor=1e10, shot=s)
                     for s in range(nshots)]
        p.stations = [Station(x=100.0 + 150.0 * k, z=500.0) for k in range(4)]
        check_forward(p, "GLL7 %s S=%d" % (label, nshots), shots=range(nshots))


@pytest.mark.parametrize("kind", ["psv", "sh", "acoustic", "coupled"])
def test_fp64_seismograms_of_given_fields(kind):
    """The receiver kernel on fields set through the ABI, all four types,
    corner / edge / interior stations and a receiver angle."""
    from oracle import bridge
    solid, fluid = Material(2700.0, 3000.0, 1732.0), Material(1020.0, 1500.0, 0.0)
    nx, nz = 10, 8
    mats, emat = [solid], None
    if kind == "acoustic":
        mats = [fluid]
    elif kind == "coupled":
        mats = [solid, fluid]
        emat = np.zeros((nz, nx), np.int32)
        emat[5:, :] = 1
        emat = emat.ravel()
    types = ("displacement", "velocity", "acceleration") if kind == "sh" else \
        ("displacement", "velocity", "acceleration", "pressure")
    stations = [Station(x=300, z=400), Station(x=350, z=400), Station(x=425, z=530, angle=30.0),
                Station(x=610, z=180), Station(x=700, z=650), Station(x=120, z=710)]
    p = StructuredProblem(nx=nx, nz=nz, x0=0, x1=1000, z0=0, z1=800, materials=mats, element_material=emat,
                          elastic_sh=(kind == "sh"), dt=1e-4, nstep=10, nshots=1,
                          sources=[ForceSource(x=500, z=250, f0=5.0)],
                          stations=stations, seismogram_types=types)
    sim = Simulation.structured(p, precision=64)
    info = sim.info()
    rng = np.random.default_rng(11)
    fields = {}
    for m, nc in ((0, 2), (1, 1), (3, 1)):
        if info.nglob[m] == 0:
            continue
        arrs = tuple(rng.standard_normal((nc, info.nglob[m])).astype(np.float32) for _ in range(3))
        for which, a in enumerate(arrs):
            sim.set_field(m, which, a)
        fields[{0: "psv", 1: "sh", 3: "acoustic"}[m]] = arrs
    sim.compute_seismograms(0)
    gpu = sim.seismograms()[0]
    ref = bridge.seismograms(sim, fields, 64, exact=True)
    for t, name in enumerate(types):  # per type: pressure is ~1e9 times the others here
        e = rel_l2(gpu[t], ref[t])
        print("%s %s: FP64 receiver kernel vs FP64 oracle %.2e" % (kind, name, e))
        assert np.abs(ref[t]).max() > 0 and e <= BAR, (kind, name, e)


def fp64_combined(nshots=1, absorb=(True, True, False, True), checkpoint_interval=0, nstep=300):
    p, model, XZ = base_model(nshots=nshots, nstep=nstep)
    obs = observed(anomaly(model, XZ, p), nstep, absorb, nshots=nshots)
    sim = Simulation.structured(problem(model, nstep, absorb, nshots), precision=64)
    if checkpoint_interval:
        sim.set_checkpoint_interval(checkpoint_interval)
    sim.run_forward()
    stfs = []
    for s in range(nshots):
        stf = (sim.seismograms(shot=s)[:, 0] - obs[s]).astype(np.float32)
        stfs.append(stf)
        sim.set_adjoint_sources(stf, shot=s)
    sim.run_combined()
    return sim, stfs


def exact_kernels(sim, stfs):
    from oracle import bridge
    total = None
    for s, stf in enumerate(stfs):
        fwd = exact(sim, s, fields=True, stacey=True)
        K = bridge.combined(sim, stf, fwd, precision=64, shot=s, threads=8, exact=True)
        total = K if total is None else total + K
    return total


@pytest.mark.parametrize("absorb", [(False,) * 4, (True, True, False, True)])
@pytest.mark.parametrize("nshots", [1, 2])
def test_fp64_combined_kernels(absorb, nshots):
    """Adjoint + backward (Stacey replay) + Frechet kernels."""
    sim, stfs = fp64_combined(nshots, absorb)
    K = np.stack([sim.kernels(q) for q in range(3)], axis=-1)
    ref = exact_kernels(sim, stfs)
    for c, name in enumerate(("rho", "mu", "kappa")):
        e = rel_l2(K[..., c], ref[..., c])
        print("S=%d absorb=%s kernel %s: FP64 rel-L2 vs FP64 oracle %.2e" % (nshots, absorb, name, e))
        assert np.abs(ref[..., c]).max() > 0
        assert e <= BAR, (name, e)


def test_fp64_backward_seismograms():
    """The backward wavefield's seismograms (reconstruction through the
    Stacey replay) against the oracle's exact backward run."""
    from oracle import bridge
    sim, stfs = fp64_combined(1)
    fwd = exact(sim, 0, fields=True, stacey=True)
    _, bseis = bridge.combined(sim, stfs[0], fwd, precision=64, threads=8, want_backward_seismograms=True,
                               exact=True)
    e = rel_l2(sim.seismograms(wavefield=2), bseis)
    print("backward seismograms: FP64 rel-L2 vs FP64 oracle %.2e" % e)
    assert e <= BAR


def test_fp64_acoustic_kernels():
    p = acoustic_problem(nstep=300)
    p.seismogram_types = ("pressure",)
    p.save_boundary_values = True
    sim = Simulation.structured(p, precision=64)
    sim.run_forward()
    rng = np.random.default_rng(5)
    t = np.arange(300) * 5e-4
    stf = np.zeros((300, 10, 2), np.float32)
    for r in range(10):
        a = (np.pi * 8.0 * (t - rng.uniform(0.03, 0.12))) ** 2
        stf[:, r, 0] = (rng.uniform(0.5, 1.5) * 1e-3 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    sim.set_adjoint_sources(stf)
    sim.run_combined()
    # The acoustic potential reconstructed backward through the Stacey replay
    # amplifies rounding far more than the elastic cases: two FP64 oracle
    # runs that differ only in their summation order (thread count) are
    # 1e-8 apart here.  The bar is 1e-10 or, above it, that measured spread.
    from oracle import bridge
    refs = []
    for threads in (1, 8):
        fwd = bridge.forward(sim, 64, threads=threads, want_fields=True, want_stacey=True, exact=True)
        refs.append(bridge.combined(sim, stf, fwd, precision=64, threads=threads, exact=True))
    for which, col in ((0, 0), (2, 1), (3, 2)):
        e = rel_l2(sim.kernels(which), refs[1][..., col])
        spread = rel_l2(refs[0][..., col], refs[1][..., col])
        print("acoustic kernel %d: FP64 rel-L2 vs FP64 oracle %.2e (two FP64 oracle runs: %.2e)" % (which, e, spread))
        assert e <= max(BAR, 2.0 * spread), (which, e, spread)


def test_fp64_checkpointed_combined_keeps_kernels():
    """Snapshots restored into the backward wavefield every 50 steps: in FP64
    the reconstruction drift is at rounding level, so the kernels equal the
    oracle's pure reconstruction to the same bar."""
    sim, stfs = fp64_combined(2, checkpoint_interval=50)
    K = np.stack([sim.kernels(q) for q in range(3)], axis=-1)
    ref = exact_kernels(sim, stfs)
    for c in range(3):
        e = rel_l2(K[..., c], ref[..., c])
        print("checkpointed kernel %d: FP64 rel-L2 vs FP64 oracle %.2e" % (c, e))
        assert e <= BAR


def test_fp64_stacey_traction_kernels():
    """The Stacey-traction model derivatives (sfb_set_stacey_kernels) of the
    FP64 build against the oracle's, all sides absorbing."""
    from oracle import bridge
    nstep = 600
    absorb = (True,) * 4
    p, model, XZ = base_model(nshots=2, nstep=nstep)
    obs = observed(anomaly(model, XZ, p), nstep, absorb, nshots=2)
    sim = Simulation.structured(problem(model, nstep, absorb, 2), precision=64)
    sim.set_stacey_kernels(True)
    sim.run_forward()
    stfs = []
    for s in range(2):
        stf = (sim.seismograms(shot=s)[:, 0] - obs[s]).astype(np.float32)
        stfs.append(stf)
        sim.set_adjoint_sources(stf, shot=s)
    sim.run_combined()
    ref = None
    for s in range(2):
        fwd = exact(sim, s, fields=True, stacey=True)
        _, kb = bridge.combined(sim, stfs[s], fwd, precision=64, shot=s, threads=8, exact=True, stacey_kernels=True)
        ref = kb if ref is None else ref + kb
    for q in (0, 1):
        e = rel_l2(sim.kernels(6 + q), ref[..., q])
        print("Stacey-traction kernel %d: FP64 build vs FP64 oracle %.2e" % (q, e))
        assert np.abs(ref[..., q]).max() > 0 and e <= BAR
