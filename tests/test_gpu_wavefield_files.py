"""Forward wavefield files in the reference's layout
(include/io/wavefield/{writer,reader}.tpp, compute/boundary_values/*),
through the C ABI:

  * Boundary/Stacey/IndexMapping numbers, per medium with a container
    (elastic_psv, acoustic) and in mesh order, the elements whose boundary
    tag is stacey -- Stacey points and no acoustic free-surface point
    (enumerations/boundary.hpp:50-105), recomputed here from the problem;
    ElasticAcceleration / AcousticAcceleration hold their element-local
    accelerations (nelements, nz, nx, nstep, ncomp) column-major, checked
    against the oracle's store; the empty poroelastic / elastic_psv_t
    groups the reference's reader opens are present;
  * a second context that reads the file runs the combined loop to the
    same kernels as the context that wrote it (deterministic mode: bit for
    bit);
  * `time_interval` snapshots (periodic_tasks/wavefield_writer.hpp) hold
    the state after their step: equal to a run stopped there.
"""
import os

import numpy as np
import pytest

from specfempp_b200 import Material, ForceSource, Simulation, Station, StructuredProblem
from specfempp_b200.__main__ import run

pytestmark = pytest.mark.gpu

NSTEP = 250


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def read_ds(folder, name):
    meta = open(os.path.join(folder, name + ".meta")).read().split("\n")
    dims = [int(x) for x in meta[1].split()[1:]]
    path = os.path.join(folder, name + ".txt")
    vals = np.loadtxt(path) if os.path.getsize(path) else np.zeros(0)
    return dims, np.atleast_1d(vals)


def coupled_problem():
    """Water over rock, free surface on top, Stacey elsewhere: the acoustic
    top corner elements are composite Stacey / Dirichlet."""
    nx, nz = 16, 12
    em = np.zeros((nz, nx), np.int32)
    em[8:, :] = 1
    return StructuredProblem(nx=nx, nz=nz, x0=0, x1=800, z0=0, z1=600,
                             materials=[Material(2700.0, 3000.0, 1732.0), Material(1020.0, 1500.0, 0.0)],
                             element_material=em.ravel(), absorb=(True, True, False, True), dt=2.5e-4,
                             nstep=NSTEP, sources=[ForceSource(x=400.0, z=250.0, f0=12.0, factor=1e10)],
                             stations=[Station(x=100.0 + 100.0 * k, z=500.0) for k in range(6)],
                             seismogram_types=("displacement",), save_boundary_values=True)


def reference_mapping(sim):
    info, v = sim.info(), sim.problem_view()
    n, nspec = info.ngll, info.nspec
    med = np.ctypeslib.as_array(v.medium, shape=(nspec,))
    bnd = np.ctypeslib.as_array(v.bnd, shape=(nspec * n * n,)).reshape(nspec, n * n)
    stacey = (bnd & 1).any(axis=1) & ~((bnd & 2).any(axis=1))
    mapping = np.full(nspec, -1)
    for m in (0, 3):
        sel = np.nonzero(stacey & (med == m))[0]
        mapping[sel] = np.arange(len(sel))
    return mapping, med


def test_stacey_store_layout_and_values(tmp_path):
    from oracle import bridge
    sim = Simulation.structured(coupled_problem())
    sim.run_forward()
    lib = sim._lib
    assert lib.sfb_write_wavefield(sim.handle, 0, str(tmp_path).encode()) == 0
    info = sim.info()
    n = info.ngll
    step = os.path.join(str(tmp_path), "ForwardWavefield", "Step%06d" % NSTEP)
    st = os.path.join(step, "Boundary", "Stacey")
    dims, mp = read_ds(st, "IndexMapping")
    mapping, med = reference_mapping(sim)
    assert dims == [info.nspec] and np.array_equal(mp.astype(int), mapping)
    # composite corners exist in this mesh and are left out
    bnd = np.ctypeslib.as_array(sim.problem_view().bnd, shape=(info.nspec * n * n,)).reshape(info.nspec, -1)
    assert ((bnd & 1).any(axis=1) & (bnd & 2).any(axis=1)).sum() > 0
    o32 = bridge.forward(sim, 32, threads=8, want_stacey=True)["stacey_store"]
    o64 = bridge.forward(sim, 64, threads=8, want_stacey=True, exact=True)["stacey_store"]
    for m, name, nc in ((0, "ElasticAcceleration", 2), (3, "AcousticAcceleration", 1)):
        ne = int((mapping[med == m] >= 0).sum())
        dims, vals = read_ds(st, name)
        assert dims == [ne, n, n, NSTEP, nc]
        arr = vals.reshape((nc, NSTEP, n, n, ne)).transpose(4, 3, 2, 1, 0)  # column-major (e, iz, ix, t, c)
        els = np.nonzero((mapping >= 0) & (med == m))[0]
        r32 = o32[:, els][..., :nc].transpose(1, 2, 3, 0, 4)
        r64 = o64[:, els][..., :nc].transpose(1, 2, 3, 0, 4)
        e32, e64, eref = rel_l2(arr, r32), rel_l2(arr, r64), rel_l2(r32, r64)
        print("%s: vs FP32 oracle store %.2e, vs FP64 %.2e (FP32 oracle vs FP64 %.2e)" % (name, e32, e64, eref))
        assert np.abs(r64).max() > 0
        assert e32 <= 1e-5 or e64 <= 1e-5 + 2.0 * eref
    dims, _ = read_ds(st, "PoroelasticAcceleration")
    assert dims == [0, n, n, NSTEP, 4]
    for extra in ("poroelastic", "elastic_psv_t"):
        assert os.path.isdir(os.path.join(step, extra))
        assert os.path.isdir(os.path.join(str(tmp_path), "ForwardWavefield", "Coordinates", extra))


def test_file_round_trip_gives_the_same_kernels(tmp_path):
    p = coupled_problem()
    rng = np.random.default_rng(2)
    stf = (1e-3 * rng.standard_normal((NSTEP, len(p.stations), 2))).astype(np.float32)
    a = Simulation.structured(p)
    a.set_deterministic(True)
    a.run_forward()
    assert a._lib.sfb_write_wavefield(a.handle, 0, str(tmp_path).encode()) == 0
    a.set_adjoint_sources(stf)
    a.run_combined()
    b = Simulation.structured(p)
    b.set_deterministic(True)
    assert b._lib.sfb_read_wavefield(b.handle, 0, str(tmp_path).encode()) == 0, b._lib.sfb_last_error(b.handle)
    b.set_adjoint_sources(stf)
    b.run_combined()
    for q in (0, 1, 2):
        assert np.abs(a.kernels(q)).max() > 0
        assert np.array_equal(a.kernels(q), b.kernels(q)), q
    assert np.array_equal(a.seismograms(wavefield=2), b.seismograms(wavefield=2))


@pytest.mark.parametrize("include_last", [True, False])
def test_time_interval_snapshots(tmp_path, monkeypatch, include_last):
    import workflow_util as WU
    monkeypatch.setenv("SFB_DETERMINISTIC", "1")
    root = str(tmp_path)
    WU.write_mesh_and_stations(root)
    src = os.path.join(root, "sources.yaml")
    with open(src, "w") as f:
        f.write("number-of-sources: 1\nsources:\n" + WU.force_entry())
    mode = """      forward:
        writer:
          wavefield:
            format: ascii
            directory: %s
            time_interval: 100
            include_last_step: %s""" % (root, "true" if include_last else "false")
    cfg = os.path.join(root, "config.yaml")
    with open(cfg, "w") as f:
        f.write(WU.config(root, NSTEP, 5e-4, mode, src))
    run(cfg)
    fw = os.path.join(root, "ForwardWavefield")
    steps = sorted(d for d in os.listdir(fw) if d.startswith("Step"))
    want = ["Step000100", "Step000200"] + (["Step%06d" % NSTEP] if include_last else [])
    assert steps == want
    assert os.path.isdir(os.path.join(fw, "Coordinates", "elastic_psv"))
    # the snapshot of step 100 is the state of a run stopped there
    sim = Simulation.from_yaml(cfg)
    sim.run_forward(100)
    for which, ds in enumerate(("Displacement", "Velocity", "Acceleration")):
        _, vals = read_ds(os.path.join(fw, "Step000100", "elastic_psv"), ds)
        g = sim.field(0, which)
        assert np.array_equal(vals.astype(np.float32), g.reshape(-1)), ds
