"""3D elastic path on the GPU (include/specfem_b200_3d.h) against the 3D
oracle (oracle/oracle3d.cpp, which builds its own mesh and arrays from the
same description) and the analytic full-space solution:

  * forward seismograms and final fields of every shot of a batched run
    (S = 3, 16, 20: the scalar and vector Newmark paths, one and two shot
    groups per element) vs the FP64 and FP32 oracles, relative L2 <= 1e-5
    (or within twice the FP32 oracle's own distance from FP64);
  * the combined run: backward seismograms and the rho / mu / kappa kernels
    summed over the shots vs the oracles;
  * segmented runs (checkpoints in device or pinned host memory,
    recomputed segments) give the kernels of the single-segment run;
  * a homogeneous medium reproduces the analytic moment-tensor solution;
  * the misfit gradient (WaveformMisfit3D) matches central finite
    differences of the FP64 oracle's misfit.
"""
import numpy as np
import pytest
import torch

from specfempp_b200.hex3d import (HexProblem, MomentTensorSource, Simulation3D, WaveformMisfit3D,
                                  depth_gradient_model, gradients_from_kernels, local_coordinates)

pytestmark = pytest.mark.gpu

BOUNDS = (0.0, 2000.0, 0.0, 2000.0, 0.0, 1500.0)
RECS = np.array([[300, 400, 1500], [1500, 1600, 1500], [1000, 1000, 700], [1700, 300, 200], [650, 1350, 1100]],
                np.float64)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make_problem(nshots=3, nstep=300, absorb=(True,) * 5 + (False,), model=None, **kw):
    nx, ny, nz = 4, 4, 3
    rho, vp, vs = model or depth_gradient_model(nx, ny, nz, BOUNDS, perturbation=0.03, corr_length=500.0, seed=1,
                                                grid=100.0)
    rng = np.random.default_rng(7)
    srcs = []
    for s in range(nshots):
        m = rng.standard_normal(6) * 1e15
        srcs.append(MomentTensorSource(x=rng.uniform(500, 1500), y=rng.uniform(500, 1500), z=rng.uniform(400, 1100),
                                       mxx=m[0], myy=m[1], mzz=m[2], mxy=m[3], mxz=m[4], myz=m[5],
                                       f0=rng.uniform(6, 9), shot=s))
    # shot 0 has a second source
    srcs.append(MomentTensorSource(x=1300, y=700, z=900, mxz=2e15, f0=7.0, tshift=0.01, shot=0))
    return HexProblem(nx=nx, ny=ny, nz=nz, x0=BOUNDS[0], x1=BOUNDS[1], y0=BOUNDS[2], y1=BOUNDS[3], z0=BOUNDS[4],
                      z1=BOUNDS[5], rho=rho, vp=vp, vs=vs, dt=2e-3, nstep=nstep, nshots=nshots, sources=srcs,
                      receivers=RECS, absorb=absorb, **kw)


def check(name, gpu, o32, o64, bar=1e-5):
    e64, e32, eref = rel_l2(gpu, o64), rel_l2(gpu, o32), rel_l2(o32, o64)
    print("%s: e(gpu,fp64) %.2e  e(gpu,fp32) %.2e  e(fp32,fp64) %.2e" % (name, e64, e32, eref))
    assert np.abs(o64).max() > 0
    assert e64 <= bar or e64 <= 2.0 * eref + 1e-6, name


@pytest.mark.parametrize("nshots", [3, 16, 20])
def test_forward_matches_oracle(nshots):
    from oracle import bridge3d
    p = make_problem(nshots=nshots)
    sim = Simulation3D(p)
    sim.run_forward()
    shots = sorted({0, 1, nshots - 1})
    for s in shots:
        o64 = bridge3d.forward(p, s, 64, want_store=False)
        o32 = bridge3d.forward(p, s, 32, want_store=False)
        check("seismograms shot %d/%d" % (s, nshots), sim.seismograms(shot=s), o32["seismograms"],
              o64["seismograms"])
        for which in range(3):
            check("field %d shot %d" % (which, s), sim.field(0, which, s), o32["final"][which], o64["final"][which])


def combined_case(nshots, **kw):
    from oracle import bridge3d
    p = make_problem(nshots=nshots, save_boundary_values=True, **kw)
    rng = np.random.default_rng(11)
    stf = [(1e-3 * rng.standard_normal((p.nstep, len(RECS), 3))).astype(np.float32) for _ in range(nshots)]
    return p, stf


def oracle_combined(p, stf, precision):
    from oracle import bridge3d
    k = np.zeros((p.nspec * 125, 3))
    bseis = []
    for s in range(p.nshots):
        f = bridge3d.forward(p, s, precision)
        c = bridge3d.combined(p, f, stf[s].astype(np.float64), s, precision, kernels=k)
        bseis.append(c["bseis"])
    return k.reshape(p.nspec, 5, 5, 5, 3), bseis


@pytest.mark.parametrize("nshots", [3, 20])
def test_combined_matches_oracle(nshots):
    p, stf = combined_case(nshots)
    sim = Simulation3D(p)
    sim.run_forward()
    for s in range(nshots):
        sim.set_adjoint_sources(stf[s], shot=s)
    sim.run_combined()
    k64, b64 = oracle_combined(p, stf, 64)
    k32, b32 = oracle_combined(p, stf, 32)
    for s in sorted({0, nshots - 1}):
        check("backward seismograms shot %d" % s, sim.seismograms(shot=s, wavefield=2), b32[s], b64[s])
    for q, name in enumerate(("rho", "mu", "kappa")):
        check("kernel %s" % name, sim.kernels(q), k32[..., q], k64[..., q], bar=1e-4)


@pytest.mark.parametrize("host", [False, True])
def test_segmented_run_gives_the_same_kernels(host):
    p, stf = combined_case(4)
    ref = Simulation3D(p)
    assert ref.info().nsegments == 1
    ref.run_forward()
    for s in range(4):
        ref.set_adjoint_sources(stf[s], shot=s)
    ref.run_combined()
    p.segment_steps = 70
    p.host_checkpoints = host
    seg = Simulation3D(p)
    i = seg.info()
    assert i.nsegments == 5 and i.segment_steps == 70 and i.checkpoints_on_host == int(host)
    seg.run_forward(123)     # stop between checkpoints
    seg.run_forward(p.nstep - 123)
    for s in range(4):
        seg.set_adjoint_sources(stf[s], shot=s)
        assert np.array_equal(seg.seismograms(shot=s), ref.seismograms(shot=s)) or \
            rel_l2(seg.seismograms(shot=s), ref.seismograms(shot=s)) < 1e-6
    seg.run_combined()
    for q in range(3):
        e = rel_l2(seg.kernels(q), ref.kernels(q))
        print("kernel %d: segmented vs single %.2e" % (q, e))
        assert e < 1e-5
    e = rel_l2(seg.seismograms(shot=1, wavefield=2), ref.seismograms(shot=1, wavefield=2))
    assert e < 1e-5
    # the forward fields hold the final state again: a second combined run
    # gives the same kernels
    k0 = seg.kernels(0)
    seg.run_combined()
    assert rel_l2(seg.kernels(0), k0) < 1e-5


def test_homogeneous_medium_matches_the_analytic_solution():
    from analytic3d import moment_tensor_displacement, ricker_stf
    ne, h = 30, 80.0
    L = ne * h
    shape = (ne ** 3, 5, 5, 5)
    rho0, vp0, vs0, f0, dt, nstep = 2700.0, 3000.0, 1732.0, 5.0, 1.2e-3, 520
    src = (L / 2 + 13, L / 2 - 7, L / 2 + 5)
    M = np.array([[1e15, 3e14, -2e14], [3e14, -5e14, 4e14], [-2e14, 4e14, 2e14]])
    recs = np.array([[src[0] + 350, src[1] + 120, src[2] - 80], [src[0] - 200, src[1] - 300, src[2] + 150],
                     [src[0] + 60, src[1] + 80, src[2] + 420], [src[0] + 500, src[1] - 100, src[2]]])
    p = HexProblem(nx=ne, ny=ne, nz=ne, x0=0, x1=L, y0=0, y1=L, z0=0, z1=L,
                   rho=np.full(shape, rho0, np.float32), vp=np.full(shape, vp0, np.float32),
                   vs=np.full(shape, vs0, np.float32), dt=dt, nstep=nstep,
                   sources=[MomentTensorSource(x=src[0], y=src[1], z=src[2], mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2],
                                               mxy=M[0, 1], mxz=M[0, 2], myz=M[1, 2], f0=f0)],
                   receivers=recs, absorb=(True,) * 6)
    sim = Simulation3D(p)
    sim.run_forward()
    t = -1.2 / f0 + np.arange(nstep) * dt
    seis = sim.seismograms()
    for r in range(len(recs)):
        ua = moment_tensor_displacement(recs[r], src, M, t, ricker_stf(f0), rho0, vp0, vs0)
        e = rel_l2(seis[:, r], ua)
        print("receiver %d at %.0f m: analytic %.2e" % (r, np.linalg.norm(recs[r] - np.array(src)), e))
        assert e < 1e-2


def test_misfit_gradient_matches_finite_differences():
    """d chi / d (rho, vp, vs) along smooth directions: the GPU adjoint
    gradient vs central differences of the FP64 oracle's misfit (free
    faces, where the kernels are the whole derivative)."""
    from oracle import bridge3d
    nx, ny, nz = 4, 4, 3
    rho, vp, vs = depth_gradient_model(nx, ny, nz, BOUNDS, perturbation=0.03, corr_length=500.0, seed=1, grid=100.0)
    free = (False,) * 6
    p = make_problem(nshots=2, absorb=free, model=(rho, vp, vs), save_boundary_values=True)
    obs_p = make_problem(nshots=2, absorb=free, model=(rho, vp * np.float32(1.02), vs * np.float32(0.99)))
    obs = [bridge3d.forward(obs_p, s, 64, want_store=False)["seismograms"] for s in range(2)]
    sim = Simulation3D(p)
    t = [torch.tensor(np.asarray(a, np.float64), requires_grad=True) for a in (rho, vp, vs)]
    chi = WaveformMisfit3D.apply(t[0], t[1], t[2], sim, obs)
    chi.backward()
    x, y, z = local_coordinates(nx, ny, nz, *BOUNDS)
    rng = np.random.default_rng(3)

    def chi64(model):
        q = make_problem(nshots=2, absorb=free, model=model)
        c = 0.0
        for s in range(2):
            r = bridge3d.forward(q, s, 64, want_store=False)["seismograms"] - obs[s]
            c += 0.5 * np.sum(r * r) * q.dt
        return c

    for idx, name in enumerate(("rho", "vp", "vs")):
        c = rng.uniform(300, 1700, 3)
        dm = np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - 0.8 * c[2]) ** 2) / (2 * 400.0 ** 2))
        base = [rho, vp, vs]
        plus = list(base)
        minus = list(base)
        plus[idx] = (base[idx] * (1 + 1e-3 * dm)).astype(np.float32)
        minus[idx] = (base[idx] * (1 - 1e-3 * dm)).astype(np.float32)
        fd = chi64(tuple(plus)) - chi64(tuple(minus))
        delta = plus[idx].astype(np.float64) - minus[idx].astype(np.float64)
        an = float(np.sum(t[idx].grad.numpy() * delta))
        e = abs(an - fd) / abs(fd)
        print("%s: FD %.6e adjoint %.6e rel %.2e" % (name, fd, an, e))
        assert e < 1e-3


def test_errors_are_reported():
    from specfempp_b200 import SfbError
    p = make_problem(nshots=2)
    sim = Simulation3D(p)
    with pytest.raises(SfbError):
        sim.run_combined()          # no adjoint state kept
    with pytest.raises(SfbError):
        sim.run_forward(p.nstep + 1)
    with pytest.raises(SfbError):
        sim.seismograms(shot=2)
    bad = make_problem(nshots=2)
    bad.sources[0].shot = 5
    with pytest.raises(SfbError):
        Simulation3D(bad)


def test_kernel_variants_agree():
    """Scalar (one shot per thread) and packed FP32x2 (two shots per thread,
    two or three resident CTAs per SM) stiffness and Frechet kernels give
    the same seismograms and kernels to FP32 rounding."""
    p, stf = combined_case(16)
    out = {}
    for v in (1, 2, 3):
        sim = Simulation3D(p)
        sim.set_variant(v)
        assert sim.variant() == v
        sim.run_forward()
        for s in range(16):
            sim.set_adjoint_sources(stf[s], shot=s)
        sim.run_combined()
        out[v] = ([sim.seismograms(shot=s) for s in (0, 7, 15)], [sim.kernels(q) for q in range(3)])
        sim.close()
    for v in (2, 3):
        for a, b in zip(out[v][0], out[1][0]):
            assert rel_l2(a, b) < 1e-5
        for q in range(3):
            e = rel_l2(out[v][1][q], out[1][1][q])
            print("variant %d vs scalar, kernel %d: %.2e" % (v, q, e))
            assert e < 1e-5
    odd = Simulation3D(make_problem(nshots=3))
    odd.set_variant(2)
    assert odd.variant() == 1      # odd shot counts keep the scalar kernels


def test_sharded_misfit_3d_matches_the_oracle():
    """The 3D per-shard GPU compute that ShardedMisfit runs on each rank
    (gpu_shard_compute3d: batched context, forward, combined run, gradient)
    against the FP64 oracle's misfit and gradient of the same shots."""
    from test_distributed import oracle_shard_compute3d, setup_case3d
    from specfempp_b200.distributed import ShardedMisfit, gpu_shard_compute3d
    prob, model, obs = setup_case3d()
    chi, grads = ShardedMisfit(prob, obs, compute=gpu_shard_compute3d)(model)
    chi64, grads64 = oracle_shard_compute3d(prob, model, obs)
    chi32, _ = oracle_shard_compute3d(prob, model, obs, precision=32)
    # the misfit of a small perturbation is a difference of nearly equal
    # traces, so FP32 rounding is amplified: the suite's rule applies (1e-5,
    # or within twice the FP32 oracle's own distance from FP64)
    e, eref = abs(chi - chi64) / chi64, abs(chi32 - chi64) / chi64
    print("3D sharded misfit: GPU vs FP64 oracle %.2e (FP32 oracle vs FP64 %.2e)" % (e, eref))
    assert e <= 1e-5 or e <= 2.0 * eref + 1e-6
    for k, (g, g64) in enumerate(zip(grads, grads64)):
        e = rel_l2(g, g64)
        print("3D sharded gradient %d: GPU vs FP64 oracle %.2e" % (k, e))
        assert e < 1e-3


def test_points_outside_the_mesh_are_rejected():
    from specfempp_b200 import SfbError
    p = make_problem(nshots=2)
    p.receivers = np.array([[300.0, 400.0, 1500.0], [2500.0, 400.0, 700.0]])
    with pytest.raises(SfbError) as e:
        Simulation3D(p)
    assert e.value.code == -1 and "outside the mesh" in str(e.value)
    q = make_problem(nshots=2)
    q.sources[0].z = -10.0
    with pytest.raises(SfbError):
        Simulation3D(q)


@pytest.mark.parametrize("nshots", [3, 20])
def test_deterministic_runs_are_bit_identical(nshots):
    """Deterministic mode (element colours, fixed-order sums): two runs of
    the forward and combined loop give the same bits, and keep parity with
    the oracle (S = 3: scalar kernels; S = 20: packed, two shot groups)."""
    p, stf = combined_case(nshots, deterministic=True)
    runs = []
    for _ in range(2):
        sim = Simulation3D(p)
        sim.run_forward()
        for s in range(nshots):
            sim.set_adjoint_sources(stf[s], shot=s)
        sim.run_combined()
        runs.append(([sim.seismograms(shot=s) for s in (0, nshots - 1)],
                     [sim.field(0, w, nshots - 1) for w in range(3)],
                     [sim.kernels(q) for q in range(3)],
                     sim.seismograms(shot=0, wavefield=2)))
        sim.close()
    for a, b in zip(runs[0][0] + runs[0][1] + runs[0][2] + [runs[0][3]],
                    runs[1][0] + runs[1][1] + runs[1][2] + [runs[1][3]]):
        assert np.array_equal(a, b)
    k64, _ = oracle_combined(p, stf, 64)
    k32, _ = oracle_combined(p, stf, 32)
    from oracle import bridge3d
    o64 = bridge3d.forward(p, 0, 64, want_store=False)["seismograms"]
    o32 = bridge3d.forward(p, 0, 32, want_store=False)["seismograms"]
    check("deterministic seismograms shot 0", runs[0][0][0], o32, o64)
    for q, name in enumerate(("rho", "mu", "kappa")):
        check("deterministic kernel %s" % name, runs[0][2][q], k32[..., q], k64[..., q], bar=1e-4)
