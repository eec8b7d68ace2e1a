"""Shot sharding over two gloo ranks on CPU: the all-reduced misfit and
gradient equal the single-process result over all shots.  The per-shard
compute is the oracle (FP64 forward + combined loop), so no GPU is needed;
the GPU path plugs `gpu_shard_compute` into the same host logic."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

NSTEP = 120
NSHOTS = 3


def oracle_shard_compute(problem, model, observed):
    from oracle import bridge
    from specfempp_b200 import Simulation
    from adjoint_util import kernel_gradient
    sim = Simulation.structured(problem)
    info = sim.info()
    chi = 0.0
    grads = [np.zeros_like(np.asarray(a, dtype=np.float64)) for a in model]
    for s in range(info.nshots):
        # one thread: the oracle's OpenMP scatter would add in varying order
        fwd = bridge.forward(sim, 64, shot=s, threads=1, want_fields=True, want_stacey=True)
        res = fwd["seismograms"][:, 0].astype(np.float64) - observed[s]
        chi += 0.5 * float(np.sum(res * res)) * info.dt
        K = bridge.combined(sim, res.astype(np.float32), fwd, precision=64, shot=s, threads=1)
        for g, gg in zip(grads, kernel_gradient(sim, K, model)):
            g += gg
    return chi, grads


ABSORB = (True, True, False, True)


def setup_case(obs_file=None):
    from adjoint_util import anomaly, base_model, observed, problem
    p, model, XZ = base_model(nshots=NSHOTS, nstep=NSTEP)
    if obs_file is None:
        obs = observed(anomaly(model, XZ, p), NSTEP, ABSORB, nshots=NSHOTS)
    else:
        obs = np.load(obs_file)
    return problem(model, NSTEP, ABSORB, NSHOTS), model, obs


def _worker(rank, world, port, outdir, obs_file):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from specfempp_b200.distributed import ShardedMisfit
    prob, model, obs = setup_case(obs_file)
    sm = ShardedMisfit(prob, obs, compute=oracle_shard_compute)
    chi, grads = sm(model)
    np.savez(os.path.join(outdir, "rank%d.npz" % rank), chi=chi, g0=grads[0], g1=grads[1], g2=grads[2],
             shots=np.array(sm.shots))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_assignment_round_robin():
    from specfempp_b200.distributed import shard_shots
    assert shard_shots(5, 2, 0) == [0, 2, 4]
    assert shard_shots(5, 2, 1) == [1, 3]
    assert sorted(shard_shots(7, 3, 0) + shard_shots(7, 3, 1) + shard_shots(7, 3, 2)) == list(range(7))


def test_two_rank_gloo_matches_single_process(tmp_path, native_lib, oracle_lib):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    prob, model, obs = setup_case()
    obs_file = str(tmp_path / "observed.npy")
    np.save(obs_file, obs)
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), obs_file)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    assert list(r0["shots"]) == [0, 2] and list(r1["shots"]) == [1]
    chi, grads = oracle_shard_compute(prob, model, obs)
    for r in (r0, r1):
        assert abs(float(r["chi"]) - chi) <= 1e-12 * abs(chi)
        for k, g in enumerate(grads):
            # only the order of the FP64 shot sums differs
            err = np.linalg.norm(r["g%d" % k] - g) / np.linalg.norm(g)
            print("gradient %d: rel-L2 %.2e" % (k, err))
            assert err <= 1e-12, (k, err)


# ---------------------------------------------------------------------------
# 3D: the same sharding of a HexProblem's shots; the per-shard compute is the
# 3D oracle (FP64 forward + combined run, gradients from its kernels).

NSTEP3 = 150


def oracle_shard_compute3d(problem, model, observed, precision=64):
    from dataclasses import replace
    from oracle import bridge3d
    from specfempp_b200.hex3d import gradients_from_kernels
    rho, vp, vs = (np.asarray(a, dtype=np.float32) for a in model)
    p = replace(problem, rho=rho, vp=vp, vs=vs, save_boundary_values=True)
    chi = 0.0
    k = np.zeros((p.nspec * 125, 3))
    for s in range(p.nshots):
        fwd = bridge3d.forward(p, s, precision, threads=1)
        res = fwd["seismograms"] - observed[s]
        chi += 0.5 * float(np.sum(res * res)) * p.dt
        bridge3d.combined(p, fwd, res, s, precision, threads=1, kernels=k)
    k = k.reshape(p.nspec, 5, 5, 5, 3)
    return chi, list(gradients_from_kernels(p, k[..., 0], k[..., 1], k[..., 2]))


def setup_case3d():
    from specfempp_b200.hex3d import HexProblem, MomentTensorSource, depth_gradient_model
    nx, ny, nz = 3, 3, 2
    bounds = (0.0, 1500.0, 0.0, 1500.0, 0.0, 1000.0)
    rho, vp, vs = depth_gradient_model(nx, ny, nz, bounds, perturbation=0.03, corr_length=400.0, seed=4, grid=100.0)
    srcs = [MomentTensorSource(x=400.0 + 300.0 * s, y=700.0, z=500.0, mxx=1e15, myz=5e14, f0=8.0, shot=s)
            for s in range(NSHOTS)]
    rec = np.array([[200.0, 300.0, 1000.0], [1200.0, 1100.0, 1000.0], [800.0, 400.0, 300.0]])
    p = HexProblem(nx=nx, ny=ny, nz=nz, x0=0, x1=1500, y0=0, y1=1500, z0=0, z1=1000, rho=rho, vp=vp, vs=vs,
                   dt=2e-3, nstep=NSTEP3, nshots=NSHOTS, sources=srcs, receivers=rec)
    from dataclasses import replace
    from oracle import bridge3d
    obs_p = replace(p, vp=vp * np.float32(1.02))
    obs = np.stack([bridge3d.forward(obs_p, s, 64, threads=1, want_store=False)["seismograms"]
                    for s in range(NSHOTS)])
    return p, (rho, vp, vs), obs


def _worker3d(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from specfempp_b200.distributed import ShardedMisfit
    prob, model, obs = setup_case3d()
    sm = ShardedMisfit(prob, obs, compute=oracle_shard_compute3d)
    chi, grads = sm(model)
    np.savez(os.path.join(outdir, "rank%d.npz" % rank), chi=chi, g0=grads[0], g1=grads[1], g2=grads[2],
             shots=np.array(sm.shots))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_matches_single_process_3d(tmp_path, oracle_lib):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker3d, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    assert list(r0["shots"]) == [0, 2] and list(r1["shots"]) == [1]
    prob, model, obs = setup_case3d()
    chi, grads = oracle_shard_compute3d(prob, model, obs)
    assert chi > 0
    for r in (r0, r1):
        assert abs(float(r["chi"]) - chi) <= 1e-12 * abs(chi)
        for k, g in enumerate(grads):
            err = np.linalg.norm(r["g%d" % k] - g) / np.linalg.norm(g)
            print("3D gradient %d: rel-L2 %.2e" % (k, err))
            assert err <= 1e-12, (k, err)
