"""Batched adjoint 3D elastic at the stated size: 96 x 96 x 48 hexahedra
over 48 x 48 x 24 km, NGLL 5, 1D depth gradient (vp = 3000 + 0.04 depth,
vs = vp / 1.73, rho = 310 vp^0.25) with a seeded +-3 % random-field
perturbation (2 km correlation), 16 random double-couple shots (Ricker
2 Hz), 1000 surface receivers, dt 2e-3 s, 5000 steps; the misfit against
data from a model with a -5 % vp / vs Gaussian anomaly; forward and the
combined adjoint + backward run of all 16 shots in one batched context.

The Stacey tractions of 5000 steps (16 shots x 445 k boundary points)
do not fit in device memory beside the six wavefields, so the context
segments the run (checkpoints, recomputed segments).  The FP64-oracle
error is measured on a slice of the same problem that the oracle finishes
in minutes (1/4 of the elements per axis, 600 steps, one shot's adjoint
sources).
"""
import os
import time

import numpy as np
import pytest

from specfempp_b200.hex3d import (Simulation3D, config5_problem, gradients_from_kernels, local_coordinates,
                                  misfit_and_residuals)

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def anomaly(p, amp=-0.05, sigma=4000.0):
    x, y, z = local_coordinates(p.nx, p.ny, p.nz, p.x0, p.x1, p.y0, p.y1, p.z0, p.z1)
    c = (0.5 * (p.x0 + p.x1), 0.5 * (p.y0 + p.y1), p.z1 - 8000.0 * (p.z1 - p.z0) / 24000.0)
    g = np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * sigma ** 2))
    return (1.0 + amp * g).astype(np.float32)


def test_config5_full_size_forward_and_gradient():
    t_setup = time.perf_counter()
    obs_p = config5_problem(save_boundary_values=False)
    a = anomaly(obs_p)
    obs_p.vp = obs_p.vp * a
    obs_p.vs = obs_p.vs * a
    obs_sim = Simulation3D(obs_p)
    obs_sim.run_forward()
    obs = [obs_sim.seismograms(shot=s) for s in range(16)]
    obs_sim.close()
    del obs_sim
    p = config5_problem()
    sim = Simulation3D(p)
    try:
        _full_size_run(sim, p, obs, t_setup)
    finally:
        sim.close()      # 181 GB of device memory, whatever the outcome


def _full_size_run(sim, p, obs, t_setup):
    i = sim.info()
    print("config 5: nspec %d nglob %d shots %d steps %d receivers %d boundary points %d" % (
        i.nspec, i.nglob, i.nshots, i.nstep, i.nreceivers, i.nboundary_points))
    print("segments %d x %d steps, checkpoints on %s, device %.1f GB, host %.1f GB, setup %.1f s" % (
        i.nsegments, i.segment_steps, "host" if i.checkpoints_on_host else "device", i.device_bytes / 1e9,
        i.host_bytes / 1e9, time.perf_counter() - t_setup))
    assert i.nspec == 96 * 96 * 48 and i.nshots == 16 and i.nreceivers == 1000 and i.nstep == 5000
    t0 = time.perf_counter()
    sim.run_forward()
    t_fwd = time.perf_counter() - t0
    chi, res = misfit_and_residuals(sim, obs)
    for s in range(16):
        sim.set_adjoint_sources(res[s].astype(np.float32), shot=s)
    t0 = time.perf_counter()
    sim.run_combined()
    t_comb = time.perf_counter() - t0
    pts = i.nglob * i.nshots * i.nstep
    print("forward %.1f s (%.2f ms/step, %.3g point-updates/s); combined %.1f s (%.2f ms/step); "
          "gradient per shot %.2f s; misfit %.6e" % (t_fwd, 1e3 * t_fwd / i.nstep, pts / t_fwd, t_comb,
                                                      1e3 * t_comb / i.nstep, (t_fwd + t_comb) / 16, chi))
    k = [sim.kernels(q) for q in range(3)]
    for q in range(3):
        assert np.isfinite(k[q]).all() and np.abs(k[q]).max() > 0
    g_rho, g_vp, g_vs = gradients_from_kernels(p, *k)
    # the vp gradient is largest where the anomaly is (and the data
    # sensitivity), not at the sources or the boundary
    x, y, z = local_coordinates(p.nx, p.ny, p.nz, p.x0, p.x1, p.y0, p.y1, p.z0, p.z1)
    w = np.abs(g_vp)
    inside = (np.abs(x - 24000) < 12000) & (np.abs(y - 24000) < 12000)
    print("|g_vp| mass inside the central half: %.2f" % (w[inside].sum() / w.sum()))
    # the backward reconstruction retraces the forward run: the backward
    # seismograms (loop order) are the forward ones reversed
    e = rel_l2(sim.seismograms(shot=0, wavefield=2)[::-1], sim.seismograms(shot=0))
    print("backward vs forward seismograms, shot 0: %.2e" % e)
    assert e < 1e-2
    # one step of each kernel on the device
    for what, name in ((0, "stiffness"), (1, "newmark"), (2, "frechet")):
        print("%s: %.3f ms per launch" % (name, sim.time_kernel(what, 5)))


def test_config5_slice_fp64_oracle_error():
    """The same model, element size, dt, shots and receivers on a quarter of
    the elements per axis, 600 steps: GPU seismograms of shots 0 and 15 and
    the kernels of shot 0's adjoint sources vs the FP64 oracle."""
    from oracle import bridge3d
    threads = max(1, min(64, os.cpu_count() or 1))
    p = config5_problem(scale=0.25, nstep=600, nrec=100)
    sim = Simulation3D(p)
    sim.run_forward()
    o = {s: bridge3d.forward(p, s, 64, threads=threads) for s in (0, 15)}
    for s in (0, 15):
        e = rel_l2(sim.seismograms(shot=s), o[s]["seismograms"])
        print("shot %d seismograms: e(gpu, fp64 oracle) %.2e" % (s, e))
        assert e < 1e-4
    rng = np.random.default_rng(0)
    stf = (1e-9 * rng.standard_normal((p.nstep, 100, 3))).astype(np.float32)
    for s in range(16):
        sim.set_adjoint_sources(stf if s == 0 else np.zeros_like(stf), shot=s)
    sim.run_combined()
    k64 = bridge3d.combined(p, o[0], stf.astype(np.float64), 0, 64, threads=threads)["kernels"]
    k64 = k64.reshape(p.nspec, 5, 5, 5, 3)
    for q, name in enumerate(("rho", "mu", "kappa")):
        e = rel_l2(sim.kernels(q), k64[..., q])
        print("kernel %s: e(gpu, fp64 oracle) %.2e" % (name, e))
        assert e < 1e-3
