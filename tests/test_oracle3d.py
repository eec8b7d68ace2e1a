"""The 3D oracle (oracle/oracle3d.cpp) pinned without a GPU.

The reference has no 3D solver, so there are no reference fixtures for
this path; the oracle is pinned instead by
  * the analytic displacement of a moment-tensor point source in a
    homogeneous full space (Stokes' solution, tests/analytic3d.py): the
    discretisation error of a 20^3-element mesh is about 1 %;
  * its adjoint: the rho / mu / kappa kernels of the combined run give the
    derivative of the FP64 waveform misfit along smooth model directions
    (central finite differences) with free faces;
  * its backward run: with the forward run's Stacey tractions replayed, the
    reconstructed wavefield retraces the forward seismograms;
  * its FP32 build agreeing with the FP64 build at FP32 rounding level.
"""
import os

import numpy as np
import pytest

from specfempp_b200.hex3d import (HexProblem, MomentTensorSource, depth_gradient_model, gradients_from_kernels,
                                  local_coordinates)

THREADS = max(1, min(16, os.cpu_count() or 1))
BOUNDS = (0.0, 2000.0, 0.0, 2000.0, 0.0, 1500.0)
RECS = np.array([[300, 400, 1500], [1500, 1600, 1500], [1000, 1000, 700], [1700, 300, 200]], np.float64)


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def small_problem(model=None, absorb=(True,) * 5 + (False,), nstep=300, save=True):
    nx, ny, nz = 4, 4, 3
    rho, vp, vs = model or depth_gradient_model(nx, ny, nz, BOUNDS, perturbation=0.03, corr_length=500.0, seed=1,
                                                grid=100.0)
    return HexProblem(nx=nx, ny=ny, nz=nz, x0=0, x1=2000, y0=0, y1=2000, z0=0, z1=1500, rho=rho, vp=vp, vs=vs,
                      dt=2e-3, nstep=nstep, nshots=1,
                      sources=[MomentTensorSource(x=900, y=1100, z=800, mxx=1e15, myy=-1e15, mxy=3e14, f0=8.0)],
                      receivers=RECS, absorb=absorb, save_boundary_values=save)


def test_oracle_matches_the_analytic_full_space_solution():
    from analytic3d import moment_tensor_displacement, ricker_stf
    from oracle import bridge3d
    ne, h = 20, 100.0
    L = ne * h
    shape = (ne ** 3, 5, 5, 5)
    rho0, vp0, vs0, f0, dt, nstep = 2700.0, 3000.0, 1732.0, 5.0, 1.5e-3, 400
    src = (L / 2 + 13, L / 2 - 7, L / 2 + 5)
    M = np.array([[1e15, 3e14, -2e14], [3e14, -5e14, 4e14], [-2e14, 4e14, 2e14]])
    recs = np.array([[src[0] + 350, src[1] + 120, src[2] - 80], [src[0] - 200, src[1] - 300, src[2] + 150],
                     [src[0] + 60, src[1] + 80, src[2] + 420]])
    p = HexProblem(nx=ne, ny=ne, nz=ne, x0=0, x1=L, y0=0, y1=L, z0=0, z1=L,
                   rho=np.full(shape, rho0, np.float32), vp=np.full(shape, vp0, np.float32),
                   vs=np.full(shape, vs0, np.float32), dt=dt, nstep=nstep,
                   sources=[MomentTensorSource(x=src[0], y=src[1], z=src[2], mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2],
                                               mxy=M[0, 1], mxz=M[0, 2], myz=M[1, 2], f0=f0)],
                   receivers=recs, absorb=(True,) * 6)
    seis = bridge3d.forward(p, 0, 64, threads=THREADS)["seismograms"]
    t = -1.2 / f0 + np.arange(nstep) * dt
    for r in range(len(recs)):
        ua = moment_tensor_displacement(recs[r], src, M, t, ricker_stf(f0), rho0, vp0, vs0)
        e = rel_l2(seis[:, r], ua)
        print("receiver %d: oracle vs analytic %.2e" % (r, e))
        assert e < 2e-2


def test_fp32_oracle_agrees_with_fp64():
    from oracle import bridge3d
    p = small_problem()
    a = bridge3d.forward(p, 0, 64, threads=THREADS)
    b = bridge3d.forward(p, 0, 32, threads=THREADS)
    e = rel_l2(b["seismograms"], a["seismograms"])
    print("FP32 oracle vs FP64: %.2e" % e)
    assert 0 < e < 1e-5


def test_backward_replay_retraces_the_forward_run():
    from oracle import bridge3d
    p = small_problem()
    f = bridge3d.forward(p, 0, 64, threads=THREADS)
    c = bridge3d.combined(p, f, np.zeros((p.nstep, len(RECS), 3)), 0, 64, threads=THREADS)
    back = c["bseis"][::-1]          # loop order -> time order
    e = rel_l2(back, f["seismograms"])
    print("backward vs forward seismograms: %.2e" % e)
    assert e < 1e-6


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_oracle_kernels_give_the_misfit_derivative(idx):
    from oracle import bridge3d
    free = (False,) * 6
    nx, ny, nz = 4, 4, 3
    rho, vp, vs = depth_gradient_model(nx, ny, nz, BOUNDS, perturbation=0.03, corr_length=500.0, seed=1, grid=100.0)
    obs = bridge3d.forward(small_problem((rho, vp * np.float32(1.02), vs * np.float32(0.99)), free, save=False), 0,
                           64, threads=THREADS)["seismograms"]

    def chi(model):
        s = bridge3d.forward(small_problem(model, free, save=False), 0, 64, threads=THREADS)["seismograms"]
        r = s - obs
        return 0.5 * np.sum(r * r) * 2e-3, r

    p = small_problem((rho, vp, vs), free)
    _, res = chi((rho, vp, vs))
    f = bridge3d.forward(p, 0, 64, threads=THREADS)
    k = bridge3d.combined(p, f, res, 0, 64, threads=THREADS)["kernels"].reshape(-1, 5, 5, 5, 3)
    g = gradients_from_kernels(p, k[..., 0], k[..., 1], k[..., 2])
    x, y, z = local_coordinates(nx, ny, nz, *BOUNDS)
    c = np.random.default_rng(3 + idx).uniform(300, 1700, 3)
    dm = np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - 0.8 * c[2]) ** 2) / (2 * 400.0 ** 2))
    base = [rho, vp, vs]
    plus, minus = list(base), list(base)
    plus[idx] = (base[idx] * (1 + 1e-3 * dm)).astype(np.float32)
    minus[idx] = (base[idx] * (1 - 1e-3 * dm)).astype(np.float32)
    fd = chi(tuple(plus))[0] - chi(tuple(minus))[0]
    an = float(np.sum(g[idx] * (plus[idx].astype(np.float64) - minus[idx].astype(np.float64))))
    e = abs(an - fd) / abs(fd)
    print("parameter %d: FD %.6e adjoint %.6e rel %.2e" % (idx, fd, an, e))
    assert e < 1e-4
