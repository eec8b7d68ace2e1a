"""Synthetic workloads with the shapes, sizes and value distributions of the
benchmark configurations (seeded; no external data):

  plain_elastic   2D isotropic elastic P-SV, 100 x 80 elements over
                  4000 m x 3000 m, rho 2700, vp 3000, vs 1732, free top,
                  Stacey bottom/left/right, vertical Ricker force (10 Hz) at
                  (2000, 1500), dt 5e-4, 4000 steps, 20 receivers on z = 2900.
  coupled         2D acoustic-elastic, 400 x 300 elements over 20 km x 15 km,
                  top 3 km water (rho 1020, vp 1500), six elastic layers with
                  vp ~ U(2500, 5500) (seed 0), vs = vp / sqrt(3),
                  rho = 310 vp^0.25, Gaussian-smoothed (sigma 500 m) +-5 % vp
                  perturbation per GLL point (seed 1), pressure Ricker 5 Hz in
                  the water, 200 hydrophones, dt 1e-3, 10000 steps.
  batched         800 x 400 elements over 40 km x 20 km, the coupled model's
                  layered + perturbed elastic part without water, S shots of
                  vertical forces at 50 m depth with f0 ~ U(4, 8) Hz (seed 2),
                  400 shared receivers, dt 1e-3, 8000 steps.
  adjoint         200 x 200 elements over 10 km x 10 km, homogeneous
                  (2600, 4000, 2310), 8 shots, 100 receivers, dt 5e-4, 6000 steps.

Every builder takes a `scale` in (0, 1] that shrinks the element counts (and
the domain, keeping element size) for tests; scale = 1 is the full size.
"""
from __future__ import annotations

import math

import numpy as np

from .simulation import ForceSource, Material, Station, StructuredProblem

NGLL = 5


def _gll_points(n=NGLL):
    from numpy.polynomial import legendre as L
    N = n - 1
    c = np.zeros(N + 1)
    c[N] = 1
    inner = np.sort(np.real(L.legroots(L.legder(c))))
    return np.concatenate([[-1.0], inner, [1.0]])


def gll_coordinates(nx, nz, x0, x1, z0, z1, ngll=NGLL):
    """Physical (x, z) of every local GLL point, [nspec, ngll, ngll] each,
    element ispec = iz * nx + ix (the structured mesher's numbering)."""
    xi = _gll_points(ngll)
    dx = (x1 - x0) / nx
    dz = (z1 - z0) / nz
    ex = x0 + dx * np.arange(nx)
    ez = z0 + dz * np.arange(nz)
    X = ex[None, :, None, None] + (xi[None, None, None, :] + 1) * dx / 2  # [1,nx,1,ngll]
    Z = ez[:, None, None, None] + (xi[None, None, :, None] + 1) * dz / 2  # [nz,1,ngll,1]
    X = np.broadcast_to(X, (nz, nx, ngll, ngll)).reshape(nz * nx, ngll, ngll)
    Z = np.broadcast_to(Z, (nz, nx, ngll, ngll)).reshape(nz * nx, ngll, ngll)
    return X, Z


def _smooth_perturbation(nx, nz, x0, x1, z0, z1, sigma, amp, seed, ngll=NGLL):
    """Per-GLL-point white noise on a regular grid of the GLL spacing, smoothed
    with a separable Gaussian (sigma in metres), scaled to max |p| = amp and
    sampled at every local GLL point."""
    rng = np.random.default_rng(seed)
    h = min((x1 - x0) / nx, (z1 - z0) / nz) / (ngll - 1)
    gx = int(round((x1 - x0) / h)) + 1
    gz = int(round((z1 - z0) / h)) + 1
    noise = rng.standard_normal((gz, gx))
    s = sigma / h
    r = int(math.ceil(3 * s))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / s) ** 2)
    k /= k.sum()
    pad = np.pad(noise, ((r, r), (r, r)), mode="reflect")
    tmp = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), 1, pad)
    sm = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), 0, tmp)
    sm *= amp / np.max(np.abs(sm))
    X, Z = gll_coordinates(nx, nz, x0, x1, z0, z1, ngll)
    ix = np.clip(np.rint((X - x0) / h).astype(np.int64), 0, gx - 1)
    iz = np.clip(np.rint((Z - z0) / h).astype(np.int64), 0, gz - 1)
    return sm[iz, ix]


def _layered_model(nx, nz, x0, x1, z0, z1, water_top, nlayers=6, seed_layers=0, seed_pert=1):
    """(rho, vp, vs) per GLL point: water above z = water_top (if any), six
    equal elastic layers below, vp perturbed by a smoothed +-5 % field."""
    rng = np.random.default_rng(seed_layers)
    vp_layers = rng.uniform(2500.0, 5500.0, nlayers)
    X, Z = gll_coordinates(nx, nz, x0, x1, z0, z1)
    zb = z0
    ztop = water_top if water_top is not None else z1
    thick = (ztop - zb) / nlayers
    layer = np.clip(((ztop - Z) / thick).astype(np.int64), 0, nlayers - 1)  # 0 = shallowest
    vp = vp_layers[layer]
    pert = _smooth_perturbation(nx, nz, x0, x1, z0, z1, 500.0, 0.05, seed_pert)
    vp = vp * (1.0 + pert)
    vs = vp / math.sqrt(3.0)
    rho = 310.0 * vp ** 0.25
    return rho.astype(np.float32), vp.astype(np.float32), vs.astype(np.float32), vp_layers


def plain_elastic(scale: float = 1.0, nstep: int = 4000, seismogram_types=("displacement",)):
    nx = max(4, int(round(100 * scale)))
    nz = max(4, int(round(80 * scale)))
    dx, dz = 40.0, 37.5
    Lx, Lz = nx * dx, nz * dz
    src = ForceSource(x=Lx / 2, z=Lz / 2, f0=10.0, factor=1e10, angle=0.0)
    zr = Lz - 100.0
    stations = [Station(x=Lx * (k + 0.5) / 20, z=zr, station="S%04d" % (k + 1)) for k in range(20)]
    return StructuredProblem(nx=nx, nz=nz, x0=0.0, x1=Lx, z0=0.0, z1=Lz,
                             materials=[Material(2700.0, 3000.0, 1732.0)],
                             absorb=(True, True, False, True), dt=5e-4, nstep=nstep,
                             sources=[src], stations=stations, seismogram_types=seismogram_types)


def coupled(scale: float = 1.0, nstep: int = 10000, seismogram_types=("pressure",)):
    nx = max(4, int(round(400 * scale)))
    nz = max(5, int(round(300 * scale)))
    d = 50.0
    Lx, Lz = nx * d, nz * d
    nwater = max(1, int(round(nz * 60 / 300)))
    water_top = Lz - nwater * d
    rho, vp, vs, _ = _layered_model(nx, nz, 0.0, Lx, 0.0, Lz, water_top)
    em = np.zeros((nz, nx), dtype=np.int32)
    em[nz - nwater:, :] = 1
    em = em.reshape(-1)
    ew = em.astype(bool)
    rho.reshape(nz * nx, -1)[ew] = 1020.0
    vp.reshape(nz * nx, -1)[ew] = 1500.0
    vs.reshape(nz * nx, -1)[ew] = 0.0
    mats = [Material(2500.0, 4000.0, 2300.0), Material(1020.0, 1500.0, 0.0)]
    src = ForceSource(x=Lx / 2, z=Lz - 0.5 * nwater * d, f0=5.0, factor=1e10)
    zr = Lz - 0.25 * nwater * d
    stations = [Station(x=Lx * (k + 0.5) / 200, z=zr, station="H%04d" % (k + 1)) for k in range(200)]
    return StructuredProblem(nx=nx, nz=nz, x0=0.0, x1=Lx, z0=0.0, z1=Lz, materials=mats,
                             element_material=em, gll_model=(rho, vp, vs),
                             absorb=(True, True, False, True), dt=1e-3, nstep=nstep,
                             sources=[src], stations=stations, seismogram_types=seismogram_types)


def batched(scale: float = 1.0, nshots: int = 64, nstep: int = 8000,
            seismogram_types=("displacement",)):
    nx = max(4, int(round(800 * scale)))
    nz = max(4, int(round(400 * scale)))
    d = 50.0
    Lx, Lz = nx * d, nz * d
    rho, vp, vs, _ = _layered_model(nx, nz, 0.0, Lx, 0.0, Lz, None)
    rng = np.random.default_rng(2)
    f0 = rng.uniform(4.0, 8.0, nshots)
    srcs = [ForceSource(x=Lx * (s + 0.5) / nshots, z=Lz - 50.0, f0=float(f0[s]), factor=1e10, shot=s)
            for s in range(nshots)]
    stations = [Station(x=Lx * (k + 0.5) / 400, z=Lz - 25.0, station="R%04d" % (k + 1)) for k in range(400)]
    return StructuredProblem(nx=nx, nz=nz, x0=0.0, x1=Lx, z0=0.0, z1=Lz,
                             materials=[Material(2500.0, 4000.0, 2300.0)],
                             gll_model=(rho, vp, vs), absorb=(True, True, False, True), dt=1e-3,
                             nstep=nstep, nshots=nshots, sources=srcs, stations=stations,
                             seismogram_types=seismogram_types)


def adjoint_model(scale: float = 1.0, nshots: int = 8, nstep: int = 6000, anomaly: bool = False):
    nx = max(4, int(round(200 * scale)))
    nz = max(4, int(round(200 * scale)))
    d = 50.0
    Lx, Lz = nx * d, nz * d
    X, Z = gll_coordinates(nx, nz, 0.0, Lx, 0.0, Lz)
    vp = np.full(X.shape, 4000.0)
    vs = np.full(X.shape, 2310.0)
    if anomaly:
        g = np.exp(-((X - Lx / 2) ** 2 + (Z - Lz / 2) ** 2) / (2 * 800.0 ** 2))
        vp *= 1 - 0.1 * g
        vs *= 1 - 0.1 * g
    rho = np.full(X.shape, 2600.0)
    srcs = [ForceSource(x=Lx * (s + 0.5) / nshots, z=Lz - 250.0, f0=10.0, factor=1e10, shot=s)
            for s in range(nshots)]
    stations = [Station(x=Lx * (k + 0.5) / 100, z=250.0, station="R%04d" % (k + 1)) for k in range(100)]
    return StructuredProblem(nx=nx, nz=nz, x0=0.0, x1=Lx, z0=0.0, z1=Lz,
                             materials=[Material(2600.0, 4000.0, 2310.0)],
                             gll_model=(rho.astype(np.float32), vp.astype(np.float32), vs.astype(np.float32)),
                             absorb=(True, True, True, True), dt=5e-4, nstep=nstep, nshots=nshots,
                             sources=srcs, stations=stations, seismogram_types=("displacement",))
