"""3D elastic path on hexahedral spectral elements (``include/specfem_b200_3d.h``).

The reference's 3D program stops after reading its mesh
(src/specfem3d.cpp:49-73); this module drives the 3D extension of its 2D
weak form on the GPU: a structured mesh of axis-aligned hexahedra, NGLL = 5,
isotropic elastic, S shots advanced together (shot index innermost in
device memory), moment-tensor sources, displacement receivers, Stacey
absorbing faces, and the combined adjoint + backward run with Frechet
kernels.  ``WaveformMisfit3D`` turns the kernels into the gradient of an L2
waveform misfit with respect to (rho, vp, vs) per local point.

The compute path is ``_lib/libspecfem_b200.so``; this module is its ctypes
binding and the host-side model and geometry helpers.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _capi
from ._capi import SfbError

NGLL = 5
ABSORB_FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


class sfb3_source(C.Structure):
    _fields_ = [("shot", C.c_int), ("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("mxx", C.c_double), ("myy", C.c_double), ("mzz", C.c_double),
                ("mxy", C.c_double), ("mxz", C.c_double), ("myz", C.c_double),
                ("f0", C.c_double), ("tshift", C.c_double), ("factor", C.c_double)]


class sfb3_desc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
                ("z0", C.c_double), ("z1", C.c_double), ("absorb", C.c_int),
                ("rho", C.POINTER(C.c_float)), ("vp", C.POINTER(C.c_float)), ("vs", C.POINTER(C.c_float)),
                ("dt", C.c_double), ("nstep", C.c_int), ("nshots", C.c_int),
                ("nsources", C.c_int), ("sources", C.POINTER(sfb3_source)),
                ("nreceivers", C.c_int), ("receivers", C.POINTER(C.c_double)),
                ("save_boundary_values", C.c_int), ("segment_steps", C.c_int), ("host_checkpoints", C.c_int),
                ("deterministic", C.c_int)]


class sfb3_info(C.Structure):
    _fields_ = [("nspec", C.c_int), ("nglob", C.c_int), ("nshots", C.c_int), ("nstep", C.c_int),
                ("nreceivers", C.c_int), ("nboundary_points", C.c_int), ("segment_steps", C.c_int),
                ("nsegments", C.c_int), ("checkpoints_on_host", C.c_int), ("dt", C.c_double),
                ("t0", C.c_double), ("device_bytes", C.c_size_t), ("host_bytes", C.c_size_t),
                ("kernel_launches", C.c_ulonglong)]


_ctx = C.c_void_p
_f = C.POINTER(C.c_float)
_d = C.POINTER(C.c_double)
SIGNATURES3 = {
    "sfb3_create": (C.c_int, [C.POINTER(sfb3_desc), C.POINTER(_ctx)]),
    "sfb3_destroy": (None, [_ctx]),
    "sfb3_last_error": (C.c_char_p, [_ctx]),
    "sfb3_get_info": (C.c_int, [_ctx, C.POINTER(sfb3_info)]),
    "sfb3_run_forward": (C.c_int, [_ctx, C.c_int]),
    "sfb3_get_seismograms": (C.c_int, [_ctx, C.c_int, C.c_int, _f, C.c_size_t]),
    "sfb3_set_adjoint_sources": (C.c_int, [_ctx, C.c_int, _f, C.c_size_t]),
    "sfb3_run_combined": (C.c_int, [_ctx]),
    "sfb3_get_kernels": (C.c_int, [_ctx, C.c_int, _d, C.c_size_t]),
    "sfb3_get_field": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_int, _f, C.c_size_t]),
    "sfb3_reset": (C.c_int, [_ctx]),
    "sfb3_time_kernel": (C.c_int, [_ctx, C.c_int, C.c_int, _d]),
    "sfb3_set_variant": (C.c_int, [_ctx, C.c_int]),
    "sfb3_get_variant": (C.c_int, [_ctx]),
}

_lib3 = None


def load3():
    """The product library with the 3D entry points' signatures set."""
    global _lib3
    if _lib3 is None:
        lib = _capi.load(32)
        for name, (res, args) in SIGNATURES3.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib3 = lib
    return _lib3


def _check(code, ctx=None):
    if code != 0:
        msg = load3().sfb3_last_error(ctx)
        raise SfbError(code, msg.decode() if msg else "")


@dataclass
class MomentTensorSource:
    x: float
    y: float
    z: float
    mxx: float = 0.0
    myy: float = 0.0
    mzz: float = 0.0
    mxy: float = 0.0
    mxz: float = 0.0
    myz: float = 0.0
    f0: float = 2.0
    tshift: float = 0.0
    factor: float = 1.0
    shot: int = 0


@dataclass
class HexProblem:
    """A structured hexahedral problem; the model is given per local point
    [nspec][5][5][5] (element (ex, ey, ez) = (ez * ny + ey) * nx + ex, local
    point (k, j, i) along z, y, x)."""
    nx: int
    ny: int
    nz: int
    x0: float
    x1: float
    y0: float
    y1: float
    z0: float
    z1: float
    rho: np.ndarray
    vp: np.ndarray
    vs: np.ndarray
    dt: float
    nstep: int
    nshots: int = 1
    sources: List[MomentTensorSource] = field(default_factory=list)
    receivers: Optional[np.ndarray] = None          # [nrec][3]
    absorb: Sequence[bool] = (True, True, True, True, True, False)
    save_boundary_values: bool = False
    segment_steps: int = 0
    host_checkpoints: bool = False
    deterministic: bool = False

    @property
    def nspec(self):
        return self.nx * self.ny * self.nz

    def to_desc(self):
        shape = (self.nspec, NGLL, NGLL, NGLL)
        keep = {}
        for name in ("rho", "vp", "vs"):
            arr = np.ascontiguousarray(np.asarray(getattr(self, name), dtype=np.float32).reshape(shape))
            keep[name] = arr
        srcs = (sfb3_source * max(1, len(self.sources)))()
        for q, s in enumerate(self.sources):
            srcs[q] = sfb3_source(s.shot, s.x, s.y, s.z, s.mxx, s.myy, s.mzz, s.mxy, s.mxz, s.myz,
                                  s.f0, s.tshift, s.factor)
        rec = np.zeros((0, 3)) if self.receivers is None else np.asarray(self.receivers, np.float64)
        rec = np.ascontiguousarray(rec.reshape(-1, 3))
        keep["rec"] = rec
        keep["srcs"] = srcs
        absorb = sum(1 << f for f, on in enumerate(self.absorb) if on)
        d = sfb3_desc(self.nx, self.ny, self.nz, self.x0, self.x1, self.y0, self.y1, self.z0, self.z1, absorb,
                      keep["rho"].ctypes.data_as(_f), keep["vp"].ctypes.data_as(_f), keep["vs"].ctypes.data_as(_f),
                      self.dt, self.nstep, self.nshots, len(self.sources), srcs, rec.shape[0],
                      rec.ctypes.data_as(_d), int(self.save_boundary_values), int(self.segment_steps),
                      int(self.host_checkpoints), int(self.deterministic))
        return d, keep


def gll_nodes():
    a = math.sqrt(3.0 / 7.0)
    return np.array([-1.0, -a, 0.0, a, 1.0]), np.array([0.1, 49 / 90, 32 / 45, 49 / 90, 0.1])


def local_coordinates(nx, ny, nz, x0, x1, y0, y1, z0, z1):
    """(x, y, z) of every local point, each [nspec][5][5][5]."""
    xi, _ = gll_nodes()
    dx, dy, dz = (x1 - x0) / nx, (y1 - y0) / ny, (z1 - z0) / nz
    ex = np.arange(nx)
    ey = np.arange(ny)
    ez = np.arange(nz)
    X = x0 + (ex[:, None] + (xi[None, :] + 1) / 2) * dx   # [nx][5]
    Y = y0 + (ey[:, None] + (xi[None, :] + 1) / 2) * dy
    Z = z0 + (ez[:, None] + (xi[None, :] + 1) / 2) * dz
    shape = (nz, ny, nx, NGLL, NGLL, NGLL)   # ez, ey, ex, k, j, i
    x = np.broadcast_to(X[None, None, :, None, None, :], shape)
    y = np.broadcast_to(Y[None, :, None, None, :, None], shape)
    z = np.broadcast_to(Z[:, None, None, :, None, None], shape)
    n = nx * ny * nz
    return (x.reshape(n, NGLL, NGLL, NGLL), y.reshape(n, NGLL, NGLL, NGLL), z.reshape(n, NGLL, NGLL, NGLL))


def quadrature_volume(problem: HexProblem):
    """w_i w_j w_k J per local point, [nspec][5][5][5]."""
    _, w = gll_nodes()
    jac = ((problem.x1 - problem.x0) / problem.nx * (problem.y1 - problem.y0) / problem.ny
           * (problem.z1 - problem.z0) / problem.nz / 8.0)
    w3 = w[:, None, None] * w[None, :, None] * w[None, None, :]
    return np.broadcast_to(w3 * jac, (problem.nspec, NGLL, NGLL, NGLL))


def gaussian_random_field(shape, spacing, corr_length, seed):
    """Zero-mean, unit-max-abs field on a regular grid with a Gaussian
    correlation of length `corr_length` (FFT filter of white noise)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n, d=spacing) * 2 * np.pi for n in shape]
    K2 = sum(np.meshgrid(*[kk ** 2 for kk in k], indexing="ij"))
    f = np.real(np.fft.ifftn(np.fft.fftn(noise) * np.exp(-K2 * corr_length ** 2 / 4.0)))
    f -= f.mean()
    return f / np.abs(f).max()


def trilinear(field3, spacing, origin, x, y, z):
    """Trilinear interpolation of a [nz][ny][nx] grid field at points."""
    out = np.empty(x.shape, np.float64)
    fx = (x - origin[0]) / spacing
    fy = (y - origin[1]) / spacing
    fz = (z - origin[2]) / spacing
    nz, ny, nx = field3.shape
    i0 = np.clip(np.floor(fx).astype(np.int64), 0, nx - 2)
    j0 = np.clip(np.floor(fy).astype(np.int64), 0, ny - 2)
    k0 = np.clip(np.floor(fz).astype(np.int64), 0, nz - 2)
    tx, ty, tz = fx - i0, fy - j0, fz - k0
    out[...] = 0.0
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                wgt = ((tx if di else 1 - tx) * (ty if dj else 1 - ty) * (tz if dk else 1 - tz))
                out += wgt * field3[k0 + dk, j0 + dj, i0 + di]
    return out


def depth_gradient_model(nx, ny, nz, bounds, perturbation=0.03, corr_length=2000.0, seed=0, grid=250.0):
    """vp = 3000 + 0.04 depth, vs = vp / 1.73, rho = 310 vp^0.25, times a
    seeded Gaussian-random-field perturbation of +-`perturbation` in vp and
    vs (correlation length `corr_length`), per local point."""
    x0, x1, y0, y1, z0, z1 = bounds
    x, y, z = local_coordinates(nx, ny, nz, *bounds)
    depth = z1 - z
    vp = 3000.0 + 0.04 * depth
    if perturbation:
        shape = (int(math.ceil((z1 - z0) / grid)) + 2, int(math.ceil((y1 - y0) / grid)) + 2,
                 int(math.ceil((x1 - x0) / grid)) + 2)
        grf = gaussian_random_field(shape, grid, corr_length, seed)
        vp = vp * (1.0 + perturbation * trilinear(grf, grid, (x0, y0, z0), x, y, z))
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    return rho.astype(np.float32), vp.astype(np.float32), vs.astype(np.float32)


def random_double_couple(rng, m0=1e15):
    """Moment tensor M0 (n d^T + d n^T) of a double couple with a random
    fault normal n and slip direction d perpendicular to it."""
    n = rng.standard_normal(3)
    n /= np.linalg.norm(n)
    t = rng.standard_normal(3)
    d = t - n * np.dot(n, t)
    d /= np.linalg.norm(d)
    M = m0 * (np.outer(n, d) + np.outer(d, n))
    return dict(mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2], mxy=M[0, 1], mxz=M[0, 2], myz=M[1, 2])


def config5_problem(scale=1.0, nstep=5000, nshots=16, nrec=1000, seed=5, perturbation=0.03,
                    save_boundary_values=True, **kw):
    """Batched adjoint 3D elastic: 96 x 96 x 48 hexahedra over 48 x 48 x 24
    km (scaled by `scale` in element count, same element size), 1D depth
    gradient with a seeded +-3 % random-field perturbation (2 km
    correlation), `nshots` random double-couple shots (Ricker 2 Hz) at 2 km
    depth, `nrec` receivers on the surface grid, dt 2e-3 s, Stacey on the
    sides and bottom, free top."""
    nx, ny, nz = max(1, round(96 * scale)), max(1, round(96 * scale)), max(1, round(48 * scale))
    h = 500.0
    bounds = (0.0, nx * h, 0.0, ny * h, 0.0, nz * h)
    rho, vp, vs = depth_gradient_model(nx, ny, nz, bounds, perturbation=perturbation, seed=seed)
    rng = np.random.default_rng(seed + 1)
    srcs = []
    for s in range(nshots):
        mt = random_double_couple(rng)
        srcs.append(MomentTensorSource(x=rng.uniform(0.2, 0.8) * bounds[1], y=rng.uniform(0.2, 0.8) * bounds[3],
                                       z=bounds[5] - min(2000.0, 0.25 * bounds[5]), f0=2.0, shot=s, **mt))
    side = int(math.ceil(math.sqrt(nrec)))
    gxr = np.linspace(0.05, 0.95, side) * bounds[1]
    gyr = np.linspace(0.05, 0.95, side) * bounds[3]
    XX, YY = np.meshgrid(gxr, gyr, indexing="xy")
    rec = np.stack([XX.ravel(), YY.ravel(), np.full(XX.size, bounds[5])], axis=1)[:nrec]
    return HexProblem(nx=nx, ny=ny, nz=nz, x0=bounds[0], x1=bounds[1], y0=bounds[2], y1=bounds[3],
                      z0=bounds[4], z1=bounds[5], rho=rho, vp=vp, vs=vs, dt=2e-3, nstep=nstep, nshots=nshots,
                      sources=srcs, receivers=rec, save_boundary_values=save_boundary_values, **kw)


class Simulation3D:
    """A 3D context on the GPU (sfb3_create)."""

    def __init__(self, problem: HexProblem):
        self._lib = load3()
        self.problem = problem
        desc, keep = problem.to_desc()
        h = C.c_void_p()
        _check(self._lib.sfb3_create(C.byref(desc), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self._lib.sfb3_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> sfb3_info:
        i = sfb3_info()
        _check(self._lib.sfb3_get_info(self.handle, C.byref(i)), self.handle)
        return i

    def run_forward(self, nstep=None):
        n = self.info().nstep if nstep is None else nstep
        _check(self._lib.sfb3_run_forward(self.handle, n), self.handle)

    def seismograms(self, shot=0, wavefield=0):
        i = self.info()
        out = np.zeros((i.nstep, i.nreceivers, 3), np.float32)
        _check(self._lib.sfb3_get_seismograms(self.handle, wavefield, shot, out.ctypes.data_as(_f), out.size),
               self.handle)
        return out

    def set_adjoint_sources(self, stf, shot=0):
        arr = np.ascontiguousarray(np.asarray(stf, np.float32))
        _check(self._lib.sfb3_set_adjoint_sources(self.handle, shot, arr.ctypes.data_as(_f), arr.size), self.handle)

    def run_combined(self):
        _check(self._lib.sfb3_run_combined(self.handle), self.handle)

    def kernels(self, which):
        i = self.info()
        out = np.zeros((i.nspec, NGLL, NGLL, NGLL), np.float64)
        _check(self._lib.sfb3_get_kernels(self.handle, which, out.ctypes.data_as(_d), out.size), self.handle)
        return out

    def field(self, wavefield=0, which=0, shot=0):
        i = self.info()
        out = np.zeros((3, i.nglob), np.float32)
        _check(self._lib.sfb3_get_field(self.handle, wavefield, which, shot, out.ctypes.data_as(_f), out.size),
               self.handle)
        return out

    def reset(self):
        _check(self._lib.sfb3_reset(self.handle), self.handle)

    def set_variant(self, variant):
        """Stiffness / Frechet kernels: 0 automatic, 1 scalar, 2 / 3 packed
        FP32x2 (two / three resident CTAs per SM)."""
        _check(self._lib.sfb3_set_variant(self.handle, variant), self.handle)

    def variant(self):
        return self._lib.sfb3_get_variant(self.handle)

    def time_kernel(self, what, reps):
        ms = C.c_double()
        _check(self._lib.sfb3_time_kernel(self.handle, what, reps, C.byref(ms)), self.handle)
        return ms.value


def gradients_from_kernels(problem: HexProblem, k_rho, k_mu, k_kappa):
    """d chi / d (rho, vp, vs) per local point from the kernels:
    d chi / d kappa = wJ K_kappa / kappa, d chi / d mu = wJ K_mu / mu,
    d chi / d rho (kappa, mu fixed) = wJ K_rho / rho, and the chain rule of
    kappa = rho (vp^2 - 4/3 vs^2), mu = rho vs^2."""
    rho = np.asarray(problem.rho, np.float64).reshape(k_rho.shape)
    vp = np.asarray(problem.vp, np.float64).reshape(k_rho.shape)
    vs = np.asarray(problem.vs, np.float64).reshape(k_rho.shape)
    kappa = rho * (vp ** 2 - 4.0 / 3.0 * vs ** 2)
    mu = rho * vs ** 2
    wJ = quadrature_volume(problem)
    with np.errstate(divide="ignore", invalid="ignore"):
        dk = np.where(kappa != 0, wJ * k_kappa / kappa, 0.0)
        dm = np.where(mu != 0, wJ * k_mu / mu, 0.0)
        dr = wJ * k_rho / rho
    g_vp = dk * rho * 2.0 * vp
    g_vs = dk * rho * (-8.0 / 3.0) * vs + dm * rho * 2.0 * vs
    g_rho = dr + dk * (vp ** 2 - 4.0 / 3.0 * vs ** 2) + dm * vs ** 2
    return g_rho, g_vp, g_vs


def misfit_and_residuals(sim: Simulation3D, observed):
    """chi = 1/2 sum_shots sum_steps sum_receivers |u - u_obs|^2 dt (FP64)
    and the residuals per shot."""
    i = sim.info()
    chi = 0.0
    res = []
    for s in range(i.nshots):
        r = sim.seismograms(shot=s).astype(np.float64) - np.asarray(observed[s], np.float64)
        res.append(r)
        chi += 0.5 * float(np.sum(r * r)) * i.dt
    return chi, res


class WaveformMisfit3D(torch.autograd.Function):
    """chi(rho, vp, vs) for the problem `sim` was built on (the model
    arguments must equal that problem's model: the context's material is
    fixed at creation); backward runs the combined loop on the GPU."""

    @staticmethod
    def forward(ctx, rho, vp, vs, sim: Simulation3D, observed):
        sim.reset()
        sim.run_forward()
        chi, res = misfit_and_residuals(sim, observed)
        ctx.sim = sim
        ctx.res = res
        ctx.device = rho.device
        ctx.dtype = rho.dtype
        return torch.tensor(chi, dtype=torch.float64, device=rho.device)

    @staticmethod
    def backward(ctx, grad_out):
        sim = ctx.sim
        for s, r in enumerate(ctx.res):
            sim.set_adjoint_sources(r.astype(np.float32), shot=s)
        sim.run_combined()
        g = gradients_from_kernels(sim.problem, sim.kernels(0), sim.kernels(1), sim.kernels(2))
        go = float(grad_out)
        to = lambda a: torch.as_tensor(a * go, dtype=ctx.dtype, device=ctx.device)
        return to(g[0]), to(g[1]), to(g[2]), None, None
