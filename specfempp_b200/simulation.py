"""Python host API over the C ABI: one ``Simulation`` per library context.

Mirrors the reference's Python surface (``specfempp_core._execute`` runs a
YAML parameter file, src/python/core.cpp:46-66) and adds array access for
seismograms, fields and Frechet kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi as A


@dataclass
class Material:
    rho: float
    vp: float
    vs: float = 0.0  # 0 -> acoustic


@dataclass
class ForceSource:
    x: float
    z: float
    f0: float
    factor: float = 1e10
    angle: float = 0.0
    tshift: float = 0.0
    stf: str = "ricker"  # ricker | dirac | dgaussian
    shot: int = 0
    kind: str = "force"  # force | moment_tensor | user_defined
    mxx: float = 0.0
    mzz: float = 0.0
    mxz: float = 0.0


@dataclass
class Station:
    x: float
    z: float
    network: str = "AA"
    station: str = ""
    angle: float = 0.0


@dataclass
class StructuredProblem:
    """A structured quad mesh problem (benchmark workloads)."""
    nx: int
    nz: int
    x0: float
    x1: float
    z0: float
    z1: float
    materials: Sequence[Material]
    element_material: Optional[np.ndarray] = None  # [nz*nx] int32
    gll_model: Optional[tuple] = None  # (rho, vp, vs) float32 arrays [nspec, ngll, ngll]
    absorb: tuple = (True, True, False, True)  # bottom, right, top, left
    ngll: int = 5
    elastic_sh: bool = False
    dt: float = 1e-3
    nstep: int = 100
    t0: float = 0.0
    nshots: int = 1
    sources: Sequence[ForceSource] = field(default_factory=list)
    stations: Sequence[Station] = field(default_factory=list)
    seismogram_types: Sequence[str] = ("displacement",)
    nstep_between_samples: int = 1
    simulation: int = 0
    save_boundary_values: bool = False


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Simulation:
    """A simulation context (device buffers are created on first GPU use).

    ``precision`` 32 (default) is the product library; 64 binds the FP64
    verification build of the same kernels, for parity tests against the
    FP64 oracle."""

    def __init__(self, handle, precision: int = 32):
        self._h = handle
        self.precision = precision
        self._lib = A.load(precision)
        self._keep = []

    # ---- construction ---------------------------------------------------
    @classmethod
    def from_yaml(cls, parameter_file: str, default_file: Optional[str] = None,
                  precision: int = 32) -> "Simulation":
        lib = A.load(precision)
        h = C.c_void_p()
        rc = lib.sfb_create_from_yaml(parameter_file.encode(),
                                      default_file.encode() if default_file else None, C.byref(h))
        A.check(rc, None, lib)
        return cls(h, precision)

    @classmethod
    def structured(cls, p: StructuredProblem, precision: int = 32) -> "Simulation":
        lib = A.load(precision)
        keep = []
        d = A.sfb_structured_desc()
        d.nx, d.nz = p.nx, p.nz
        d.x0, d.x1, d.z0, d.z1 = p.x0, p.x1, p.z0, p.z1
        for k in range(4):
            d.absorb[k] = 1 if p.absorb[k] else 0
        d.ngll = p.ngll
        d.elastic_sh = 1 if p.elastic_sh else 0
        mats = (A.sfb_material * len(p.materials))(*[A.sfb_material(m.rho, m.vp, m.vs) for m in p.materials])
        keep.append(mats)
        d.nmaterials = len(p.materials)
        d.materials = mats
        em = p.element_material
        if em is None:
            em = np.zeros(p.nx * p.nz, dtype=np.int32)
        em = np.ascontiguousarray(em, dtype=np.int32)
        keep.append(em)
        d.element_material = em.ctypes.data_as(C.POINTER(C.c_int))
        if p.gll_model is not None:
            arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in p.gll_model]
            keep += arrs
            d.gll_rho, d.gll_vp, d.gll_vs = (_fptr(a) for a in arrs)
        d.dt, d.nstep, d.t0, d.nshots = p.dt, p.nstep, p.t0, p.nshots
        srcs = (A.sfb_source_desc * max(1, len(p.sources)))()
        stf_code = {"ricker": 0, "dirac": 1, "dgaussian": 2}
        for i, s in enumerate(p.sources):
            srcs[i].kind = {"force": 0, "moment_tensor": 1, "user_defined": 2}[s.kind]
            srcs[i].shot = s.shot
            srcs[i].wavefield = 0
            srcs[i].stf = stf_code[s.stf]
            srcs[i].x, srcs[i].z, srcs[i].angle = s.x, s.z, s.angle
            srcs[i].mxx, srcs[i].mzz, srcs[i].mxz = s.mxx, s.mzz, s.mxz
            srcs[i].f0 = s.f0 if s.stf != "dirac" else 1.0 / (10.0 * p.dt)
            srcs[i].tshift, srcs[i].factor = s.tshift, s.factor
        keep.append(srcs)
        d.nsources, d.sources = len(p.sources), srcs
        recs = (A.sfb_receiver_desc * max(1, len(p.stations)))()
        names = []
        for i, r in enumerate(p.stations):
            net = r.network.encode()
            sta = (r.station or "S%04d" % (i + 1)).encode()
            names += [net, sta]
            recs[i].network, recs[i].station = net, sta
            recs[i].x, recs[i].z, recs[i].angle = r.x, r.z, r.angle
        keep += [recs, names]
        d.nreceivers, d.receivers = len(p.stations), recs
        types = np.array([A.SEISMOGRAM_TYPES[t] for t in p.seismogram_types], dtype=np.int32)
        keep.append(types)
        d.nseismogram_types = len(types)
        d.seismogram_types = types.ctypes.data_as(C.POINTER(C.c_int))
        d.nstep_between_samples = p.nstep_between_samples
        d.simulation = p.simulation
        d.save_boundary_values = 1 if p.save_boundary_values else 0
        h = C.c_void_p()
        A.check(lib.sfb_create_structured(C.byref(d), C.byref(h)), None, lib)
        return cls(h, precision)

    def close(self):
        if self._h:
            self._lib.sfb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        return A.check(rc, self._h, self._lib)

    # ---- info / view ----------------------------------------------------
    def info(self) -> A.sfb_info:
        i = A.sfb_info()
        self._check(self._lib.sfb_get_info(self._h, C.byref(i)))
        return i

    def problem_view(self) -> A.sfb_problem_view:
        v = A.sfb_problem_view()
        self._check(self._lib.sfb_get_problem_view(self._h, C.byref(v)))
        return v

    # ---- reference-granularity entry points ------------------------------
    def initialize(self, wavefield: int = 0, dt: Optional[float] = None):
        if dt is None:
            dt = self.info().dt
        self._check(self._lib.sfb_domain_initialize(self._h, wavefield, dt))

    def run_forward(self, nstep: Optional[int] = None, graph: bool = True):
        if nstep is None:
            nstep = self.info().nstep
        self._check(self._lib.sfb_run_forward(self._h, nstep, 1 if graph else 0))

    def run_forward_unfused(self, nstep: Optional[int] = None):
        if nstep is None:
            nstep = self.info().nstep
        self._check(self._lib.sfb_run_forward_unfused(self._h, nstep))

    def compute_seismograms(self, isig_step: int = 0, wavefield: int = 0):
        """Record seismogram sample `isig_step` of the current fields
        (``domain_kernels::compute_seismograms``)."""
        self._check(self._lib.sfb_domain_compute_seismograms(self._h, wavefield, isig_step))

    def seismograms(self, wavefield: int = 0, shot: int = 0) -> np.ndarray:
        """[max_sig_step][ntypes][nreceivers][2]; float32, or float64 (every
        bit the device computed) for an FP64 context."""
        i = self.info()
        shape = (i.max_sig_step, i.nseismogram_types, i.nreceivers, 2)
        if self.precision == 64:
            out = np.zeros(shape, dtype=np.float64)
            self._check(self._lib.sfb_get_seismograms_f64(self._h, wavefield, shot,
                                                          out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
            return out
        out = np.zeros(shape, dtype=np.float32)
        self._check(self._lib.sfb_get_seismograms(self._h, wavefield, shot, _fptr(out), out.size))
        return out

    def field(self, medium: int, which: int, wavefield: int = 0, shot: int = 0) -> np.ndarray:
        """[ncomp][nglob] of u, v, a (which 0-2) or the inverse mass (3);
        float32, or float64 for an FP64 context."""
        i = self.info()
        nc = 2 if medium == A.MEDIUM_ELASTIC_PSV else 1
        if self.precision == 64:
            out = np.zeros((nc, i.nglob[medium]), dtype=np.float64)
            self._check(self._lib.sfb_get_field_f64(self._h, wavefield, medium, which, shot,
                                                    out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
            return out
        out = np.zeros((nc, i.nglob[medium]), dtype=np.float32)
        self._check(self._lib.sfb_get_field(self._h, wavefield, medium, which, shot, _fptr(out), out.size))
        return out

    def set_field(self, medium: int, which: int, values: np.ndarray, wavefield: int = 0, shot: int = 0):
        v = np.ascontiguousarray(values, dtype=np.float32)
        self._check(self._lib.sfb_set_field(self._h, wavefield, medium, which, shot, _fptr(v), v.size))

    def write_seismograms(self, directory: str, wavefield: int = 0, shot: int = 0):
        self._check(self._lib.sfb_write_seismograms(self._h, wavefield, shot, directory.encode()))

    def seismogram_times(self) -> np.ndarray:
        i = self.info()
        k = np.arange(i.max_sig_step, dtype=np.float32)
        return (k * np.float32(i.dt) * np.float32(i.nstep_between_samples) + np.float32(i.t0)).astype(np.float32)

    # ---- combined (adjoint + backward) run --------------------------------
    def set_adjoint_sources(self, stf: np.ndarray, shot: int = 0):
        """Adjoint source time functions [nstep][nreceivers][2] of `shot`
        (receiver r acts at its station with its Lagrange weights)."""
        a = np.ascontiguousarray(stf, dtype=np.float32)
        self._check(self._lib.sfb_set_adjoint_sources(self._h, shot, _fptr(a), a.size))

    def run_combined(self, graph: bool = True):
        self._check(self._lib.sfb_run_combined(self._h, self.info().nstep, 1 if graph else 0))

    def kernels(self, which: int) -> np.ndarray:
        """Frechet kernel summed over shots, [nspec][ngll][ngll] FP64:
        0 rho, 1 mu, 2 kappa, 3 rhop, 4 alpha, 5 beta (acoustic points:
        0 rho, 2 kappa, 3 rhop, 4 alpha)."""
        i = self.info()
        out = np.zeros((i.nspec, i.ngll, i.ngll), dtype=np.float64)
        self._check(self._lib.sfb_get_kernels(self._h, which, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    def set_model(self, rho, vp, vs):
        """Per-local-point model [nspec][ngll][ngll] (density, vp, vs)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (rho, vp, vs)]
        self._check(self._lib.sfb_set_model(self._h, _fptr(arrs[0]), _fptr(arrs[1]), _fptr(arrs[2]), arrs[0].size))

    def reset(self):
        self._check(self._lib.sfb_reset(self._h))

    def set_newmark_compensation(self, enable: bool = True):
        """Kahan-compensated u / v sums in the fused forward run."""
        self._check(self._lib.sfb_set_newmark_compensation(self._h, 1 if enable else 0))

    def set_checkpoint_interval(self, interval: int):
        """Forward snapshots every `interval` steps restored into the
        backward wavefield of the combined run (0: pure reconstruction)."""
        self._check(self._lib.sfb_set_checkpoint_interval(self._h, interval))

    def synchronize(self):
        """Wait for the context's work, run the NaN / Inf watchdog and report
        recorded device errors (SfbError)."""
        self._check(self._lib.sfb_synchronize(self._h))

    def set_stacey_kernels(self, enable: bool = True):
        """Also accumulate the Stacey traction's model derivatives in combined
        runs (kernels 6, 7: dchi/d(rho vp), dchi/d(rho vs))."""
        self._check(self._lib.sfb_set_stacey_kernels(self._h, 1 if enable else 0))

    def set_deterministic(self, enable: bool = True):
        """Bit-reproducible assembly (element colours, fixed-order sums);
        before the first device use."""
        self._check(self._lib.sfb_set_deterministic(self._h, 1 if enable else 0))

    def set_stiffness_variant(self, medium: int, variant: int):
        """Batched stiffness kernel of `medium` (1 packed two-shot, 2 scalar
        two-shot, 3 one shot per lane; 0 autotuned)."""
        self._check(self._lib.sfb_set_stiffness_variant(self._h, medium, variant))

    def write_properties(self, directory: str, element_chunk: int = 1):
        """Write the model as the reference's property writer does
        (<directory>/Properties/<medium>_isotropic/...)."""
        self._check(self._lib.sfb_write_properties(self._h, directory.encode(), element_chunk))

    def read_properties(self, directory: str, element_chunk: int = 1):
        """Replace the model from files in the reference's property layout."""
        self._check(self._lib.sfb_read_properties(self._h, directory.encode(), element_chunk))

    def quadrature_volume(self) -> np.ndarray:
        """w_x w_z J per local point [nspec][ngll][ngll] (FP64)."""
        v = self.problem_view()
        i = self.info()
        n = i.ngll
        w = np.ctypeslib.as_array(v.wgll, shape=(n,)).astype(np.float64)
        J = np.ctypeslib.as_array(v.jacobian, shape=(i.nspec * n * n,)).reshape(i.nspec, n, n).astype(np.float64)
        return w[None, :, None] * w[None, None, :] * J

    def material(self):
        """(kappa, mu, rho) per local point as stored (FP32 -> FP64)."""
        v = self.problem_view()
        i = self.info()
        shape = (i.nspec, i.ngll, i.ngll)
        get = lambda p: np.ctypeslib.as_array(p, shape=(int(np.prod(shape)),)).reshape(shape).astype(np.float64)
        return get(v.kappa), get(v.mu), get(v.rho)
