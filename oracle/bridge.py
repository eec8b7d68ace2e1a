"""ORACLE (test infrastructure): Python bridge to ``oracle/_build/liboracle.so``.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, as the checker.  It runs the CPU
restatement of the reference on the problem view exported by a product
``Simulation`` so both sides start from identical discrete inputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build():
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def load():
    global _lib
    if _lib is None:
        srcs = [os.path.join(HERE, f) for f in ("oracle.cpp", "oracle3d.cpp")]
        if not os.path.exists(LIB) or max(os.path.getmtime(f) for f in srcs) > os.path.getmtime(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.oracle_forward.restype = C.c_int
        lib.oracle_forward.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_float), C.POINTER(C.POINTER(C.c_float)),
                                       C.POINTER(C.c_float)]
        lib.oracle_combined.restype = C.c_int
        lib.oracle_combined.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(C.c_float), C.POINTER(C.POINTER(C.c_float)),
                                        C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_float)]
        lib.oracle_forward_f64.restype = C.c_int
        lib.oracle_forward_f64.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_double), C.POINTER(C.POINTER(C.c_double)),
                                           C.POINTER(C.c_double)]
        lib.oracle_combined_f64.restype = C.c_int
        lib.oracle_combined_f64.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                            C.POINTER(C.c_float), C.POINTER(C.POINTER(C.c_double)),
                                            C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
        lib.oracle_seismograms_f64.restype = C.c_int
        lib.oracle_seismograms_f64.argtypes = [C.c_void_p, C.POINTER(C.POINTER(C.c_double)),
                                               C.POINTER(C.c_double)]
        lib.oracle_seismograms.restype = C.c_int
        lib.oracle_seismograms.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.POINTER(C.c_double)),
                                           C.POINTER(C.c_float)]
        lib.oracle_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def forward(sim, precision: int = 32, shot: int = 0, nstep=None, threads: int = 1,
            want_fields: bool = False, want_stacey: bool = False, exact: bool = False):
    """Run the oracle forward on ``sim``'s problem.  Returns a dict with
    ``seismograms`` [nsig][ntypes][nrec][2] and optionally the final fields
    (keys ``psv``, ``sh``, ``acoustic`` -> (u, v, a, minv) arrays [nc][nglob]).
    ``exact`` (precision 64 only): every output in FP64 instead of rounded
    to FP32, for comparisons at FP64 rounding level."""
    lib = load()
    view = sim.problem_view()
    info = sim.info()
    if nstep is None:
        nstep = info.nstep
    if exact and precision != 64:
        raise ValueError("exact outputs need precision 64")
    dt, ct = (np.float64, C.c_double) if exact else (np.float32, C.c_float)
    seis = np.zeros((info.max_sig_step, info.nseismogram_types, info.nreceivers, 2), dtype=dt)
    fields = {}
    ptrs = (C.POINTER(ct) * 12)()
    bufs = []
    if want_fields:
        k = 0
        for name, med, nc in (("psv", 0, 2), ("sh", 1, 1), ("acoustic", 3, 1)):
            arrs = [np.zeros((nc, info.nglob[med]), dtype=dt) for _ in range(4)]
            fields[name] = arrs
            for a in arrs:
                ptrs[k] = a.ctypes.data_as(C.POINTER(ct))
                bufs.append(a)
                k += 1
    store = None
    if want_stacey:
        store = np.zeros((nstep, info.nspec, info.ngll, info.ngll, 2), dtype=dt)
    if exact:
        rc = lib.oracle_forward_f64(C.addressof(view), shot, nstep, threads,
                                    seis.ctypes.data_as(C.POINTER(ct)),
                                    ptrs if want_fields else None,
                                    store.ctypes.data_as(C.POINTER(ct)) if store is not None else None)
    else:
        rc = lib.oracle_forward(C.addressof(view), precision, shot, nstep, threads,
                                seis.ctypes.data_as(C.POINTER(C.c_float)),
                                ptrs if want_fields else None,
                                store.ctypes.data_as(C.POINTER(C.c_float)) if store is not None else None)
    if rc != 0:
        raise RuntimeError("oracle failed: " + lib.oracle_last_error().decode())
    out = {"seismograms": seis}
    if want_fields:
        out.update(fields)
    if store is not None:
        out["stacey_store"] = store
    return out


def seismograms(sim, fields, precision: int = 64, exact: bool = False):
    """Seismograms of given fields (one record, [ntypes][nrec][2]), as the
    reference's compute_seismograms(0) on a loaded wavefield.  ``fields``
    maps ``psv`` / ``sh`` / ``acoustic`` to (u, v, a) arrays [nc][nglob] in
    this library's numbering; missing media are zero.  ``exact``
    (precision 64): FP64 output."""
    lib = load()
    view = sim.problem_view()
    info = sim.info()
    ptrs = (C.POINTER(C.c_double) * 9)()
    keep = []
    k = 0
    for name in ("psv", "sh", "acoustic"):
        for which in range(3):
            if name in fields:
                a = np.ascontiguousarray(fields[name][which], dtype=np.float64)
                keep.append(a)
                ptrs[k] = a.ctypes.data_as(C.POINTER(C.c_double))
            k += 1
    if exact:
        seis = np.zeros((info.nseismogram_types, info.nreceivers, 2), dtype=np.float64)
        rc = lib.oracle_seismograms_f64(C.addressof(view), ptrs, seis.ctypes.data_as(C.POINTER(C.c_double)))
    else:
        seis = np.zeros((info.nseismogram_types, info.nreceivers, 2), dtype=np.float32)
        rc = lib.oracle_seismograms(C.addressof(view), precision, ptrs, seis.ctypes.data_as(C.POINTER(C.c_float)))
    if rc != 0:
        raise RuntimeError("oracle failed: " + lib.oracle_last_error().decode())
    return seis


def combined(sim, adjoint_stf, fwd, precision: int = 64, shot: int = 0, threads: int = 1,
             want_backward_seismograms: bool = False, exact: bool = False, stacey_kernels: bool = False):
    """Run the oracle's combined (adjoint + backward) loop.  ``fwd`` is the
    result of ``forward(..., want_fields=True, want_stacey=True)`` (the
    forward run's last state and Stacey store; with ``exact``, of an exact
    forward); ``adjoint_stf`` is [nstep][nrec][2].  Returns FP64 kernels
    [nspec, ngll, ngll, 3] (elastic: rho, mu, kappa; acoustic: rho, kappa,
    sum of per-step rho * kappa) and optionally the backward seismograms.
    ``stacey_kernels`` (exact only): also the P-SV Stacey-traction
    derivatives [nspec, ngll, ngll, 2] (dchi/d(rho vp), dchi/d(rho vs)),
    returned after the kernels."""
    lib = load()
    view = sim.problem_view()
    info = sim.info()
    nstep = info.nstep
    if exact and precision != 64:
        raise ValueError("exact outputs need precision 64")
    dt, ct = (np.float64, C.c_double) if exact else (np.float32, C.c_float)
    stf = np.ascontiguousarray(adjoint_stf, dtype=np.float32)
    assert stf.shape == (nstep, info.nreceivers, 2)
    bufs = (C.POINTER(ct) * 9)()
    keep = []
    k = 0
    for name in ("psv", "sh", "acoustic"):
        for which in range(3):
            a = np.ascontiguousarray(fwd[name][which], dtype=dt)
            keep.append(a)
            bufs[k] = a.ctypes.data_as(C.POINTER(ct))
            k += 1
    store = np.ascontiguousarray(fwd["stacey_store"], dtype=dt)
    kernels = np.zeros((info.nspec, info.ngll, info.ngll, 3), dtype=np.float64)
    bseis = None
    if want_backward_seismograms:
        bseis = np.zeros((info.max_sig_step, info.nseismogram_types, info.nreceivers, 2), dtype=dt)
    kb = None
    if stacey_kernels:
        if not exact:
            raise ValueError("the Stacey-traction derivatives come with exact outputs")
        kb = np.zeros((info.nspec, info.ngll, info.ngll, 2), dtype=np.float64)
    if exact:
        rc = lib.oracle_combined_f64(C.addressof(view), shot, nstep, threads,
                                     stf.ctypes.data_as(C.POINTER(C.c_float)), bufs,
                                     store.ctypes.data_as(C.POINTER(ct)),
                                     kernels.ctypes.data_as(C.POINTER(C.c_double)),
                                     bseis.ctypes.data_as(C.POINTER(ct)) if bseis is not None else None,
                                     kb.ctypes.data_as(C.POINTER(C.c_double)) if kb is not None else None)
    else:
        rc = lib.oracle_combined(C.addressof(view), precision, shot, nstep, threads,
                                 stf.ctypes.data_as(C.POINTER(C.c_float)), bufs,
                                 store.ctypes.data_as(C.POINTER(C.c_float)),
                                 kernels.ctypes.data_as(C.POINTER(C.c_double)),
                                 bseis.ctypes.data_as(C.POINTER(C.c_float)) if bseis is not None else None)
    if rc != 0:
        raise RuntimeError("oracle failed: " + lib.oracle_last_error().decode())
    out = [kernels]
    if want_backward_seismograms:
        out.append(bseis)
    if kb is not None:
        out.append(kb)
    return tuple(out) if len(out) > 1 else kernels
