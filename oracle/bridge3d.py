"""ORACLE (test infrastructure): Python bridge to the 3D restatement in
``oracle/oracle3d.cpp`` (``oracle/_build/liboracle.so``).

Only tests import this module, as the checker.  The oracle builds its own
mesh, numbering, quadrature and source / receiver arrays from the same
``sfb3_desc`` the product receives.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import bridge

_d = C.POINTER(C.c_double)
_ready = False


def _lib():
    global _ready
    lib = bridge.load()
    if not _ready:
        lib.oracle3d_forward.restype = C.c_int
        lib.oracle3d_forward.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _d, _d, _d]
        lib.oracle3d_combined.restype = C.c_int
        lib.oracle3d_combined.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _d, _d, _d, _d, _d]
        lib.oracle3d_nentries.restype = C.c_int
        lib.oracle3d_nentries.argtypes = [C.c_void_p]
        lib.oracle3d_last_error.restype = C.c_char_p
        _ready = True
    return lib


def _nglob(p):
    return (4 * p.nx + 1) * (4 * p.ny + 1) * (4 * p.nz + 1)


def forward(problem, shot=0, precision=64, threads=8, want_store=None):
    """Seismograms [nstep][nrec][3], final (u, v, a) [3][3][nglob] and, for
    problems that keep boundary values, the Stacey store."""
    lib = _lib()
    desc, keep = problem.to_desc()
    nrec = desc.nreceivers
    seis = np.zeros((problem.nstep, nrec, 3))
    final = np.zeros((3, 3, _nglob(problem)))
    if want_store is None:
        want_store = problem.save_boundary_values
    store = None
    if want_store:
        store = np.zeros((problem.nstep, lib.oracle3d_nentries(C.byref(desc)), 3))
    rc = lib.oracle3d_forward(C.byref(desc), shot, precision, threads, seis.ctypes.data_as(_d),
                              final.ctypes.data_as(_d), store.ctypes.data_as(_d) if store is not None else None)
    if rc != 0:
        raise RuntimeError(lib.oracle3d_last_error().decode())
    return {"seismograms": seis, "final": final, "store": store}


def combined(problem, fwd, adj_stf, shot=0, precision=64, threads=8, kernels=None):
    """Kernels [nspec*125][3] (rho, mu, kappa; added to `kernels` when given)
    and backward seismograms [nstep][nrec][3] of one shot."""
    lib = _lib()
    desc, keep = problem.to_desc()
    nloc = problem.nspec * 125
    if kernels is None:
        kernels = np.zeros((nloc, 3))
    bseis = np.zeros((problem.nstep, desc.nreceivers, 3))
    stf = np.ascontiguousarray(np.asarray(adj_stf, np.float64))
    final = np.ascontiguousarray(fwd["final"])
    store = fwd["store"]
    rc = lib.oracle3d_combined(C.byref(desc), shot, precision, threads, stf.ctypes.data_as(_d),
                               final.ctypes.data_as(_d), store.ctypes.data_as(_d) if store is not None else None,
                               kernels.ctypes.data_as(_d), bseis.ctypes.data_as(_d))
    if rc != 0:
        raise RuntimeError(lib.oracle3d_last_error().decode())
    return {"kernels": kernels, "bseis": bseis}
