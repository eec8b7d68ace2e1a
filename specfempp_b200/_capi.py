"""ctypes binding of the C ABI in ``include/specfem_b200.h``.

This is the binding a Python maintainer of the reference would add next to
``python/specfempp_core`` (the reference's pybind11 module only exposes
``_execute(yaml)``; arrays never cross that boundary).  Every struct here
mirrors the header field for field.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libspecfem_b200.so")
# Verification build: the same driver and generic kernels in FP64 (test
# infrastructure for parity against the FP64 oracle; not a product path).
LIB64_PATH = os.path.join(HERE, "_lib", "libspecfem_b200_fp64.so")

SFB_OK = 0
ERRORS = {
    -1: "SFB_E_INVALID",
    -2: "SFB_E_CUDA",
    -3: "SFB_E_IO",
    -4: "SFB_E_STATE",
    -5: "SFB_E_ACCOUNTING",
    -6: "SFB_E_NONFINITE",
    -7: "SFB_E_NOMEM",
}

MEDIUM_ELASTIC_PSV = 0
MEDIUM_ELASTIC_SH = 1
MEDIUM_ACOUSTIC = 3
WAVEFIELD_FORWARD = 0
WAVEFIELD_ADJOINT = 1
WAVEFIELD_BACKWARD = 2
SEISMOGRAM_TYPES = {"displacement": 0, "velocity": 1, "acceleration": 2, "pressure": 3}


class sfb_material(C.Structure):
    _fields_ = [("rho", C.c_double), ("vp", C.c_double), ("vs", C.c_double)]


class sfb_source_desc(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("shot", C.c_int), ("wavefield", C.c_int), ("stf", C.c_int),
        ("x", C.c_double), ("z", C.c_double), ("angle", C.c_double),
        ("mxx", C.c_double), ("mzz", C.c_double), ("mxz", C.c_double),
        ("f0", C.c_double), ("tshift", C.c_double), ("factor", C.c_double),
        ("stf_table", C.POINTER(C.c_float)),
    ]


class sfb_receiver_desc(C.Structure):
    _fields_ = [("network", C.c_char_p), ("station", C.c_char_p),
                ("x", C.c_double), ("z", C.c_double), ("angle", C.c_double)]


class sfb_structured_desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("nz", C.c_int),
        ("x0", C.c_double), ("x1", C.c_double), ("z0", C.c_double), ("z1", C.c_double),
        ("absorb", C.c_int * 4), ("ngll", C.c_int), ("elastic_sh", C.c_int),
        ("nmaterials", C.c_int), ("materials", C.POINTER(sfb_material)),
        ("element_material", C.POINTER(C.c_int)),
        ("gll_rho", C.POINTER(C.c_float)), ("gll_vp", C.POINTER(C.c_float)),
        ("gll_vs", C.POINTER(C.c_float)),
        ("dt", C.c_double), ("nstep", C.c_int), ("t0", C.c_double), ("nshots", C.c_int),
        ("nsources", C.c_int), ("sources", C.POINTER(sfb_source_desc)),
        ("nreceivers", C.c_int), ("receivers", C.POINTER(sfb_receiver_desc)),
        ("nseismogram_types", C.c_int), ("seismogram_types", C.POINTER(C.c_int)),
        ("nstep_between_samples", C.c_int), ("simulation", C.c_int),
        ("save_boundary_values", C.c_int),
    ]


class sfb_info(C.Structure):
    _fields_ = [
        ("ngll", C.c_int), ("nspec", C.c_int), ("nshots", C.c_int), ("nstep", C.c_int),
        ("nstep_between_samples", C.c_int), ("max_sig_step", C.c_int),
        ("nglob", C.c_int * 4), ("nelements", C.c_int * 4),
        ("nreceivers", C.c_int), ("nseismogram_types", C.c_int), ("nsources", C.c_int),
        ("simulation", C.c_int), ("dt", C.c_double), ("t0", C.c_double),
        ("device_bytes", C.c_size_t), ("kernel_launches", C.c_uint64),
        ("stiffness_variant", C.c_int * 4), ("private_points", C.c_int), ("nadjoint_sources", C.c_int),
    ]


_P = C.POINTER
class sfb_problem_view(C.Structure):
    _fields_ = [
        ("ngll", C.c_int), ("nspec", C.c_int), ("nshots", C.c_int), ("nstep", C.c_int),
        ("nstep_between_samples", C.c_int), ("dt", C.c_double), ("t0", C.c_double),
        ("xi", _P(C.c_double)), ("wgll", _P(C.c_double)), ("hprime", _P(C.c_double)),
        ("medium", _P(C.c_int)), ("iglob", _P(C.c_int)), ("nglob", C.c_int * 4),
        ("xix", _P(C.c_float)), ("xiz", _P(C.c_float)), ("gammax", _P(C.c_float)),
        ("gammaz", _P(C.c_float)), ("jacobian", _P(C.c_float)),
        ("kappa", _P(C.c_float)), ("mu", _P(C.c_float)), ("rho", _P(C.c_float)),
        ("rho_inverse", _P(C.c_float)),
        ("bnd", _P(C.c_uint8)), ("bnd_nx", _P(C.c_float)), ("bnd_nz", _P(C.c_float)),
        ("bnd_w", _P(C.c_float)),
        ("ncouple_acoustic", C.c_int), ("ncouple_elastic", C.c_int),
        ("couple_acoustic_self", _P(C.c_int)), ("couple_acoustic_other", _P(C.c_int)),
        ("couple_acoustic_factor", _P(C.c_float)), ("couple_acoustic_nx", _P(C.c_float)),
        ("couple_acoustic_nz", _P(C.c_float)),
        ("couple_elastic_self", _P(C.c_int)), ("couple_elastic_other", _P(C.c_int)),
        ("couple_elastic_factor", _P(C.c_float)), ("couple_elastic_nx", _P(C.c_float)),
        ("couple_elastic_nz", _P(C.c_float)),
        ("nsources", C.c_int), ("src_ispec", _P(C.c_int)), ("src_shot", _P(C.c_int)),
        ("src_wavefield", _P(C.c_int)), ("src_array", _P(C.c_float)), ("src_stf", _P(C.c_float)),
        ("nreceivers", C.c_int), ("rec_ispec", _P(C.c_int)), ("rec_lagrange", _P(C.c_float)),
        ("rec_sin", _P(C.c_float)), ("rec_cos", _P(C.c_float)),
        ("nseismogram_types", C.c_int), ("seismogram_types", _P(C.c_int)),
    ]


# Every entry point the header declares, with its ctypes signature.
_ctx = C.c_void_p
SIGNATURES = {
    "sfb_create_from_yaml": (C.c_int, [C.c_char_p, C.c_char_p, _P(_ctx)]),
    "sfb_create_structured": (C.c_int, [_P(sfb_structured_desc), _P(_ctx)]),
    "sfb_destroy": (None, [_ctx]),
    "sfb_last_error": (C.c_char_p, [_ctx]),
    "sfb_get_info": (C.c_int, [_ctx, _P(sfb_info)]),
    "sfb_domain_initialize": (C.c_int, [_ctx, C.c_int, C.c_double]),
    "sfb_domain_update_wavefields": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_int, _P(C.c_int)]),
    "sfb_domain_compute_seismograms": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "sfb_newmark_predictor": (C.c_int, [_ctx, C.c_int, C.c_int, _P(C.c_int)]),
    "sfb_newmark_corrector": (C.c_int, [_ctx, C.c_int, C.c_int, _P(C.c_int)]),
    "sfb_frechet_compute_derivatives": (C.c_int, [_ctx, C.c_double]),
    "sfb_run_forward": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "sfb_run_forward_unfused": (C.c_int, [_ctx, C.c_int]),
    "sfb_synchronize": (C.c_int, [_ctx]),
    "sfb_probe_device_wait": (C.c_int, [_ctx, C.c_longlong]),
    "sfb_run_combined": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "sfb_get_seismograms": (C.c_int, [_ctx, C.c_int, C.c_int, _P(C.c_float), C.c_size_t]),
    "sfb_get_seismograms_f64": (C.c_int, [_ctx, C.c_int, C.c_int, _P(C.c_double), C.c_size_t]),
    "sfb_get_field_f64": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_int, C.c_int, _P(C.c_double), C.c_size_t]),
    "sfb_real_bytes": (C.c_int, []),
    "sfb_get_field": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_int, C.c_int, _P(C.c_float), C.c_size_t]),
    "sfb_set_field": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_int, C.c_int, _P(C.c_float), C.c_size_t]),
    "sfb_set_adjoint_sources": (C.c_int, [_ctx, C.c_int, _P(C.c_float), C.c_size_t]),
    "sfb_get_kernels": (C.c_int, [_ctx, C.c_int, _P(C.c_double), C.c_size_t]),
    "sfb_copy_forward_to_backward": (C.c_int, [_ctx, _ctx]),
    "sfb_write_seismograms": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_char_p]),
    "sfb_get_problem_view": (C.c_int, [_ctx, _P(sfb_problem_view)]),
    "sfb_set_source_time_function": (C.c_int, [_ctx, C.c_int, _P(C.c_float), C.c_size_t]),
    "sfb_get_stream": (C.c_int, [_ctx, _P(C.c_void_p)]),
    "sfb_time_stiffness": (C.c_int, [_ctx, C.c_int, C.c_int, _P(C.c_double)]),
    "sfb_set_stiffness_variant": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "sfb_set_deterministic": (C.c_int, [_ctx, C.c_int]),
    "sfb_set_stacey_kernels": (C.c_int, [_ctx, C.c_int]),
    "sfb_set_newmark_compensation": (C.c_int, [_ctx, C.c_int]),
    "sfb_set_checkpoint_interval": (C.c_int, [_ctx, C.c_int]),
    "sfb_write_wavefield": (C.c_int, [_ctx, C.c_int, C.c_char_p]),
    "sfb_write_wavefield_step": (C.c_int, [_ctx, C.c_int, C.c_char_p]),
    "sfb_load_backward_from_forward": (C.c_int, [_ctx]),
    "sfb_read_wavefield": (C.c_int, [_ctx, C.c_int, C.c_char_p]),
    "sfb_write_kernels": (C.c_int, [_ctx, C.c_char_p, C.c_int]),
    "sfb_write_properties": (C.c_int, [_ctx, C.c_char_p, C.c_int]),
    "sfb_read_properties": (C.c_int, [_ctx, C.c_char_p, C.c_int]),
    "sfb_execute": (C.c_int, [C.c_char_p, C.c_char_p]),
    "sfb_execute_text": (C.c_int, [C.c_char_p, C.c_char_p]),
    "sfb_create_from_yaml_text": (C.c_int, [C.c_char_p, C.c_char_p, _P(_ctx)]),
    "sfb_assemble_inverse_mass_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    _P(C.c_double), C.c_double, C.c_void_p, C.c_void_p]),
    "sfb_noalloc_last_error": (C.c_char_p, []),
    "sfb_set_model": (C.c_int, [_ctx, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_size_t]),
    "sfb_reset": (C.c_int, [_ctx]),
}

# entry points that only the product (FP32) library has
FP32_ONLY = ("sfb_assemble_inverse_mass_noalloc", "sfb_noalloc_last_error")

_libs = {}


def load(precision: int = 32):
    """Load the product library (precision 32) or the FP64 verification
    build (precision 64); raises if it has not been built."""
    if precision in _libs:
        return _libs[precision]
    if precision not in (32, 64):
        raise ValueError("precision must be 32 or 64")
    path = LIB_PATH if precision == 32 else LIB64_PATH
    if not os.path.exists(path):
        raise RuntimeError(
            "specfempp_b200 native library not built (%s); run "
            "`python -m specfempp_b200.build` or __graft_entry__.build()" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        if precision == 64 and name in FP32_ONLY:
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.sfb_real_bytes() * 8 != precision:
        raise RuntimeError("%s computes in %d-bit reals, expected %d" % (path, lib.sfb_real_bytes() * 8, precision))
    _libs[precision] = lib
    return lib


class SfbError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, message))
        self.code = code


def check(code: int, ctx=None, lib=None):
    if code != SFB_OK:
        lib = lib or load()
        msg = lib.sfb_last_error(ctx)
        raise SfbError(code, msg.decode() if msg else "")
    return code
