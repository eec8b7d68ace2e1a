"""B200-native spectral-element time marching (SPECFEM++ 2D path).

The compute path is the CUDA library ``_lib/libspecfem_b200.so`` reached
through the C ABI of ``include/specfem_b200.h``; this package is the host-side
Python binding.  Importing it does not load the library; the first
``Simulation`` does, and fails loudly when it has not been built.
"""
from ._capi import (MEDIUM_ACOUSTIC, MEDIUM_ELASTIC_PSV, MEDIUM_ELASTIC_SH, SfbError,
                    WAVEFIELD_ADJOINT, WAVEFIELD_BACKWARD, WAVEFIELD_FORWARD, load)
from .simulation import (ForceSource, Material, Simulation, Station, StructuredProblem)

__all__ = [
    "Simulation", "StructuredProblem", "Material", "ForceSource", "Station", "SfbError", "load",
    "MEDIUM_ELASTIC_PSV", "MEDIUM_ELASTIC_SH", "MEDIUM_ACOUSTIC",
    "WAVEFIELD_FORWARD", "WAVEFIELD_ADJOINT", "WAVEFIELD_BACKWARD",
]
