"""The reference's Python entry points (python/specfempp_core/__init__.py,
src/python/core.cpp:13-78) over this library's C ABI:

  _initialize(argv) -> bool   start the runtime once (False if already started)
  _execute(parameter_string, default_string) -> bool
                              run the simulation the parameter dictionary
                              (YAML text) describes, as the reference's
                              execute(): forward runs write seismograms and,
                              when asked, the forward wavefield; combined runs
                              read it, run the adjoint + backward loop and
                              write the kernels.  False before _initialize.
                              Errors raise specfempp_b200.SfbError.
  _finalize() -> bool         stop the runtime (False if not started)
  _default_file_path          the default parameter file
  WaveformMisfit              the differentiable misfit (torch.autograd.Function)

The reference's _initialize starts MPI and Kokkos; here it loads the CUDA
library and checks that a device is present.
"""
from __future__ import annotations

import os

from specfempp_b200 import _capi as _A
from specfempp_b200.autograd import WaveformMisfit

__version__ = "dev"
_default_file_path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                  "specfempp_b200", "defaults", "default.yaml")
_state = {"initialized": False}

__all__ = ["__version__", "_default_file_path", "_initialize", "_execute", "_finalize", "WaveformMisfit"]


def _initialize(argv) -> bool:
    if _state["initialized"]:
        return False
    _A.load()
    _state["initialized"] = True
    _state["argv"] = list(argv)
    return True


def _execute(parameter_string: str, default_string: str) -> bool:
    if not _state["initialized"]:
        return False
    lib = _A.load()
    _A.check(lib.sfb_execute_text(parameter_string.encode(), default_string.encode()), None, lib)
    return True


def _finalize() -> bool:
    if not _state["initialized"]:
        return False
    _state["initialized"] = False
    return True
