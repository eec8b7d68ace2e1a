"""Run a parameter file end to end, as the reference's `specfem2d -p` does:

  python -m specfempp_b200 -p specfem_config.yaml [-d default.yaml]

Forward mode runs the forward simulation and writes what its writers ask
(seismograms, the forward wavefield); combined mode reads the forward
wavefield, runs the adjoint + backward loop and writes the kernels.
"""
from __future__ import annotations

import argparse
import sys

from . import _capi as A


def run(parameter_file: str, default_file: str | None = None) -> None:
    lib = A.load()
    rc = lib.sfb_execute(parameter_file.encode(), default_file.encode() if default_file else None)
    A.check(rc, None)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m specfempp_b200")
    ap.add_argument("-p", "--parameters_file", required=True)
    ap.add_argument("-d", "--default_file", default=None)
    args = ap.parse_args(argv)
    try:
        run(args.parameters_file, args.default_file)
    except A.SfbError as e:
        print("error: %s" % e, file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
