"""Adjoint sources from seismograms: the reference's `xadj_seismogram`
(fortran/meshfem2d/adj_seismogram.f90) and the L2 waveform residual.

Cross-correlation traveltime adjoint source (Tromp, Tape & Liu 2005, eq. 42;
adj_seismogram.f90:214-300): with s(t) the synthetic trace, w(t) a Welch
window over [tstart, tend], v = ds/dt and a = d2s/dt2 by centred differences
(one-sided at the ends),

    N = dt * sum(w * s * a),     f(t) = w(t) * v(t) / N    (0 when |N| <= 1e-40)

and the file written is two columns "time value" per sample, the format the
reference's external source-time-function reader takes
(src/source_time_function/external.cpp).

CLI, same arguments as xadj_seismogram:

  python -m specfempp_b200.adjoint_sources t1 t2 NET.STA synthetics/ adjoint/ adj_comp

reads `synthetics/NET.STA.BXX.semd` (and BXZ, or BXY for adj_comp 2) and
writes `adjoint/NET.STA.BX{X,Y,Z}.adj`; adj_comp 1 = X, 2 = Y (SH), 3 = Z,
4 = X and Z.
"""
from __future__ import annotations

import math
import os
import sys
from typing import Tuple

import numpy as np

EPS = 1e-40
SMALLVAL = 1e-9


def read_trace(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """Two-column ASCII trace -> (time, value) as float64."""
    data = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if data.shape[0] < 2 or data.shape[1] < 2:
        raise ValueError("%s: need at least two 'time value' lines" % path)
    return data[:, 0], data[:, 1]


def write_trace(path: str, t0: float, dt: float, values: np.ndarray):
    with open(path, "w") as f:
        for i, v in enumerate(values):
            f.write("%.15e %.15e\n" % (t0 + i * dt, v))


def window_indices(nstep: int, t0: float, dt: float, tstart: float, tend: float) -> Tuple[int, int]:
    """0-based inclusive [istart, iend] of the window, clamped to the trace as
    adj_seismogram.f90:190-207 does (1-based there)."""
    istart = math.floor((tstart - t0) / dt) + 1
    iend = math.ceil((tend - t0) / dt) + 1
    if istart < 1:
        istart = 1
    if istart > nstep:
        istart = nstep - 1
    if iend < istart:
        iend = istart + 1
    if iend > nstep:
        iend = nstep
    if istart >= iend:
        raise ValueError("empty time window")
    return istart - 1, iend - 1


def welch_window(nstep: int, istart: int, iend: int) -> np.ndarray:
    """w = 1 - (2 (i - istart) / (iend - istart) - 1)^2 on [istart, iend], 0 elsewhere."""
    w = np.zeros(nstep)
    i = np.arange(istart, iend + 1, dtype=np.float64)
    w[istart:iend + 1] = 1.0 - (2.0 * (i - istart) / (iend - istart) - 1.0) ** 2
    return w


def centred_derivative(x: np.ndarray, dt: float) -> np.ndarray:
    d = np.zeros_like(x)
    d[1:-1] = (x[2:] - x[:-2]) / (2.0 * dt)
    d[0] = (x[1] - x[0]) / dt
    d[-1] = (x[-1] - x[-2]) / dt
    return d


def traveltime_adjoint_source(trace: np.ndarray, t0: float, dt: float, tstart: float, tend: float) -> np.ndarray:
    s = np.asarray(trace, dtype=np.float64)
    istart, iend = window_indices(len(s), t0, dt, tstart, tend)
    w = welch_window(len(s), istart, iend)
    v = centred_derivative(s, dt)
    a = centred_derivative(v, dt)
    norm = dt * float(np.sum(w * s * a))
    if abs(norm) <= EPS:
        return np.zeros_like(s)
    return v * w / norm


def waveform_adjoint_source(synthetic: np.ndarray, observed: np.ndarray) -> np.ndarray:
    """Adjoint source of chi = 1/2 sum |s - d|^2 dt: the residual s - d."""
    return np.asarray(synthetic, dtype=np.float64) - np.asarray(observed, dtype=np.float64)


def xadj_seismogram(tstart: float, tend: float, station: str, synthetics_folder: str,
                    adjoint_folder: str, adj_comp: int):
    """The reference tool's file-level behaviour (one station)."""
    if adj_comp not in (1, 2, 3, 4):
        raise ValueError("adj_comp must be 1 (X), 2 (Y), 3 (Z) or 4 (X & Z)")
    if tstart >= tend:
        raise ValueError("tstart must be less than tend")
    read = ["BXY"] if adj_comp == 2 else ["BXX", "BXZ"]
    traces = {}
    t0 = dt = None
    for comp in read:
        t, s = read_trace(os.path.join(synthetics_folder, "%s.%s.semd" % (station, comp)))
        tt0, tdt = t[0], (t[-1] - t[0]) / (len(t) - 1)
        if t0 is None:
            t0, dt, n = tt0, tdt, len(t)
        elif len(t) != n or abs(tt0 - t0) > SMALLVAL or abs(tdt - dt) > SMALLVAL:
            raise ValueError("traces of %s disagree in length, start or step" % station)
        traces[comp] = s
    os.makedirs(adjoint_folder, exist_ok=True)
    out = {}
    for comp in (["BXY"] if adj_comp == 2 else ["BXX", "BXZ"]):
        active = (comp == "BXX" and adj_comp in (1, 4)) or (comp == "BXZ" and adj_comp in (3, 4)) or comp == "BXY"
        f = traveltime_adjoint_source(traces[comp], t0, dt, tstart, tend) if active else np.zeros(n)
        write_trace(os.path.join(adjoint_folder, "%s.%s.adj" % (station, comp)), t0, dt, f)
        out[comp] = f
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 6:
        print(__doc__)
        return 1
    xadj_seismogram(float(argv[0]), float(argv[1]), argv[2], argv[3], argv[4], int(argv[5]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
