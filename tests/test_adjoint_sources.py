"""Adjoint-source generation (the reference's xadj_seismogram,
fortran/meshfem2d/adj_seismogram.f90): vectorised restatement against a
plain-loop restatement, window clamping, the zero-norm branch, the file-level
tool, and the traveltime property dT = dt * sum(f * ds) for a shifted pulse."""
import math
import os

import numpy as np
import pytest

from specfempp_b200 import adjoint_sources as AS


def ricker(t, f0, tc):
    a = (math.pi * f0 * (t - tc)) ** 2
    return (1 - 2 * a) * np.exp(-a)


def loop_reference(s, t0, dt, tstart, tend):
    """Line-by-line loop form of adj_seismogram.f90:190-300 (1-based there)."""
    n = len(s)
    istart = math.floor((tstart - t0) / dt) + 1
    iend = math.ceil((tend - t0) / dt) + 1
    istart = max(istart, 1)
    if istart > n:
        istart = n - 1
    if iend < istart:
        iend = istart + 1
    iend = min(iend, n)
    w = [0.0] * (n + 1)
    for it in range(istart, iend + 1):
        w[it] = 1.0 - (2 * (it - istart) / (iend - istart) - 1.0) ** 2
    x = [0.0] + list(s)
    v = [0.0] * (n + 1)
    for it in range(2, n):
        v[it] = (x[it + 1] - x[it - 1]) / (2 * dt)
    v[1] = (x[2] - x[1]) / dt
    v[n] = (x[n] - x[n - 1]) / dt
    a = [0.0] * (n + 1)
    for it in range(2, n):
        a[it] = (v[it + 1] - v[it - 1]) / (2 * dt)
    a[1] = (v[2] - v[1]) / dt
    a[n] = (v[n] - v[n - 1]) / dt
    norm = dt * sum(w[i] * x[i] * a[i] for i in range(1, n + 1))
    if abs(norm) <= 1e-40:
        return np.zeros(n)
    return np.array([v[i] * w[i] / norm for i in range(1, n + 1)])


def test_matches_loop_restatement():
    rng = np.random.default_rng(0)
    s = rng.standard_normal(400)
    for (t0, dt, ts, te) in [(-1.0, 0.01, 0.2, 2.0), (0.0, 0.02, -5.0, 100.0), (0.5, 0.005, 1.0, 1.02)]:
        np.testing.assert_allclose(AS.traveltime_adjoint_source(s, t0, dt, ts, te),
                                   loop_reference(s, t0, dt, ts, te), rtol=1e-12, atol=1e-300)


def test_window_clamping_and_zero_norm():
    assert AS.window_indices(100, 0.0, 0.1, -3.0, 50.0) == (0, 99)
    assert AS.window_indices(100, 0.0, 0.1, 20.0, 30.0) == (98, 99)
    with pytest.raises(ValueError):
        AS.window_indices(1, 0.0, 0.1, 0.0, 1.0)
    assert np.all(AS.traveltime_adjoint_source(np.zeros(50), 0.0, 0.01, 0.1, 0.3) == 0.0)


def test_traveltime_shift_property():
    dt, t0 = 0.001, 0.0
    t = t0 + dt * np.arange(3000)
    s = ricker(t, 5.0, 1.5)
    f = AS.traveltime_adjoint_source(s, t0, dt, 0.9, 2.1)
    for tau in (2 * dt, 5 * dt):
        ds = ricker(t - tau, 5.0, 1.5) - s  # the same pulse arriving tau later
        dT = dt * float(np.sum(f * ds))
        assert abs(dT / tau - 1.0) < 0.02, (tau, dT)


def test_file_tool(tmp_path):
    dt, t0 = 0.01, -1.2
    t = t0 + dt * np.arange(500)
    syn = tmp_path / "syn"
    syn.mkdir()
    for comp, amp in (("BXX", 1.0), ("BXZ", -2.0)):
        AS.write_trace(str(syn / ("AA.S0001.S2.%s.semd" % comp)), t0, dt, amp * ricker(t, 3.0, 1.0))
    out = tmp_path / "adj"
    AS.main(["0.2", "2.0", "AA.S0001.S2", str(syn), str(out), "3"])
    tx, fx = AS.read_trace(str(out / "AA.S0001.S2.BXX.adj"))
    tz, fz = AS.read_trace(str(out / "AA.S0001.S2.BXZ.adj"))
    assert np.all(fx == 0.0) and np.abs(fz).max() > 0
    np.testing.assert_allclose(tz, t, atol=1e-12)
    np.testing.assert_allclose(fz, AS.traveltime_adjoint_source(-2.0 * ricker(t, 3.0, 1.0), t0, dt, 0.2, 2.0),
                               rtol=1e-12)
    assert not os.path.exists(out / "AA.S0001.S2.BXY.adj")
