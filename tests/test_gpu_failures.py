"""Failure detection on the GPU without faulting it, through the C ABI.

  * NaN / Inf watchdog: a NaN put into a source time function from the host
    makes the forward run return SFB_E_NONFINITE; the context stays usable
    (reset, a finite time function, and the next run is clean);
  * bounded device waits: a probe enqueues the stiffness kernels' bounded
    mbarrier wait on a barrier nothing arrives at, with a short limit; the
    next reporting call returns the timeout (SFB_E_CUDA), the
    reference-granularity entry points report it without synchronising,
    and the context stays usable;
  * the combined run's watchdog covers the adjoint and backward wavefields.
No kernel is made to fault, trap or hang: every wait is bounded and every
error is a value the host reads.
"""
import ctypes as C

import time

import numpy as np
import pytest

from specfempp_b200 import SfbError, Simulation
from specfempp_b200 import _capi as A
from specfempp_b200 import workloads as W

pytestmark = pytest.mark.gpu

SFB_E_CUDA, SFB_E_NONFINITE = -2, -6


def small():
    return W.plain_elastic(scale=0.2, nstep=200, seismogram_types=("displacement",))


def test_nan_in_source_time_function_is_reported():
    sim = Simulation.structured(small())
    sim.run_forward(50)  # clean
    view = sim.problem_view()
    n = sim.info().nstep * 2
    stf = np.ctypeslib.as_array(view.src_stf, shape=(n,)).copy()
    bad = stf.copy()
    bad[2 * 60] = np.nan  # step 60, first component
    lib = A.load()
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    assert lib.sfb_set_source_time_function(sim.handle, 0, ptr(bad), n) == 0
    with pytest.raises(SfbError) as e:
        sim.run_forward(50)
    assert e.value.code == SFB_E_NONFINITE
    # the context is still usable
    assert lib.sfb_set_source_time_function(sim.handle, 0, ptr(stf), n) == 0
    sim.reset()
    sim.run_forward(200)
    assert np.isfinite(sim.seismograms()).all()
    ref = Simulation.structured(small())
    ref.run_forward()
    assert np.abs(ref.seismograms() - sim.seismograms()).max() <= 1e-5 * np.abs(ref.seismograms()).max()


def test_bounded_wait_that_runs_out_is_reported():
    sim = Simulation.structured(small())
    sim.run_forward(20)
    lib = A.load()
    # about 0.5 ms at 2 GHz
    assert lib.sfb_probe_device_wait(sim.handle, 1 << 20) == 0
    with pytest.raises(SfbError) as e:
        sim.synchronize()
    assert e.value.code == SFB_E_CUDA and "wait timed out" in str(e.value)
    # reported once: the context is usable again
    sim.synchronize()
    sim.run_forward(20)
    assert np.isfinite(sim.seismograms()).all()


def test_reference_granularity_entry_points_report_without_sync():
    sim = Simulation.structured(small())
    lib = A.load()
    h = sim.handle
    n = C.c_int()
    assert lib.sfb_domain_initialize(h, 0, sim.info().dt) == 0
    assert lib.sfb_probe_device_wait(h, 1 << 20) == 0
    codes = []
    # the probe gives up after about half a millisecond; its record reaches
    # the host copy that the entry points poll soon after (the calls below
    # are paced so that the loop outlasts it)
    for istep in range(200):
        codes.append(lib.sfb_newmark_predictor(h, 0, 0, C.byref(n)))
        codes.append(lib.sfb_domain_update_wavefields(h, 0, 0, istep, C.byref(n)))
        codes.append(lib.sfb_newmark_corrector(h, 0, 0, C.byref(n)))
        if SFB_E_CUDA in codes:
            break
        time.sleep(0.002)
    assert SFB_E_CUDA in codes, codes
    assert "wait timed out" in lib.sfb_last_error(h).decode()
    assert lib.sfb_synchronize(h) == 0


def test_combined_run_watchdog():
    from adjoint_util import problem, base_model
    p, model, _ = base_model(nstep=120)
    sim = Simulation.structured(problem(model, 120, (True, True, False, True)))
    sim.run_forward()
    stf = np.zeros((120, sim.info().nreceivers, 2), np.float32)
    stf[40, 0, 0] = np.inf
    sim.set_adjoint_sources(stf)
    with pytest.raises(SfbError) as e:
        sim.run_combined()
    assert e.value.code == SFB_E_NONFINITE
