"""The reference's two-phase adjoint workflow through parameter files
(src/execute.cpp): a forward run that writes seismograms and its wavefield
(include/io/wavefield/writer.tpp), traveltime adjoint sources made from the
seismograms by the xadj_seismogram restatement, then a combined run that
reads the wavefield and the External adjoint sources and writes the kernels
(include/io/kernel/writer.tpp).  The kernel files must agree with the kernels
of one in-memory context given the same adjoint sources, and the written
wavefield with that context's final fields, to the run-to-run spread of
FP32 red-add order (the file round trip itself is exact in FP32)."""
import os

import numpy as np
import pytest

from specfempp_b200 import Simulation
from specfempp_b200 import adjoint_sources as AS
from specfempp_b200.__main__ import run
from workflow_util import NX, NZ, STATIONS, read_kernel, structured, write_combined, write_forward

pytestmark = pytest.mark.gpu

NSTEP, DT = 400, 5e-4


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def test_two_phase_workflow_matches_in_memory(tmp_path):
    root = str(tmp_path)
    run(write_forward(root, NSTEP, DT))
    seis = os.path.join(root, "seismograms")
    names = ["AA.S%04d.S2" % (k + 1) for k in range(len(STATIONS))]
    t, _ = AS.read_trace(os.path.join(seis, names[0] + ".BXZ.semd"))
    adj = os.path.join(root, "adjoint_sources")
    for name in names:
        AS.xadj_seismogram(t[0] + 0.02, t[-1] - 0.02, name, seis, adj, 4)
    run(write_combined(root, NSTEP, DT, adj, names))

    # in memory: same case, same adjoint sources
    sim = Simulation.structured(structured(NSTEP, DT))
    sim.run_forward()
    stf = np.zeros((NSTEP, len(STATIONS), 2), np.float32)
    for r, name in enumerate(names):
        for c, comp in enumerate(("BXX", "BXZ")):
            stf[:, r, c] = AS.read_trace(os.path.join(adj, "%s.%s.adj" % (name, comp)))[1][:NSTEP]
    # the written forward wavefield is the forward run's final state
    for which, ds in enumerate(("Displacement", "Velocity", "Acceleration")):
        f = np.loadtxt(os.path.join(root, "ForwardWavefield", "Step%06d" % NSTEP, "elastic_psv", ds + ".txt"))
        # two runs differ by the order of the FP32 red-adds (5e-5 seen on the acceleration)
        assert rel_l2(f, sim.field(0, which).reshape(-1)) <= 1e-3, ds
    sim.set_adjoint_sources(stf)
    sim.run_combined()
    info = sim.info()
    for q, name in enumerate(("rho", "mu", "kappa", "rhop", "alpha", "beta")):
        k_file = read_kernel(os.path.join(root, "kernels"), "elastic_psv_isotropic", name, NX * NZ, info.ngll)
        k_mem = sim.kernels(q)
        err = rel_l2(k_file, k_mem)
        print("kernel %s: file vs in-memory rel-L2 %.2e" % (name, err))
        assert np.abs(k_mem).max() > 0
        assert err <= 1e-3, (name, err)
