"""The oracle's restatement of the reference's combined (adjoint + backward)
loop and Frechet kernels yields the gradient of the L2 waveform misfit:
checked against central finite differences of the FP64 oracle.  The
reference ships no numeric kernel fixtures (its Tromp 2005 benchmark is a
picture), so this pins the restatement mathematically."""
import numpy as np
import pytest

from adjoint_util import (anomaly, base_model, directions, kernel_gradient, misfit_fd_oracle, observed,
                          problem)

NSTEP = 300


@pytest.mark.parametrize("absorb,tol", [((False,) * 4, 2e-4), ((True,) * 4, 1e-2)])
def test_oracle_adjoint_gradient_matches_finite_differences(absorb, tol, native_lib, oracle_lib):
    from oracle import bridge
    from specfempp_b200 import Simulation
    p, model, XZ = base_model(nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb)
    sim = Simulation.structured(problem(model, NSTEP, absorb))
    fwd = bridge.forward(sim, 64, threads=8, want_fields=True, want_stacey=True)
    res = fwd["seismograms"][:, 0].astype(np.float64) - obs[0]
    K = bridge.combined(sim, res.astype(np.float32), fwd, precision=64, threads=8)
    grads = kernel_gradient(sim, K, model)
    for trial in range(2):
        d = directions(model, XZ, trial)
        fd = misfit_fd_oracle(model, obs, NSTEP, absorb, d)
        ad = sum(float(np.sum(g * dd)) for g, dd in zip(grads, d))
        assert abs(ad - fd) <= tol * abs(fd), (trial, ad, fd)
