"""Shared set-up of the adjoint tests: a small homogeneous elastic model
(the adjoint workload shrunk), 'observed' data from a model with a
Gaussian -10 % vp/vs anomaly, and smooth perturbation directions (the same
value at coincident GLL points)."""
import numpy as np

from specfempp_b200 import Simulation
from specfempp_b200 import workloads as W


def problem(model, nstep, absorb, nshots=1):
    p = W.adjoint_model(scale=0.1, nshots=nshots, nstep=nstep)
    p.absorb = absorb
    p.gll_model = tuple(np.asarray(a, dtype=np.float32) for a in model)
    p.save_boundary_values = True
    return p


def base_model(nshots=1, nstep=300):
    p = W.adjoint_model(scale=0.1, nshots=nshots, nstep=nstep)
    rho, vp, vs = [a.astype(np.float64) for a in p.gll_model]
    X, Z = W.gll_coordinates(p.nx, p.nz, p.x0, p.x1, p.z0, p.z1)
    return p, (rho, vp, vs), (X, Z)


def anomaly(model, XZ, p):
    rho, vp, vs = model
    X, Z = XZ
    g = np.exp(-((X - p.x1 / 2) ** 2 + (Z - p.z1 / 2) ** 2) / (2 * 200.0 ** 2))
    return rho, vp * (1 - 0.1 * g), vs * (1 - 0.1 * g)


def directions(model, XZ, trial):
    rho, vp, vs = model
    X, Z = XZ
    return (rho * np.sin((X + Z) / 1000.0 + trial),
            vp * np.sin(X / 700.0 + trial) * np.cos(Z / 900.0),
            vs * np.cos(X / 800.0) * np.sin(Z / 600.0 + trial))


def misfit_fd_oracle(model, obs, nstep, absorb, direction, h=1e-4, nshots=1):
    """Central finite difference of the misfit with the FP64 oracle."""
    from oracle import bridge
    vals = []
    for sgn in (1, -1):
        m = tuple(a + sgn * h * d for a, d in zip(model, direction))
        sim = Simulation.structured(problem(m, nstep, absorb, nshots))
        chi = 0.0
        dt = sim.info().dt
        for s in range(nshots):
            syn = bridge.forward(sim, 64, shot=s, threads=8)["seismograms"][:, 0].astype(np.float64)
            chi += 0.5 * np.sum((syn - obs[s]) ** 2) * dt
        vals.append(chi)
    return (vals[0] - vals[1]) / (2 * h)


def observed(model_obs, nstep, absorb, nshots=1):
    from oracle import bridge
    sim = Simulation.structured(problem(model_obs, nstep, absorb, nshots))
    return np.stack([bridge.forward(sim, 64, shot=s, threads=8)["seismograms"][:, 0].astype(np.float64)
                     for s in range(nshots)])


def kernel_gradient(sim, kernels, model):
    """d chi / d (rho, vp, vs) from kernels [nspec][ngll][ngll][3] (rho, mu, kappa)."""
    rho, vp, vs = model
    kappa, mu, rho_s = sim.material()
    wJ = sim.quadrature_volume()
    dk = wJ * kernels[..., 2] / (kappa + mu / 3.0)
    dm = wJ * kernels[..., 1] / mu
    dr = wJ * kernels[..., 0] / rho_s
    return (dr + dk * (vp ** 2 - 4.0 / 3.0 * vs ** 2) + dm * vs ** 2,
            dk * rho * 2.0 * vp,
            dk * rho * (-8.0 / 3.0) * vs + dm * rho * 2.0 * vs)
