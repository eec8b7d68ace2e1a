"""Differentiable waveform misfit through the GPU adjoint path.

``WaveformMisfit.apply(rho, vp, vs, sim, observed)`` runs the forward
simulation of every shot for the per-local-point model (rho, vp, vs)
[nspec][ngll][ngll], returns the L2 waveform misfit

    chi = 1/2 * sum_shots sum_samples sum_receivers |u_syn - u_obs|^2 * dt

(FP64 reduction over the displacement seismograms), and in backward runs
the combined adjoint + backward loop of the reference
(include/solver/time_marching.tpp:126-247) with the residuals as adjoint
sources, turning its Frechet kernels into the gradient with respect to the
model.  With the reference's kernels (frechet_derivative.hpp:14-138,
kappa' = lambda + mu):

    d chi / d kappa = wJ * K_kappa / kappa',  d chi / d mu = wJ * K_mu / mu,
    d chi / d rho   = wJ * K_rho / rho       (wJ = w_x w_z J per point)

and kappa = rho (vp^2 - 4/3 vs^2), mu = rho vs^2 give the gradient with
respect to (rho, vp, vs).  The Stacey traction's own dependence on the model
is not part of the reference's kernels; by default it is absent here too (the
gradient is the reference's).  With ``boundary_term=True`` (sixth argument)
the combined run also accumulates dchi/d(rho vp) and dchi/d(rho vs) at the
absorbing boundary points (sfb_set_stacey_kernels) and the gradient adds

    d chi / d rho += vp dchi/d(rho vp) + vs dchi/d(rho vs),
    d chi / d vp  += rho dchi/d(rho vp),   d chi / d vs += rho dchi/d(rho vs),

the derivative of the discrete misfit on absorbing meshes.  Elastic P-SV
models only.
"""
from __future__ import annotations

import numpy as np
import torch

from .simulation import Simulation

DISPLACEMENT = 0


def _np(t):
    return t.detach().to("cpu", torch.float64).numpy()


def gradients_from_kernels(sim: Simulation, rho, vp, vs):
    """d chi / d (rho, vp, vs) per local point from the accumulated kernels."""
    k_rho, k_mu, k_kappa = sim.kernels(0), sim.kernels(1), sim.kernels(2)
    kappa, mu, rho_s = sim.material()
    wJ = sim.quadrature_volume()
    kap_ref = kappa + mu / 3.0  # lambda + mu, the reference's kernel modulus
    with np.errstate(divide="ignore", invalid="ignore"):
        dk = np.where(kap_ref != 0, wJ * k_kappa / kap_ref, 0.0)
        dm = np.where(mu != 0, wJ * k_mu / mu, 0.0)
        dr = np.where(rho_s != 0, wJ * k_rho / rho_s, 0.0)
    g_vp = dk * rho * 2.0 * vp
    g_vs = dk * rho * (-8.0 / 3.0) * vs + dm * rho * 2.0 * vs
    g_rho = dr + dk * (vp ** 2 - 4.0 / 3.0 * vs ** 2) + dm * vs ** 2
    return g_rho, g_vp, g_vs


class WaveformMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, vp, vs, sim: Simulation, observed, boundary_term: bool = False):
        info = sim.info()
        if info.nelements[3] or info.nelements[1]:
            raise NotImplementedError("WaveformMisfit supports elastic P-SV models")
        r, p, s = _np(rho), _np(vp), _np(vs)
        sim.set_model(r, p, s)
        sim.reset()
        sim.run_forward()
        v = sim.problem_view()
        types = [v.seismogram_types[k] for k in range(info.nseismogram_types)]
        it = types.index(DISPLACEMENT)
        obs = observed.detach().to("cpu", torch.float64).numpy() if torch.is_tensor(observed) else np.asarray(observed)
        chi = 0.0
        res = []
        for shot in range(info.nshots):
            syn = sim.seismograms(shot=shot)[:, it].astype(np.float64)  # [nsig][nrec][2]
            rr = syn - obs[shot]
            res.append(rr)
            chi += 0.5 * float(np.sum(rr * rr)) * info.dt
        ctx.sim = sim
        ctx.boundary_term = bool(boundary_term)
        ctx.res = res
        ctx.model = (r, p, s)
        ctx.device = rho.device
        ctx.dtype = rho.dtype
        return torch.tensor(chi, dtype=torch.float64, device=rho.device)

    @staticmethod
    def backward(ctx, grad_out):
        sim = ctx.sim
        info = sim.info()
        if info.nstep_between_samples != 1:
            raise NotImplementedError("adjoint sources need one seismogram sample per step")
        for shot, rr in enumerate(ctx.res):
            sim.set_adjoint_sources(rr.astype(np.float32), shot=shot)
        sim.set_stacey_kernels(ctx.boundary_term)
        sim.run_combined()
        g_rho, g_vp, g_vs = gradients_from_kernels(sim, *ctx.model)
        if ctx.boundary_term:
            rho, vp, vs = ctx.model
            b_vp, b_vs = sim.kernels(6), sim.kernels(7)
            g_rho = g_rho + vp * b_vp + vs * b_vs
            g_vp = g_vp + rho * b_vp
            g_vs = g_vs + rho * b_vs
        go = float(grad_out)
        to = lambda g: torch.as_tensor(g * go, dtype=ctx.dtype, device=ctx.device)
        return to(g_rho), to(g_vp), to(g_vs), None, None, None
