"""Analytic displacement of a moment-tensor point source in a homogeneous,
isotropic, unbounded elastic solid (test helper).

The point-force response is Stokes' solution (Aki & Richards, Quantitative
Seismology, 2nd ed., eq. 4.23): for a force f(t) along x_p at the origin,

  u_n = 1/(4 pi rho) (3 g_n g_p - d_np) / r^3  int_{r/a}^{r/b} tau f(t - tau) dtau
      + 1/(4 pi rho a^2) g_n g_p / r  f(t - r/a)
      - 1/(4 pi rho b^2) (g_n g_p - d_np) / r  f(t - r/b),

g = x / r the direction cosines.  A moment tensor M_pq m(t) at xi gives
u_n = M_pq d/dxi_q G_np = -M_pq d/dx_q G_np (G the response to f = m),
evaluated here by central differences in the receiver position (step
1e-4 r), which keeps the formula to the one above.
"""
from __future__ import annotations

import numpy as np


def _stokes(x, t, stf, rho, vp, vs, nquad=400):
    """G[n][p] at receiver offset x (3,) for times t (nt,)."""
    r = float(np.linalg.norm(x))
    g = x / r
    ta, tb = r / vp, r / vs
    tau = np.linspace(ta, tb, nquad)
    wq = np.full(nquad, (tb - ta) / (nquad - 1))
    wq[0] *= 0.5
    wq[-1] *= 0.5
    near = (stf(t[:, None] - tau[None, :]) * tau[None, :]) @ wq   # (nt,)
    fa = stf(t - ta)
    fb = stf(t - tb)
    G = np.empty((len(t), 3, 3))
    for n in range(3):
        for p in range(3):
            d = 1.0 if n == p else 0.0
            G[:, n, p] = ((3 * g[n] * g[p] - d) / r ** 3 * near / (4 * np.pi * rho)
                          + g[n] * g[p] / r * fa / (4 * np.pi * rho * vp ** 2)
                          - (g[n] * g[p] - d) / r * fb / (4 * np.pi * rho * vs ** 2))
    return G


def moment_tensor_displacement(rec, src, M, t, stf, rho, vp, vs):
    """Displacement [nt][3] at `rec` of the moment tensor M (3x3) at `src`
    with time function stf(t) (vectorised callable)."""
    x = np.asarray(rec, float) - np.asarray(src, float)
    r = float(np.linalg.norm(x))
    h = 1e-4 * r
    u = np.zeros((len(t), 3))
    for q in range(3):
        e = np.zeros(3)
        e[q] = h
        dG = (_stokes(x + e, t, stf, rho, vp, vs) - _stokes(x - e, t, stf, rho, vp, vs)) / (2 * h)
        for p in range(3):
            u -= M[p][q] * dG[:, :, p]
    return u


def ricker_stf(f0, factor=1.0, tshift=0.0):
    """The reference's Ricker source time function: -factor (1 - 2 a t^2)
    exp(-a t^2), a = (pi f0)^2, t measured from tshift."""
    a = (np.pi * f0) ** 2

    def stf(t):
        tt = np.asarray(t) - tshift
        return -factor * (1.0 - 2.0 * a * tt * tt) * np.exp(-a * tt * tt)
    return stf
