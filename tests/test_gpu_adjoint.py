"""GPU combined (adjoint + backward) loop and Frechet kernels, through the C
ABI, against the oracle's restatement of the reference
(include/solver/time_marching.tpp:126-247), and the differentiable misfit
against finite differences.

Kernels: relative L2 within 1e-3 of the FP32 oracle (the reference's
arithmetic) and of the FP64 oracle, or, where even the FP32 oracle is
further than that from FP64, of the same order from FP64 as the FP32 oracle
is: within 1e-3 + 2x its distance.  A kernel sums products of two
wavefields over every step, one of them reconstructed backward in time
through the Stacey replay, so its FP32 error is that reconstruction's
drift; the GPU's and the oracle's FP32 runs are two independent
realisations of it (their red-add order differs from run to run), which
one realisation's size bounds only up to a factor of order one.
Gradients: within 1e-3 of central finite differences.
"""
import numpy as np
import pytest
import torch

from adjoint_util import (anomaly, base_model, directions, misfit_fd_oracle, observed, problem)
from specfempp_b200 import Simulation

pytestmark = pytest.mark.gpu

NSTEP = 300
TOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def parity_ok(e32, e64, e_ref):
    return e32 <= TOL or e64 <= TOL + 1.5 * e_ref


def kernel_ok(e32, e64, e_ref):
    """Kernels: within 1e-3 of the reference's FP32 arithmetic (the oracle)
    and of its FP64 run -- the gradient bar -- or, where the FP32 problem is
    itself worse conditioned than that, of the same order from FP64 as the
    FP32 oracle (module docstring)."""
    return (e32 <= 1e-3 and e64 <= 1e-3) or e64 <= 1e-3 + 2.0 * e_ref


def gpu_combined(model, obs, absorb, nshots=1, checkpoint_interval=0):
    sim = Simulation.structured(problem(model, NSTEP, absorb, nshots))
    if checkpoint_interval:
        sim.set_checkpoint_interval(checkpoint_interval)
    sim.run_forward()
    stfs = []
    for s in range(nshots):
        syn = sim.seismograms(shot=s)[:, 0].astype(np.float64)
        stf = (syn - obs[s]).astype(np.float32)
        stfs.append(stf)
        sim.set_adjoint_sources(stf, shot=s)
    sim.run_combined()
    K = np.stack([sim.kernels(0), sim.kernels(1), sim.kernels(2)], axis=-1)
    return sim, K, stfs


def oracle_kernels(sim, stfs, precision):
    from oracle import bridge
    total = None
    for s, stf in enumerate(stfs):
        fwd = bridge.forward(sim, precision, shot=s, threads=8, want_fields=True, want_stacey=True)
        K = bridge.combined(sim, stf, fwd, precision=precision, shot=s, threads=8)
        total = K if total is None else total + K
    return total


@pytest.mark.parametrize("absorb", [(False,) * 4, (True, True, False, True)])
def test_gpu_kernels_match_oracle(absorb):
    p, model, XZ = base_model(nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb)
    sim, K, stfs = gpu_combined(model, obs, absorb)
    o32 = oracle_kernels(sim, stfs, 32)
    o64 = oracle_kernels(sim, stfs, 64)
    for c, name in enumerate(("rho", "mu", "kappa")):
        e32, e64, eref = rel_l2(K[..., c], o32[..., c]), rel_l2(K[..., c], o64[..., c]), rel_l2(o32[..., c], o64[..., c])
        print("kernel %s: vs FP32 %.2e vs FP64 %.2e (FP32 oracle vs FP64 %.2e)" % (name, e32, e64, eref))
        assert kernel_ok(e32, e64, eref), (name, e32, e64, eref)


@pytest.mark.parametrize("nshots", [3, 4])
def test_batched_kernels_sum_over_shots(nshots):
    """Odd S: separate Frechet launch; even S: Frechet fused into the
    batched backward stiffness launch."""
    absorb = (True, True, False, True)
    p, model, XZ = base_model(nshots=nshots, nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb, nshots=nshots)
    sim, K, stfs = gpu_combined(model, obs, absorb, nshots=nshots)
    o32 = oracle_kernels(sim, stfs, 32)
    o64 = oracle_kernels(sim, stfs, 64)
    for c in range(3):
        e32, e64, eref = rel_l2(K[..., c], o32[..., c]), rel_l2(K[..., c], o64[..., c]), rel_l2(o32[..., c], o64[..., c])
        print("S=%d kernel %d: vs FP32 %.2e vs FP64 %.2e (FP32 oracle vs FP64 %.2e)" % (nshots, c, e32, e64, eref))
        assert kernel_ok(e32, e64, eref)


def test_backward_reconstructs_forward_seismograms():
    absorb = (True, True, False, True)
    p, model, XZ = base_model(nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb)
    sim, _, _ = gpu_combined(model, obs, absorb)
    fwd = sim.seismograms(wavefield=0)
    # backward samples are numbered in loop order, last step first (as the
    # reference's combined loop stores them)
    bwd = sim.seismograms(wavefield=2)[::-1]
    err = rel_l2(bwd, fwd)
    print("backward reconstruction rel-L2 %.2e" % err)
    assert err < 1e-3


@pytest.mark.parametrize("nshots", [1, 2])
def test_autograd_gradient_matches_finite_differences(nshots):
    from specfempp_b200.autograd import WaveformMisfit
    absorb = (False,) * 4
    p, model, XZ = base_model(nshots=nshots, nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb, nshots=nshots)
    sim = Simulation.structured(problem(model, NSTEP, absorb, nshots))
    params = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in model]
    chi = WaveformMisfit.apply(*params, sim, torch.from_numpy(obs))
    chi.backward()
    grads = [t.grad.numpy() for t in params]
    for trial in range(2):
        d = directions(model, XZ, trial)
        fd = misfit_fd_oracle(model, obs, NSTEP, absorb, d, nshots=nshots)
        ad = sum(float(np.sum(g * dd)) for g, dd in zip(grads, d))
        print("trial %d: adjoint %.6e FD %.6e rel %.2e" % (trial, ad, fd, abs(ad - fd) / abs(fd)))
        assert abs(ad - fd) <= 1e-3 * abs(fd), (trial, ad, fd)


@pytest.mark.parametrize("nshots", [1, 2])
def test_checkpoints_bound_backward_reconstruction(nshots):
    """Forward snapshots every 50 steps restored into the backward wavefield:
    the backward seismograms stay at least as close to the forward ones as
    with pure reconstruction, and the kernels keep oracle parity."""
    absorb = (True, True, False, True)
    p, model, XZ = base_model(nshots=nshots, nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb, nshots=nshots)
    plain, K0, stfs = gpu_combined(model, obs, absorb, nshots=nshots)
    ck, K1, _ = gpu_combined(model, obs, absorb, nshots=nshots, checkpoint_interval=50)
    for s in range(nshots):
        e_plain = rel_l2(plain.seismograms(wavefield=2, shot=s)[::-1], plain.seismograms(wavefield=0, shot=s))
        e_ck = rel_l2(ck.seismograms(wavefield=2, shot=s)[::-1], ck.seismograms(wavefield=0, shot=s))
        print("shot %d backward vs forward seismograms: reconstruction %.2e, with snapshots %.2e" % (s, e_plain, e_ck))
        assert e_ck <= e_plain
    o32 = oracle_kernels(ck, stfs, 32)
    o64 = oracle_kernels(ck, stfs, 64)
    for c in range(3):
        assert kernel_ok(rel_l2(K1[..., c], o32[..., c]), rel_l2(K1[..., c], o64[..., c]),
                         rel_l2(o32[..., c], o64[..., c]))


def test_acoustic_kernels_match_oracle():
    """Acoustic combined run: rho, kappa and the derived rhop (sum over steps
    of rho_kl * kappa_kl) and alpha (2 kappa), point/kernels.hpp:189-192."""
    from specfempp_b200 import StructuredProblem, Material, ForceSource, Station
    p = StructuredProblem(nx=16, nz=12, x0=0, x1=800, z0=0, z1=600,
                          materials=[Material(1020.0, 1500.0, 0.0)],
                          absorb=(True, True, False, True), dt=5e-4, nstep=NSTEP,
                          sources=[ForceSource(x=400, z=300, f0=8.0, factor=1e10)],
                          stations=[Station(x=100 + 120 * k, z=500) for k in range(6)],
                          seismogram_types=("pressure",), save_boundary_values=True)
    sim = Simulation.structured(p)
    sim.run_forward()
    # smooth band-limited adjoint sources (Ricker pulses with seeded delays
    # and amplitudes), the kind a residual has
    rng = np.random.default_rng(5)
    t = np.arange(NSTEP) * 5e-4
    stf = np.zeros((NSTEP, 6, 2), np.float32)
    for r in range(6):
        a = (np.pi * 8.0 * (t - rng.uniform(0.03, 0.12))) ** 2
        stf[:, r, 0] = (rng.uniform(0.5, 1.5) * 1e-3 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    sim.set_adjoint_sources(stf)
    sim.run_combined()
    o32 = oracle_kernels(sim, [stf], 32)
    o64 = oracle_kernels(sim, [stf], 64)
    for which, ref in ((0, lambda o: o[..., 0]), (2, lambda o: o[..., 1]), (3, lambda o: o[..., 2]),
                       (4, lambda o: 2.0 * o[..., 1])):
        g = sim.kernels(which)
        e32, e64, eref = rel_l2(g, ref(o32)), rel_l2(g, ref(o64)), rel_l2(ref(o32), ref(o64))
        print("acoustic kernel %d: vs FP32 %.2e vs FP64 %.2e (FP32 oracle vs FP64 %.2e)" % (which, e32, e64, eref))
        assert np.abs(g).max() > 0
        assert kernel_ok(e32, e64, eref), (which, e32, e64, eref)


def test_reference_granularity_combined_loop():
    """time_marching<combined>::run (time_marching.tpp:126-247) driven from
    the host through the domain_kernels / newmark / frechet_kernels entry
    points, as the reference's own loop would call them, after the fused
    forward run: its kernels meet the kernel bar against the oracle."""
    import ctypes as C
    from specfempp_b200 import _capi as A
    absorb = (True, True, False, True)
    p, model, XZ = base_model(nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb)
    sim = Simulation.structured(problem(model, NSTEP, absorb))
    sim.run_forward()
    stf = (sim.seismograms()[:, 0].astype(np.float64) - obs[0]).astype(np.float32)
    sim.set_adjoint_sources(stf)
    lib, h, dt = A.load(), sim.handle, sim.info().dt
    ADJ, BWD, PSV, AC = 1, 2, 0, 3
    n = C.c_int()

    def call(rc):
        A.check(rc, h)

    for w in (ADJ, BWD):
        call(lib.sfb_domain_initialize(h, w, dt))
    for istep in range(NSTEP - 1, -1, -1):
        for m in (AC, PSV):
            call(lib.sfb_newmark_predictor(h, ADJ, m, C.byref(n)))
        for m in (AC, PSV):
            call(lib.sfb_domain_update_wavefields(h, ADJ, m, istep, C.byref(n)))
            call(lib.sfb_newmark_corrector(h, ADJ, m, C.byref(n)))
        for m in (PSV, AC):
            call(lib.sfb_newmark_predictor(h, BWD, m, C.byref(n)))
        for m in (PSV, AC):
            call(lib.sfb_domain_update_wavefields(h, BWD, m, istep, C.byref(n)))
            call(lib.sfb_newmark_corrector(h, BWD, m, C.byref(n)))
        if istep == NSTEP - 1:
            call(lib.sfb_load_backward_from_forward(h))
        call(lib.sfb_frechet_compute_derivatives(h, dt))
    K = np.stack([sim.kernels(0), sim.kernels(1), sim.kernels(2)], axis=-1)
    o32 = oracle_kernels(sim, [stf], 32)
    o64 = oracle_kernels(sim, [stf], 64)
    for c, name in enumerate(("rho", "mu", "kappa")):
        e32, e64, eref = rel_l2(K[..., c], o32[..., c]), rel_l2(K[..., c], o64[..., c]), rel_l2(o32[..., c], o64[..., c])
        print("host-driven combined loop, kernel %s: vs FP32 %.2e vs FP64 %.2e (FP32 oracle vs FP64 %.2e)"
              % (name, e32, e64, eref))
        assert kernel_ok(e32, e64, eref), (name, e32, e64, eref)
