"""Shot-parallel misfit and gradient over torch.distributed ranks.

Shots are independent simulations on the same mesh and model, so the work
shards by shot: shot s runs on rank s % world_size, each rank advancing its
shots together on its own GPU (the batched kernels), and the only exchange is
one all-reduce of the FP64 misfit and one of the FP64 gradient at the end
(NCCL over NVLink on GPUs, gloo on CPU).  There is no per-step
communication; the reference has no distributed solver (its MPI layer only
wraps scalar reductions, include/specfem_mpi/specfem_mpi.hpp:44-230).

`ShardedMisfit` takes a problem (a 2D StructuredProblem or a 3D
HexProblem; each rank keeps its shots, renumbered 0..k-1) and a per-shard
compute function; the default compute runs the GPU forward + combined loop
of this package (`gpu_shard_compute`, or `gpu_shard_compute3d` for the 3D
path).
"""
from __future__ import annotations

from dataclasses import replace
from typing import Callable, List, Sequence

import numpy as np
import torch
import torch.distributed as dist


def shard_shots(nshots: int, world: int, rank: int) -> List[int]:
    """Round-robin assignment: shot s belongs to rank s % world."""
    return [s for s in range(nshots) if s % world == rank]


def restrict_to_shots(problem, shots: Sequence[int]):
    """Copy of a StructuredProblem keeping only `shots` (renumbered)."""
    index = {s: k for k, s in enumerate(shots)}
    sources = [replace(src, shot=index[src.shot]) for src in problem.sources if src.shot in index]
    return replace(problem, nshots=max(1, len(shots)), sources=sources)


def gpu_shard_compute(problem, model, observed):
    """Misfit and gradient of one shard on this rank's GPU."""
    from .autograd import WaveformMisfit
    from .simulation import Simulation
    sim = Simulation.structured(replace(problem, save_boundary_values=True))
    params = [torch.tensor(np.asarray(a, dtype=np.float64), requires_grad=True) for a in model]
    chi = WaveformMisfit.apply(*params, sim, torch.from_numpy(np.asarray(observed, dtype=np.float64)))
    chi.backward()
    return float(chi.detach()), [p.grad.numpy() for p in params]


def gpu_shard_compute3d(problem, model, observed):
    """Misfit and gradient of one shard of a 3D problem (HexProblem, the
    model per local point) on this rank's GPU: a batched context of the
    shard's shots, forward and combined run (WaveformMisfit3D)."""
    from .hex3d import Simulation3D, WaveformMisfit3D
    rho, vp, vs = (np.asarray(a, dtype=np.float32) for a in model)
    sim = Simulation3D(replace(problem, rho=rho, vp=vp, vs=vs, save_boundary_values=True))
    params = [torch.tensor(np.asarray(a, dtype=np.float64), requires_grad=True) for a in model]
    chi = WaveformMisfit3D.apply(*params, sim, np.asarray(observed, dtype=np.float64))
    chi.backward()
    sim.close()
    return float(chi.detach()), [p.grad.numpy() for p in params]


class ShardedMisfit:
    def __init__(self, problem, observed: np.ndarray,
                 compute: Callable = gpu_shard_compute, group=None, device: str = "cpu"):
        """problem: StructuredProblem (or HexProblem) with all shots;
        observed: displacement seismograms [nshots][nsig][nrec][2] (3D:
        [nshots][nstep][nrec][3])."""
        self.problem = problem
        self.observed = np.asarray(observed)
        self.compute = compute
        self.group = group
        self.device = device
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.shots = shard_shots(problem.nshots, self.world, self.rank)

    def __call__(self, model):
        """model: (rho, vp, vs) per local point.  Returns (misfit, [g_rho,
        g_vp, g_vs]) summed over every rank's shots."""
        if self.shots:
            local = restrict_to_shots(self.problem, self.shots)
            chi, grads = self.compute(local, model, self.observed[self.shots])
        else:
            chi, grads = 0.0, [np.zeros_like(np.asarray(a, dtype=np.float64)) for a in model]
        if self.world > 1:
            t = torch.tensor([chi], dtype=torch.float64, device=self.device)
            dist.all_reduce(t, group=self.group)
            chi = float(t.item())
            flat = torch.from_numpy(np.concatenate([g.reshape(-1) for g in grads])).to(self.device)
            dist.all_reduce(flat, group=self.group)
            flat = flat.cpu().numpy()
            out, k = [], 0
            for g in grads:
                out.append(flat[k:k + g.size].reshape(g.shape))
                k += g.size
            grads = out
        return chi, grads
