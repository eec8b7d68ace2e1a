"""The shot-sharded gradient on the GPU through torch.distributed with NCCL,
one rank (the only GPU a run here has): ShardedMisfit with the GPU shard
compute equals WaveformMisfit on the same shots, and the FP64 all-reduce
runs on the device."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch

from adjoint_util import anomaly, base_model, observed, problem

pytestmark = pytest.mark.gpu

NSTEP = 300  # long enough for the waves to reach the receivers


def test_sharded_misfit_one_rank_nccl(monkeypatch):
    # both sides with the deterministic assembly: the same shots give the
    # same bits
    monkeypatch.setenv("SFB_DETERMINISTIC", "1")
    import torch.distributed as dist
    from specfempp_b200 import Simulation
    from specfempp_b200.autograd import WaveformMisfit
    from specfempp_b200.distributed import ShardedMisfit, gpu_shard_compute
    absorb = (False,) * 4
    p, model, XZ = base_model(nshots=2, nstep=NSTEP)
    obs = observed(anomaly(model, XZ, p), NSTEP, absorb, nshots=2)
    prob = problem(model, NSTEP, absorb, 2)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        chi, grads = ShardedMisfit(prob, obs, compute=gpu_shard_compute, device="cuda")(model)
    finally:
        dist.destroy_process_group()
    sim = Simulation.structured(prob)
    params = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in model]
    ref = WaveformMisfit.apply(*params, sim, torch.from_numpy(obs))
    ref.backward()
    assert chi == float(ref.detach())
    for g, t in zip(grads, params):
        err = np.linalg.norm(g - t.grad.numpy()) / np.linalg.norm(t.grad.numpy())
        print("sharded gradient vs single process: %.2e" % err)
        assert err == 0.0, err
