#!/usr/bin/env python
"""Benchmark of the SEM time-marching hot path on B200.

Workload (default): the coupled acoustic-elastic forward of 400 x 300 NGLL=5
elements over 20 km x 15 km (see specfempp_b200/workloads.py), synthetic
seeded model, FP32.  A "step" is one Newmark time step of the whole domain.
The metric is GLL point updates per second: nshots * nglob * steps / time,
nglob summed over media.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload coupled|plain|batched|hex3d] [--no-secondary]

On one GPU the default line also carries `batched` (the 64-shot 800 x 400
batched forward: rate and whole-step HBM fraction) and `fwi` (forward +
adjoint gradient of 64 shots batched against one shot alone on the
200 x 200 adjoint mesh: per-shot device time and speed-up).

`--workload hex3d` times the 3D batched elastic forward on config 5's
hexahedral mesh (16 shots; `--scale` shrinks the element counts) and
reports its stiffness launch against max(bytes / HBM peak, flops / FP32
peak).

Under torchrun each rank runs an independent replica (the forward path does
not shard; "replicas only"); the reported value sums all ranks' point updates
over the slowest rank's device time.  `--impl reference` times the CPU
restatement of the reference (oracle/) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

GRAPH_STEPS = 26  # one CUDA-graph chunk (25 fused steps) + the closing step


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


SCALE = 1.0  # element-count scale of the workload (1 = the full configuration)
VARIANT = 0  # batched stiffness kernel (0: autotuned; see sfb_set_stiffness_variant)


def pin_variant(sim):
    """Pin the stiffness kernel of every medium (the numbers mean different
    kernels for single-shot and batched contexts)."""
    if VARIANT:
        for medium in (0, 1, 3):
            sim.set_stiffness_variant(medium, VARIANT)


def make_problem(workload: str, nstep: int):
    from specfempp_b200 import workloads as W
    if workload == "coupled":
        return W.coupled(SCALE, nstep=nstep, seismogram_types=("pressure",))
    if workload == "plain":
        return W.plain_elastic(SCALE, nstep=nstep)
    if workload == "batched":
        return W.batched(SCALE, nshots=64, nstep=nstep)
    raise SystemExit("unknown workload " + workload)


def workload_config(workload, info, p):
    return {
        "workload": {"coupled": "coupled acoustic-elastic 2D forward, 400x300 NGLL=5 elements, 20x15 km",
                     "plain": "plain elastic P-SV 2D forward, 100x80 NGLL=5 elements, 4x3 km",
                     "batched": "batched elastic P-SV 2D forward, 800x400 NGLL=5 elements, 64 shots"}[workload],
        "nspec": int(info.nspec),
        "nglob": int(sum(info.nglob)),
        "nshots": int(info.nshots),
        "dt": float(info.dt),
        "receivers": int(info.nreceivers),
        "stiffness_variant": {name: int(info.stiffness_variant[m])
                              for name, m in (("elastic_psv", 0), ("elastic_sh", 1), ("acoustic", 3))
                              if info.nelements[m] > 0},
    }


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if s[5 + k].lower() in ("active", "1")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name, variant):
    """DRAM bytes per launch of the dominant kernel, stiffness `variant` (a
    number, or a name), from the committed ncu summary (null when that
    variant was not captured)."""
    path = os.path.join(ROOT, "profiles", name)
    key = ("dram_bytes_per_launch_full_size[variant %d]:" % variant if isinstance(variant, int)
           else "dram_bytes_per_launch_full_size[%s]:" % variant)
    try:
        for line in open(path):
            if line.startswith(key):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def affine_block(info, medium):
    """True when the single-shot stiffness of `medium` reads the compact block
    of affine elements (variant 3): geometry per element, not per point."""
    return info.nshots == 1 and info.stiffness_variant[medium] == 3


def static_bytes(info, medium, P):
    """Static words of one launch over `medium`: per local point 4 (global
    index) + 4 * P (material; P = 3 elastic, 2 acoustic) and the geometry,
    4 * 5 per local point, or 4 * 5 per element with the compact block."""
    nel, nn = info.nelements[medium], info.ngll * info.ngll
    geometry = nel * 20 if affine_block(info, medium) else nel * nn * 20
    return nel * nn * (4 + 4 * P) + geometry


def stiffness_bytes(info, problem_view, medium):
    """Algorithmic bytes of one stiffness launch of `medium`: the static words
    plus one read of the displacement and one write of the force per shot and
    DOF."""
    P = 3 if medium in (0, 1) else 2
    C = 2 if medium == 0 else 1
    return static_bytes(info, medium, P) + info.nshots * info.nglob[medium] * C * 4 * 2


def step_bytes(info):
    """Algorithmic HBM bytes of one whole time step: the static words of every
    medium, per global point the inverse mass (4 C), and per shot and global
    point 28 C bytes (displacement read by the stiffness; u, v, a read and
    written by the update)."""
    total = 0
    for m, (P, C) in ((0, (3, 2)), (1, (3, 1)), (3, (2, 1))):
        total += static_bytes(info, m, P) + info.nglob[m] * 4 * C
        total += info.nshots * info.nglob[m] * 28 * C
    return total


def event_time(stream, fn):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def sim_stream(sim):
    import ctypes as C
    import torch
    from specfempp_b200 import _capi as A
    ptr = C.c_void_p()
    A.check(A.load().sfb_get_stream(sim.handle, C.byref(ptr)), sim.handle)
    return torch.cuda.ExternalStream(ptr.value)


def e2e_run(sim, stream, steps):
    """End to end through the C ABI with host buffers: upload every source's
    time function from pinned host memory (H2D), run `steps` fused steps,
    read all seismograms back (D2H); device time of the whole sequence and
    the bytes copied per step."""
    import ctypes as C
    import torch
    from specfempp_b200 import _capi as A
    lib = A.load()
    info = sim.info()
    view = sim.problem_view()
    nsrc = view.nsources
    n = info.nstep * 2
    flat = np.ctypeslib.as_array(view.src_stf, shape=(nsrc * n,))
    stf_pinned = [torch.from_numpy(flat[i * n:(i + 1) * n].copy()).pin_memory() for i in range(nsrc)]
    seis = torch.empty((info.nshots, info.max_sig_step, info.nseismogram_types, info.nreceivers, 2),
                       dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(nsrc):
        A.check(lib.sfb_set_source_time_function(sim.handle, i, C.cast(stf_pinned[i].data_ptr(), C.POINTER(C.c_float)),
                                                 stf_pinned[i].numel()), sim.handle)
    sim.run_forward(steps)
    per_shot = seis[0].numel()
    for s in range(info.nshots):
        A.check(lib.sfb_get_seismograms(sim.handle, 0, s, C.cast(seis[s].data_ptr(), C.POINTER(C.c_float)),
                                        per_shot), sim.handle)
    f1.record(stream)
    f1.synchronize()
    h2d = sum(t.numel() * 4 for t in stf_pinned)
    d2h = seis.numel() * 4
    return f0.elapsed_time(f1), h2d / steps, d2h / steps


def batched_forward(steps, cpu_seconds=None):
    """The 64-shot batched forward (800 x 400 elements): device time per step
    and whole-step algorithmic HBM bytes against the measured peak, the same
    run end to end through the C ABI with host buffers, and the oracle's
    per-shot rate on the host cores."""
    import ctypes as C
    from specfempp_b200 import Simulation, _capi as A
    p = make_problem("batched", GRAPH_STEPS + 3 + 3 * steps + 1)
    with Simulation.structured(p) as sim:
        pin_variant(sim)
        sim.initialize()
        stream = sim_stream(sim)
        sim.run_forward(GRAPH_STEPS)
        sim.run_forward(steps)  # set-up: captures the graph of the remainder chunk
        sim.run_forward(3)
        ms = event_time(stream, lambda: sim.run_forward(steps))
        ms_e2e, h2d, d2h = e2e_run(sim, stream, steps)
        info = sim.info()
        mean_ms = C.c_double()
        A.check(A.load().sfb_time_stiffness(sim.handle, 0, 10, C.byref(mean_ms)), sim.handle)
    peak, _ = measured_peak()
    per_step = ms / steps
    b = step_bytes(info)
    updates = info.nshots * sum(info.nglob) * steps
    out = {
        "workload": workload_config("batched", info, p)["workload"],
        "value": updates / (ms / 1000.0), "unit": "GLL-point-updates/s",
        "ms_per_step": per_step, "steps": steps,
        "step_roofline": {"bound": "hbm", "algorithmic_bytes_per_step": b,
                          "achieved": b / (per_step / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": b / (per_step / 1000.0) / 1e9 / peak},
        "stiffness_ms": mean_ms.value,
        "e2e": {"value": updates / (ms_e2e / 1000.0), "unit": "GLL-point-updates/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
    }
    if cpu_seconds:
        threads = os.cpu_count() or 1
        rate, n, dt, _ = cpu_rate("batched", None, threads, budget_s=cpu_seconds)
        out["cpu_baseline"] = {"value": rate, "unit": "GLL-point-updates/s", "cores": threads, "kind": "port",
                               "sample": "shot 0 of the 64, %d full time steps (oracle FP32, OpenMP over "
                                         "elements; shots are independent, so the per-shot rate is the "
                                         "whole job's), %.1f s" % (n, dt)}
    return out


def deterministic_forward(workload, steps):
    """The same forward with the deterministic assembly (element colours,
    fixed-order sums): device time per step, beside the atomic mode's."""
    from specfempp_b200 import Simulation
    p = make_problem(workload, GRAPH_STEPS + 3 + 2 * steps + 1)
    with Simulation.structured(p) as sim:
        sim.set_deterministic(True)
        pin_variant(sim)
        sim.initialize()
        stream = sim_stream(sim)
        sim.run_forward(GRAPH_STEPS)
        sim.run_forward(steps)  # set-up: captures the graph of the remainder chunk
        sim.run_forward(3)
        ms = event_time(stream, lambda: sim.run_forward(steps))
        info = sim.info()
    return {"ms_per_step": ms / steps, "value": info.nshots * sum(info.nglob) * steps / (ms / 1000.0),
            "unit": "GLL-point-updates/s", "steps": steps,
            "stiffness_variant": {name: int(info.stiffness_variant[m])
                                  for name, m in (("elastic_psv", 0), ("elastic_sh", 1), ("acoustic", 3))
                                  if info.nelements[m] > 0}}


def fwi_comparison(nshots=64, nstep=400, reps=2):
    """Forward + combined (adjoint + backward + Frechet kernels) run of the
    200 x 200 adjoint mesh: `nshots` shots batched in one context against one
    shot alone (the plain single-shot path), per-shot device time, same GPU.
    The adjoint sources are seeded synthetic residuals (cost does not depend
    on their values)."""
    from specfempp_b200 import Simulation
    from specfempp_b200 import workloads as W

    def timed(S):
        p = W.adjoint_model(1.0, nshots=S, nstep=nstep)
        p.save_boundary_values = True
        with Simulation.structured(p) as sim:
            pin_variant(sim)
            info = sim.info()
            rng = np.random.default_rng(3)
            for s in range(S):
                sim.set_adjoint_sources((1e-3 * rng.standard_normal((nstep, info.nreceivers, 2))).astype(np.float32),
                                        shot=s)
            stream = sim_stream(sim)
            best = None
            for r in range(reps + 1):  # the first run captures the graphs
                sim.reset()
                ms = event_time(stream, lambda: (sim.run_forward(), sim.run_combined()))
                if r:
                    best = ms if best is None else min(best, ms)
            return best, info

    ms_b, info_b = timed(nshots)
    ms_1, info_1 = timed(1)
    return {
        "workload": "forward + adjoint gradient, 200x200 NGLL=5 elements, 10x10 km, %d receivers, "
                    "%d steps (a slice of the 6000-step run; per-step cost is constant)" % (info_b.nreceivers, nstep),
        "shots": nshots, "batched_ms_per_shot": ms_b / nshots, "single_shot_ms": ms_1,
        "batched_shots_per_s": nshots / (ms_b / 1000.0), "single_shots_per_s": 1.0 / (ms_1 / 1000.0),
        "per_shot_speedup": ms_1 / (ms_b / nshots),
    }


def cpu_rate(workload, nstep_hint, threads, budget_s=15.0, sample_steps=None):
    """GLL point updates/s of the oracle (FP32 CPU restatement) on the host cores."""
    from oracle import bridge
    from specfempp_b200 import Simulation
    probe = 3
    p = make_problem(workload, max(probe, 4))
    sim = Simulation.structured(p)
    t = time.perf_counter()
    bridge.forward(sim, 32, nstep=probe, threads=threads)
    per_step = (time.perf_counter() - t) / probe
    n = sample_steps or max(4, min(5000, int(budget_s / max(per_step, 1e-6))))
    p = make_problem(workload, n)
    sim = Simulation.structured(p)
    info = sim.info()
    t = time.perf_counter()
    bridge.forward(sim, 32, nstep=n, threads=threads)
    dt = time.perf_counter() - t
    updates = sum(info.nglob) * n  # the oracle runs one shot of the workload
    return updates / dt, n, dt, info


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    # warm-up (untimed), then the timed sample: each step is one full time step
    cpu_rate(args.workload, None, threads, sample_steps=max(1, min(args.warmup, 3)))
    steps = max(1, min(args.steps, 200))
    rate, n, dt, info = cpu_rate(args.workload, None, threads, sample_steps=steps)
    line = {
        "impl": "reference", "metric": "GLL pt-updates/s", "value": rate, "unit": "GLL-point-updates/s",
        "n_gpus": args.gpus, "steps": n, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded model with the workload's shapes and distributions)",
        "config": workload_config(args.workload, info, None),
        "cpu_baseline": {"value": rate, "unit": "GLL-point-updates/s", "cores": threads, "kind": "port",
                         "sample": "%d full time steps of the workload (oracle FP32, OpenMP over elements)" % n},
        "e2e": {"value": rate, "unit": "GLL-point-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import ctypes as C
    import torch
    import torch.distributed as dist
    from specfempp_b200 import Simulation, _capi as A

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    K, Wm = args.steps, args.warmup
    nstep_total = GRAPH_STEPS + Wm + 3 * K + 2
    p = make_problem(args.workload, nstep_total)
    sim = Simulation.structured(p)
    pin_variant(sim)
    sim.initialize()
    info = sim.info()
    lib = A.load()
    ptr = C.c_void_p()
    A.check(lib.sfb_get_stream(sim.handle, C.byref(ptr)), sim.handle)
    stream = torch.cuda.ExternalStream(ptr.value)

    # set-up: capture the CUDA graphs of a 25-step chunk and of the remainder
    # chunk of a K-step run (so the timed run is graph-launched for any K),
    # then W warm-up steps
    sim.run_forward(GRAPH_STEPS)
    sim.run_forward(K)
    sim.run_forward(Wm)
    launches0 = sim.info().kernel_launches

    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run_forward(K)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = sim.info().kernel_launches - launches0
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    npts = sum(info.nglob)
    value = world * info.nshots * npts * K / (ms / 1000.0)

    # end to end through the C ABI with host buffers: upload the source time
    # functions (H2D), run K steps, read the seismograms back (D2H)
    if world > 1:
        dist.barrier()
    ms_e2e, h2d, d2h = e2e_run(sim, stream, K)
    if world > 1:
        t = torch.tensor([ms_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = world * info.nshots * npts * K / (ms_e2e / 1000.0)
    view = sim.problem_view()

    # roofline of the dominant kernel (elastic stiffness)
    dominant = 0 if info.nelements[0] > 0 else (3 if info.nelements[3] > 0 else 1)
    mean_ms = C.c_double()
    A.check(lib.sfb_time_stiffness(sim.handle, dominant, 20, C.byref(mean_ms)), sim.handle)
    bytes_launch = stiffness_bytes(info, view, dominant)
    achieved = bytes_launch / (mean_ms.value / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic("stiffness_%s.txt" % args.workload, info.stiffness_variant[dominant])

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    line = {
        "metric": "GLL pt-updates/s", "value": value, "unit": "GLL-point-updates/s", "n_gpus": world,
        "steps": K, "warmup": Wm, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded model with the workload's shapes and distributions)",
        "config": dict(workload_config(args.workload, info, p), scale=SCALE,
                       parallelism="replicas" if world > 1 else "single",
                       l2_policy="working set %.0f MB > 126 MB L2; no flush" % (info.device_bytes / 1e6)),
        "roofline": {"bound": "hbm", "kernel": "stiffness (medium %d)" % dominant, "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": bytes_launch, "mean_launch_ms": mean_ms.value},
        "e2e": {"value": e2e_value, "unit": "GLL-point-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    step_b = step_bytes(info)
    line["step_roofline"] = {"bound": "hbm", "algorithmic_bytes_per_step": step_b,
                             "achieved": step_b / (ms / K / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": step_b / (ms / K / 1000.0) / 1e9 / peak}
    if world == 1 and args.workload == "coupled" and not args.no_secondary:
        sim.close()
        line["deterministic"] = dict(deterministic_forward("coupled", K),
                                     note="bit-reproducible assembly (sfb_set_deterministic) on the same workload")
        line["batched"] = batched_forward(min(K, 100), None if args.no_cpu_baseline else args.cpu_seconds)
        line["batched"]["deterministic"] = deterministic_forward("batched", min(K, 100))
        line["fwi"] = fwi_comparison()
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, dt, _ = cpu_rate(args.workload, None, threads, budget_s=args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "GLL-point-updates/s", "cores": threads, "kind": "port",
                                "sample": "%d full time steps of the workload (oracle FP32, OpenMP over elements), %.1f s" % (n, dt)}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# 3D batched elastic forward (config 5's mesh, model, shots and receivers)
FP32_FLOPS_PER_POINT_SHOT = 250  # stiffness arithmetic per local point and shot (see hex3d_flops)


def hex3d_stiffness_bytes(info):
    """Algorithmic bytes of one 3D stiffness launch: per local point the
    global index, kappa and mu (12 B), per element the geometry (16 B), and
    per global point and shot one read of the displacement and one write
    of the force (2 x 12 B)."""
    return info.nspec * 125 * 12 + info.nspec * 16 + info.nshots * info.nglob * 24


def hex3d_flops(info):
    """FP32 operations of one 3D stiffness launch: per local point and shot
    the three directional derivatives (45 FMA), the strain-stress map and
    F = J T dxi/dx (about 50), the weak divergence (45 FMA) and the weights
    (about 20): 250."""
    return FP32_FLOPS_PER_POINT_SHOT * info.nspec * 125 * info.nshots


def hex3d_step_bytes(info):
    """Algorithmic bytes of one 3D forward step: the stiffness launch, the
    Newmark update (per global point and shot u, v, force read, u, v
    written, force zeroed: 6 x 12 B; the inverse mass 12 B per point) and
    the Stacey points (velocity read, force read and written: 3 x 12 B per
    point and shot, 16 B per point of static data)."""
    return (hex3d_stiffness_bytes(info) + info.nshots * info.nglob * 72 + info.nglob * 12
            + info.nboundary_points * (info.nshots * 36 + 16))


def fp32_peak_tflops():
    """Nominal FP32 FMA throughput of the 148 SMs (128 lanes each) at the
    maximum SM clock (MEASURED_PEAKS.json sm_max_mhz, else 1965 MHz)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f).get("sm_max_mhz", 1965.0))
    except Exception:
        mhz = 1965.0
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


def hex3d_cpu_rate(budget_s, threads):
    """The 3D oracle (FP32, OpenMP over elements) on an eighth of config 5's
    elements per axis (one shot), timed over as many steps as fit in about
    `budget_s` seconds: GLL point updates per second."""
    from oracle import bridge3d
    from specfempp_b200.hex3d import config5_problem
    probe = config5_problem(scale=0.125, nstep=4, nshots=1, nrec=16, save_boundary_values=False)
    t0 = time.perf_counter()
    bridge3d.forward(probe, 0, 32, threads=threads, want_store=False)
    per_step = (time.perf_counter() - t0) / 4
    n = max(4, int(budget_s / max(per_step, 1e-6)))
    p = config5_problem(scale=0.125, nstep=n, nshots=1, nrec=16, save_boundary_values=False)
    t0 = time.perf_counter()
    bridge3d.forward(p, 0, 32, threads=threads, want_store=False)
    dt = time.perf_counter() - t0
    nglob = (4 * p.nx + 1) * (4 * p.ny + 1) * (4 * p.nz + 1)
    return nglob * n / dt, n, dt, (p.nx, p.ny, p.nz)


def run_hex3d(args):
    """3D batched forward: config 5's mesh (96 x 96 x 48 hexahedra at full
    scale), model, 16 shots and 1000 receivers; K forward steps timed with
    CUDA events on the context's stream (sfb3_time_kernel)."""
    import torch
    from specfempp_b200.hex3d import Simulation3D, config5_problem
    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    K, Wm = args.steps, args.warmup
    p = config5_problem(scale=SCALE, nstep=Wm + 2 * K + 1, save_boundary_values=False)
    sim = Simulation3D(p)
    info = sim.info()
    sim.run_forward(Wm)
    launches0 = sim.info().kernel_launches
    sampler = ClockSampler(env_int("LOCAL_RANK", 0))
    torch.cuda.synchronize()
    sampler.start()
    ms = sim.time_kernel(3, K)           # mean per step over K steps
    clocks = sampler.stop()
    launches = sim.info().kernel_launches - launches0
    pts = info.nglob * info.nshots
    value = pts / (ms / 1000.0)
    # end to end through the public API: K steps and every shot's
    # seismograms read back to the host (synchronous calls, wall clock)
    t0 = time.perf_counter()
    sim.run_forward(K)
    seis = [sim.seismograms(shot=s) for s in range(info.nshots)]
    t_e2e = time.perf_counter() - t0
    d2h = sum(a.nbytes for a in seis)
    ms_stiff = sim.time_kernel(0, 5)
    ms_newmark = sim.time_kernel(1, 5)
    sim.close()
    # the deterministic assembly (element colours, fixed-order sums) on the
    # same workload
    pd = config5_problem(scale=SCALE, nstep=Wm + min(K, 20) + 1, save_boundary_values=False, deterministic=True)
    sd = Simulation3D(pd)
    sd.run_forward(Wm)
    ms_det = sd.time_kernel(3, min(K, 20))
    sd.close()
    # the gradient path: forward + combined (adjoint, backward, kernels) of
    # all shots over a slice of the run, adjoint sources = the synthetics
    pa = config5_problem(scale=SCALE, nstep=min(K, 100), save_boundary_values=True)
    sa = Simulation3D(pa)
    ms_fwd = sa.time_kernel(3, pa.nstep)
    for s in range(info.nshots):
        sa.set_adjoint_sources(sa.seismograms(shot=s), shot=s)
    ms_comb = sa.time_kernel(5, 1)
    ia = sa.info()
    sa.close()
    peak, peak_kind = measured_peak()
    b = hex3d_stiffness_bytes(info)
    f = hex3d_flops(info)
    fp32 = fp32_peak_tflops()
    t_mem, t_fp = b / (peak * 1e9), f / (fp32 * 1e12)
    target = max(t_mem, t_fp)
    sb = hex3d_step_bytes(info)
    traffic = profiled_traffic("stiffness_hex3d.txt", "hex3d")
    if traffic is not None:
        traffic *= info.nglob / 28607425.0  # the summary's figure is for the full-size mesh
    line = {
        "metric": "GLL pt-updates/s", "value": value, "unit": "GLL-point-updates/s", "n_gpus": 1,
        "steps": K, "warmup": Wm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded depth-gradient model with a random-field perturbation, random double couples)",
        "config": {"workload": "3D batched elastic forward (config 5 mesh, model, shots, receivers)",
                   "elements": [p.nx, p.ny, p.nz], "ngll": 5, "nglob": info.nglob, "nshots": info.nshots,
                   "nreceivers": info.nreceivers, "scale": SCALE, "dt": p.dt,
                   "l2_policy": "working set %.1f GB > 126 MB L2; no flush" % (info.device_bytes / 1e9)},
        "roofline": {"bound": "hbm" if t_mem >= t_fp else "fp32", "kernel": "k3_stiffness",
                     "achieved": b / (ms_stiff / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": target / (ms_stiff / 1000.0),
                     "frac_definition": "max(bytes / HBM peak, flops / FP32 peak) / measured launch time",
                     "algorithmic_bytes_per_launch": b, "flops_per_launch": f,
                     "fp32_peak_tflops": fp32, "achieved_tflops": f / (ms_stiff / 1000.0) / 1e12,
                     "mean_launch_ms": ms_stiff, "peak_kind": peak_kind, "traffic": traffic},
        "step_roofline": {"bound": "hbm", "algorithmic_bytes_per_step": sb,
                          "achieved": sb / (ms / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": sb / (ms / 1000.0) / 1e9 / peak,
                          "newmark_ms": ms_newmark, "stiffness_ms": ms_stiff},
        "e2e": {"value": pts * K / t_e2e, "unit": "GLL-point-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": d2h / K,
                "note": "K steps + all seismograms to host through sfb3_run_forward / sfb3_get_seismograms"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "deterministic": {"ms_per_step": ms_det, "value": pts / (ms_det / 1000.0), "unit": "GLL-point-updates/s",
                          "steps": min(K, 20), "note": "bit-reproducible assembly (element colours) on the same workload"},
        "adjoint": {"steps": pa.nstep, "forward_ms_per_step": ms_fwd, "combined_ms_per_step": ms_comb,
                    "gradient_ms_per_shot_per_step": (ms_fwd + ms_comb) / info.nshots,
                    "segments": ia.nsegments,
                    "note": "forward then the combined run (adjoint + backward + Frechet kernels) of all "
                            "%d shots, CUDA events" % info.nshots},
    }
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, dt, els = hex3d_cpu_rate(args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": rate, "unit": "GLL-point-updates/s", "cores": threads, "kind": "port",
                                "sample": "%d steps of the 3D oracle (FP32, OpenMP) on %dx%dx%d elements of the "
                                          "same model, one shot, %.1f s" % (n, els[0], els[1], els[2], dt)}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="coupled", choices=["coupled", "plain", "batched", "hex3d"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="length of the timed CPU-baseline sample (about 10-30 s of CPU work)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the batched-forward and batched-vs-single adjoint measurements")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="shrink the workload's element counts (profiling captures); 1 = full size")
    ap.add_argument("--stiffness-variant", type=int, default=0, choices=[0, 1, 2, 3],
                    help="pin the stiffness kernel (sfb_set_stiffness_variant; profiling: the autotuner's "
                         "timings are distorted under a profiler); 0 = autotuned")
    ap.add_argument("--fwi-only", action="store_true",
                    help="only the batched-vs-single forward + adjoint comparison, over --steps time steps")
    args = ap.parse_args()
    global SCALE, VARIANT
    SCALE = args.scale
    VARIANT = args.stiffness_variant
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.workload == "hex3d":
            if env_int("RANK", 0) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no 3D solver "
                                  "(src/specfem3d.cpp stops after reading the mesh)"}), flush=True)
            return 0
        return run_reference(args)
    if args.workload == "hex3d":
        return run_hex3d(args)
    if args.fwi_only:
        import torch
        torch.cuda.set_device(env_int("LOCAL_RANK", 0))
        print(json.dumps(dict(fwi_comparison(nstep=args.steps), steps=args.steps)), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
