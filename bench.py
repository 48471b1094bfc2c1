#!/usr/bin/env python
"""Benchmark of the k-space pseudospectral time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload: hetero3d_256 — 256^3 heterogeneous (12 spheres) nonlinear (B/A 6) power-law
absorbing (alpha 0.75, y 1.5) forward with an additive 1 MPa tone-burst plane source and a full
xy sensor plane recording p and pMax, FP32 on the device. A "step" is one time step of that
simulation; the window is steps W .. W+K-1 (K = 20 by default; --steps 0 times the rest of the
simulation). The metric is grid-point-steps per second over the whole job.

`value`   device throughput: K time steps timed with CUDA events on the library's stream, inputs
          resident in HBM (every field is 67 MB, far above the 126 MB L2 in aggregate).
`e2e`     the same metric through the public C ABI from host buffers: kw_sim_create (host->device
          copies and setup) + K steps + copy-out of p, pMax and pFinal, host wall clock.
`roofline` the dominant pass kernel of a step: algorithmic HBM bytes per launch / mean CUDA-event
          duration per launch, against the measured HBM copy bandwidth of this pool.
`cpu_baseline` the FP64 oracle (a restatement of the reference's update equations; the Swift/MLX
          reference cannot run here) on this host's cores for a bounded sample of the workload.
`batched_over_plain` the 64-simulation uneven 2D batch in one engine against the same simulations
          run one at a time (grid-point-steps/s ratio); `grad_over_forward` the 512^2 adjoint
          gradient time over the forward time of the same simulation. Both are measured in the same
          process after the main window (--no-extras skips them).
--impl reference times the FP64 oracle on the host cores over the same window (W untimed warm-up
          steps, then K timed ones) and prints the same config.
With --gpus N > 1 every rank runs an independent replica (no collective on the data path):
"scaling": "weak", value = all ranks' grid-point-steps / max-over-ranks time. Without torchrun's
environment, --gpus N > 1 relaunches this script under torch.distributed.run with N local ranks.
--profile-step runs one step of the workload after W warm-up steps with every kernel launched on
          its own inside the NVTX range "step" and prints its per-launch profile (the command the
          ncu summaries under profiles/ are taken with).
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "k-wave-swift_b200"))

METRIC = "grid-pt-steps/s"
UNIT = "grid-pt-steps/s"
BATCH = "batch2d_64"
ADJ = "adjoint2d_512"
ADJ3 = "adjoint3d_384"


def measured_peak_gbs() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clk", suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", self.gpu_id], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        time.sleep(0.25)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.remove(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload(name: str):
    from kwave import workloads
    if name == "hetero3d_256":
        return workloads.hetero3d(256)
    if name == "hetero3d_128":
        return workloads.hetero3d(128)
    if name == "ivp2d_128":
        return workloads.ivp2d_128()
    raise SystemExit(f"unknown workload {name}")


def window(args, nt: int) -> tuple[int, int]:
    """(W, K): W untimed warm-up steps, then K timed ones (K = 0 asks for the rest of the run)."""
    W = args.warmup
    K = args.steps if args.steps else nt - W
    if W + K > nt:
        raise SystemExit(f"workload has nt={nt} < warmup+steps={W + K}")
    return W, K


def forward_config(args, b) -> dict:
    """The `config` of both arms for the forward workloads (identical dicts)."""
    hetero = args.workload.startswith("hetero")
    npts = b.grid.totalGridPoints
    return {"workload": args.workload, "grid": list(b.grid.shape), "nt": b.grid.nt,
            "window": "time steps warmup .. warmup+steps-1 of the simulation (source active)" if hetero
            else "time steps warmup .. warmup+steps-1 of the simulation",
            "physics": "heterogeneous c0/rho0, power law y=1.5 with dispersion, B/A=6, additive p source"
            if hetero else "homogeneous IVP",
            "l2": "inputs larger than L2 (every field >= 67 MB)" if npts >= 2 ** 24 else "small grid",
            "parallelism": f"replicas{args.gpus}"}


def cpu_sample(builder, warm: int, steps: int, threads: int) -> dict:
    """Time the FP64 oracle on this host: `warm` untimed steps, then `steps` timed ones."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    _, loop_s = oracle.run(builder, nthreads=threads, max_steps=warm + steps, timed_from=warm)
    n = builder.grid.totalGridPoints
    return {"value": n * steps / loop_s, "unit": UNIT, "cores": threads, "kind": "port",
            "seconds": loop_s, "steps": steps}


# ---------------------------------------------------------------------------------------------
# reference arm: the FP64 oracle (the reference's update equations) on the host cores
# ---------------------------------------------------------------------------------------------
def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload == BATCH:
        return run_reference_batch(args, threads)
    if args.workload in (ADJ, ADJ3):
        return run_reference_adjoint(args, threads)
    b = workload(args.workload)
    W, K = window(args, b.grid.nt)
    r = cpu_sample(b, W, K, threads)
    sample = (f"{args.workload}: time steps {W} .. {W + K - 1} of the workload after {W} untimed warm-up "
              f"steps, FP64 oracle on {threads} threads, time loop only")
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": K, "warmup": W, "ms_per_step": 1e3 * r["seconds"] / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": forward_config(args, b),
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_batch(args, threads: int) -> None:
    """The FP64 oracle on this host over a bounded sample of the batch: the first steps of one
    simulation of each grid size."""
    from kwave import workloads
    builders = workloads.batch2d()
    seen, work, secs = set(), 0.0, 0.0
    steps = max(1, args.steps or 20) * 5
    for b in builders:
        n = b.grid.shape[0]
        if n in seen:
            continue
        seen.add(n)
        r = cpu_sample(b, 0, steps, threads)
        work += b.grid.totalGridPoints * steps
        secs += r["seconds"]
    value = work / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": batch_config(args, builders),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {steps} steps of one simulation per grid size {sorted(seen)}, FP64, "
                                   f"{threads} threads, time loop only"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_adjoint(args, threads: int) -> None:
    """The FP64 oracle adjoint (forward + reverse) on this host over a bounded sample: the first
    steps of the same problem."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from kwave import workloads
    three_d = args.workload == ADJ3
    steps = 2 if three_d else max(2, (args.steps or 20) // 5)
    bp, bt = workloads.adjoint3d(384, steps) if three_d else workloads.adjoint2d(512, steps)
    data, _ = oracle.run(bt, nthreads=threads)
    t0 = time.perf_counter()
    oracle.adjoint(bp, data["p"], nthreads=threads)
    secs = time.perf_counter() - t0
    value = bp.grid.totalGridPoints * steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": 0, "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": adjoint_config(args, bp),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {steps} steps of the {args.workload} problem: FP64 oracle forward + "
                                   f"discrete adjoint, {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
def _gpu_setup():
    import torch

    from kwave import replicas
    from kwave.runtime import Context
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rep = replicas.init("nccl")   # one replica per GPU; no collective on the data path
    ctx = Context(rep.local)
    # a dedicated (non-default) stream shared by the library and the CUDA events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(rep.local).uuid)
    except Exception:
        gpu_id = str(rep.local)
    return rep, ctx, stream, gpu_id


def _event():
    import torch
    return torch.cuda.Event(enable_timing=True)


def batch_config(args, builders) -> dict:
    return {"workload": BATCH, "sims": len(builders), "sizes": sorted({b.grid.shape[0] for b in builders}),
            "grid_pt_steps": float(sum(b.grid.totalGridPoints * b.grid.nt for b in builders)),
            "l2": "small grids (each simulation's fields are L2-resident)", "parallelism": f"replicas{args.gpus}"}


def measure_batch(ctx, stream, rep, W: int, clk=None) -> dict:
    """C3: 64 independent uneven 2D forwards in one engine (one launch per pass and size class, the
    steady step a CUDA graph) against the same 64 run one after another through the
    single-simulation path. Work = sum over simulations of grid points x time steps."""
    import torch

    from kwave import workloads
    builders = workloads.batch2d()
    work = float(sum(b.grid.totalGridPoints * b.grid.nt for b in builders))
    batch = ctx.create_batch(builders)
    batch.step(W)
    batch.reset()
    torch.cuda.synchronize()
    rep.barrier()
    steps = max(b.grid.nt for b in builders)
    e0, e1 = _event(), _event()
    e0.record(stream)
    batch.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_batch = e0.elapsed_time(e1)
    batch.close()
    ms_plain = 0.0
    for b in builders:
        sim = ctx.create_sim(b)
        sim.step(W)
        sim.reset()
        torch.cuda.synchronize()
        a, z = _event(), _event()
        a.record(stream)
        sim.step(b.grid.nt)
        z.record(stream)
        torch.cuda.synchronize()
        ms_plain += a.elapsed_time(z)
        sim.close()
    # end to end through the public API from host buffers: create + run + sensor data, batched
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch = ctx.create_batch(builders)
    batch.run()
    outs = [batch.output(i, "p", b.grid.nt, 256) for i, b in enumerate(builders)]
    t1 = time.perf_counter()
    batch.close()
    ms_batch = rep.max_over_ranks(ms_batch, device="cuda")
    ms_plain = rep.max_over_ranks(ms_plain, device="cuda")
    return {"builders": builders, "work": work, "steps": steps, "ms_batch": ms_batch, "ms_plain": ms_plain,
            "e2e_s": t1 - t0, "h2d": sum(sum(a.nbytes for a in b.keep) for b in builders),
            "d2h": sum(o.nbytes for o in outs if o is not None)}


def adjoint_config(args, bp) -> dict:
    three_d = len(bp.shape) == 3
    nt = bp.grid.nt
    if three_d:
        return {"workload": ADJ3, "grid": list(bp.shape), "nt": nt, "sensor": "128x128 receive plane",
                "physics": "3 layers + 8 spheres, power law y=1.5 with dispersion, B/A=5, focused 32x32 array",
                "l2": "inputs larger than L2", "parallelism": f"replicas{args.gpus}"}
    return {"workload": ADJ, "grid": list(bp.shape), "nt": nt, "sensor": "512-point Cartesian ring",
            "physics": "power law y=1.1 with dispersion, heterogeneous c0, p0",
            "l2": "small grid (fields L2-resident)", "parallelism": f"replicas{args.gpus}"}


def measure_adjoint(ctx, stream, rep, W: int, three_d: bool, adjoint_nt: int = 0, store_all: bool = True) -> dict:
    """C4 / C5: the sound-speed gradient of a sensor-data misfit by the discrete adjoint against the
    forward run of the same simulation."""
    import numpy as np
    import torch

    from kwave import abi, workloads
    if adjoint_nt:   # a shorter run of the same configuration (profiling captures)
        bp, bt = workloads.adjoint3d(384, adjoint_nt) if three_d else workloads.adjoint2d(512, adjoint_nt)
    else:
        bp, bt = workloads.adjoint3d() if three_d else workloads.adjoint2d()
    nt, npts = bp.grid.nt, bp.grid.totalGridPoints
    # observed data: the forward run at the true sound speed
    sim = ctx.create_sim(bt)
    sim.run()
    data = sim.output("p")
    sim.close()
    # forward time of the perturbed model (warm-up, restart, the whole run)
    sim = ctx.create_sim(bp)
    sim.step(W)
    sim.reset()
    torch.cuda.synchronize()
    e0, e1 = _event(), _event()
    e0.record(stream)
    sim.step(nt)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    sim.close()
    if three_d:
        # the checkpoint schedule sized to the free device memory (less room for the simulation's
        # own fields and the adjoint's work fields)
        torch.cuda.empty_cache()
        free, _ = torch.cuda.mem_get_info()
        budget = free - 40 * npts * 4 - (4 << 30)
        opts = dict(policy=abi.KW_CHECKPOINT_BUDGET, memory_budget=float(budget))
    else:
        opts = dict(policy=abi.KW_CHECKPOINT_SQRT)
        ctx.adjoint(bp, data, **opts)   # warm-up of the adjoint path
    t0 = time.perf_counter()
    r = ctx.adjoint(bp, data, **opts)
    e2e_s = time.perf_counter() - t0
    r_all = ctx.adjoint(bp, data, policy=abi.KW_CHECKPOINT_STORE_ALL) if (store_all and not three_d) else None
    grad_ms = r["forward_ms"] + r["reverse_ms"]
    all_ms = r_all["forward_ms"] + r_all["reverse_ms"] if r_all else None
    grad_ms = rep.max_over_ranks(grad_ms, device="cuda")
    fwd_ms = rep.max_over_ranks(fwd_ms, device="cuda")
    g = r["grad_c0"]
    return {"bp": bp, "nt": nt, "npts": npts, "fwd_ms": fwd_ms, "grad_ms": grad_ms, "all_ms": all_ms, "r": r,
            "e2e_s": e2e_s, "grad_c0_l2": float(np.sqrt(np.sum(g.astype(np.float64) ** 2))),
            "h2d": sum(a.nbytes for a in bp.keep) + data.nbytes, "d2h": g.nbytes + npts * 4}


def run_batch(args) -> None:
    rep, ctx, stream, gpu_id = _gpu_setup()
    with ClockSampler(gpu_id) as clk:
        m = measure_batch(ctx, stream, rep, args.warmup)
    if rep.rank == 0:
        world, steps, work = rep.world, m["steps"], m["work"]
        line = {
            "metric": METRIC, "value": work * world / (m["ms_batch"] / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": m["ms_batch"] / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": batch_config(args, m["builders"]),
            "plain": {"value": work * world / (m["ms_plain"] / 1e3), "unit": UNIT, "ms": m["ms_plain"],
                      "what": "the same simulations run one after another through the single-simulation path"},
            "batched_over_plain": m["ms_plain"] / m["ms_batch"],
            "roofline": None, "cpu_baseline": None,
            "e2e": {"value": work * world / m["e2e_s"], "unit": UNIT, "h2d_bytes_per_step": m["h2d"] / steps,
                    "d2h_bytes_per_step": m["d2h"] / steps, "seconds": m["e2e_s"]},
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    rep.close()


def run_adjoint(args) -> None:
    rep, ctx, stream, gpu_id = _gpu_setup()
    three_d = args.workload == ADJ3
    with ClockSampler(gpu_id) as clk:
        m = measure_adjoint(ctx, stream, rep, args.warmup, three_d, args.adjoint_nt)
    if rep.rank == 0:
        world, nt, npts, r = rep.world, m["nt"], m["npts"], m["r"]
        line = {
            "metric": METRIC, "value": npts * nt * world / (m["grad_ms"] / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": nt, "warmup": args.warmup, "ms_per_step": m["grad_ms"] / nt, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": adjoint_config(args, m["bp"]),
            "grad_over_forward": m["grad_ms"] / m["fwd_ms"],
            "forward_ms": m["fwd_ms"],
            "gradient_ms": {"checkpointed_forward": r["forward_ms"], "reverse_sweep": r["reverse_ms"]},
            "checkpointing": {"policy": "memory budget" if three_d else "sqrt(nt)", "interval": r["interval"],
                              "checkpoints": r["checkpoints"]},
            "store_all": {"gradient_ms": m["all_ms"], "grad_over_forward": m["all_ms"] / m["fwd_ms"]}
            if m["all_ms"] else None,
            "misfit": r["misfit"], "grad_c0_l2": m["grad_c0_l2"],
            "roofline": None, "cpu_baseline": None,
            "e2e": {"value": npts * nt * world / m["e2e_s"], "unit": UNIT,
                    "h2d_bytes_per_step": m["h2d"] / nt, "d2h_bytes_per_step": m["d2h"] / nt, "seconds": m["e2e_s"]},
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    rep.close()


def run_profile_step(args) -> None:
    """One time step of the workload after W warm-up steps, every kernel launched on its own inside
    the NVTX range "step" (for ncu --nvtx --nvtx-include "step/"); prints the per-launch CUDA-event
    profile as one JSON line. Not a bench line: nothing here is timed as a metric."""
    import torch
    rep, ctx, stream, gpu_id = _gpu_setup()
    b = workload(args.workload)
    sim = ctx.create_sim(b)
    sim.step(max(args.warmup, 1))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("step")
    prof = sim.profile_step(1)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    sim.close()
    print(json.dumps({"workload": args.workload, "after_steps": max(args.warmup, 1),
                      "launches": [[k["name"], round(k["ms"], 4), k["bytes"]] for k in prof]}))


def run_ours(args) -> None:
    import torch
    rep, ctx, stream, gpu_id = _gpu_setup()
    world, rank = rep.world, rep.rank
    b = workload(args.workload)
    W, K = window(args, b.grid.nt)
    npts = b.grid.totalGridPoints

    sim = ctx.create_sim(b)
    sim.step(W)
    torch.cuda.synchronize()
    rep.barrier()
    torch.cuda.synchronize()
    e0, e1 = _event(), _event()
    with ClockSampler(gpu_id) as clk:
        e0.record(stream)
        sim.step(K)
        e1.record(stream)
        torch.cuda.synchronize()
    rep.barrier()
    torch.cuda.synchronize()
    ms = rep.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    value = npts * K * world / (ms / 1e3)

    # per-launch device profile of a step, taken on a restarted run right after its warm-up steps
    # (the same steps as the window's start; not part of `value`)
    sim.reset()
    sim.step(W)
    prof = sim.profile_step(3)
    launches_per_step = len(prof)
    groups: dict[str, dict] = {}
    for k in prof:
        kern = k["name"].split(":")[0]
        g = groups.setdefault(kern, {"ms": 0.0, "bytes": 0.0, "launches": 0})
        g["ms"] += k["ms"]
        g["bytes"] += k["bytes"]
        g["launches"] += 1
    # the dominant kernel: the single launch of a step with the longest device time
    top = max(prof, key=lambda k: k["ms"])
    peak, peak_kind = measured_peak_gbs()
    achieved = top["bytes"] / (top["ms"] / 1e3) / 1e9 if top["ms"] > 0 else 0.0
    step_bytes = sum(k["bytes"] for k in prof)
    step_ms = sum(k["ms"] for k in prof)
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get(args.workload, {}).get(top["name"])
        except Exception:
            traffic = None
    sim.close()

    # end to end through the public ABI from host buffers (setup + K steps + outputs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim2 = ctx.create_sim(b)
    sim2.step(K)
    outs = {k: sim2.output(k) for k in ("p", "pMax", "pFinal")}
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    h2d = sum(a.nbytes for a in b.keep)
    d2h = sum(v.nbytes for v in outs.values() if v is not None)
    sim2.close()
    e2e_val = npts * K * world / (t1 - t0)

    # the other two ratios of the metric, in the same process (every rank runs them: replicas)
    extras = {}
    if not args.no_extras:
        with ClockSampler(gpu_id) as clk2:
            mb = measure_batch(ctx, stream, rep, W)
            ma = measure_adjoint(ctx, stream, rep, W, three_d=False, store_all=False)
        extras = {
            "batched_over_plain": mb["ms_plain"] / mb["ms_batch"],
            "batched": {"workload": BATCH, "value": mb["work"] * world / (mb["ms_batch"] / 1e3),
                        "plain_value": mb["work"] * world / (mb["ms_plain"] / 1e3), "unit": UNIT,
                        "ms_batch": mb["ms_batch"], "ms_plain": mb["ms_plain"]},
            "grad_over_forward": ma["grad_ms"] / ma["fwd_ms"],
            "adjoint": {"workload": ADJ, "forward_ms": ma["fwd_ms"], "gradient_ms": ma["grad_ms"],
                        "checkpoints": ma["r"]["checkpoints"], "interval": ma["r"]["interval"]},
            "extras_clocks": clk2.summary(),
        }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cw, cs = args.cpu_warmup, args.cpu_steps
        r = cpu_sample(b, cw, cs, threads)
        cpu = {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{args.workload}: time steps {cw} .. {cw + cs - 1} (after {cw} untimed) in FP64 "
                         f"(oracle restatement) on {threads} threads, time loop only ({r['seconds']:.1f} s)"}

    if rank == 0:
        hetero = args.workload.startswith("hetero3d")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": forward_config(args, b),
            "roofline": {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "step_achieved": step_bytes / (ms / K / 1e3) / 1e9,
                         "step_bytes_per_pt": step_bytes / npts,
                         "kernel_share": top["ms"] / step_ms if step_ms else None,
                         # the step against the fixed algorithmic byte model of a maximally fused
                         # 3D nonlinear absorbing step (332 B per grid point and step, source off)
                         "model_bytes_per_pt": 332 if hetero else None,
                         "model_frac": (value / world * 332 / 1e9 / peak) if hetero else None},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
                    "d2h_bytes_per_step": d2h / K, "seconds": t1 - t0,
                    "what": "kw_sim_create from host buffers + `steps` time steps + copy-out of p, pMax, pFinal"},
            "gpu_launches": launches_per_step * K,
            "clocks": clk.summary(),
            "kernels": {k: {"ms": round(v["ms"], 4), "GBps": round(v["bytes"] / (v["ms"] / 1e3) / 1e9, 1) if v["ms"] > 0 else 0,
                            "launches": v["launches"]} for k, v in groups.items()},
            # every launch of one step in issue order: mean event time and algorithmic GB/s
            "step_profile": [[k["name"], round(k["ms"], 4), round(k["bytes"] / (k["ms"] / 1e3) / 1e9, 1) if k["ms"] > 0 else 0]
                             for k in prof],
            **extras,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    rep.close()


def _relaunch_under_torchrun(args) -> int:
    """--gpus N > 1 without torchrun's environment: run this script as N local ranks."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="timed steps (0: the rest of the simulation)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hetero3d_256")
    ap.add_argument("--cpu-warmup", type=int, default=1)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched/plain and gradient/forward ratios")
    ap.add_argument("--profile-step", action="store_true",
                    help="one step of the forward workload, each kernel launched alone in the NVTX range 'step' (for ncu)")
    ap.add_argument("--adjoint-nt", type=int, default=0,
                    help="adjoint workloads: time steps (default: the configuration's; shorter runs for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "0"))
    if args.gpus > 1 and world == 0:
        sys.exit(_relaunch_under_torchrun(args))
    if world and world != args.gpus:
        sys.exit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    if args.profile_step:
        run_profile_step(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == BATCH:
        run_batch(args)
    elif args.workload in (ADJ, ADJ3):
        run_adjoint(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
