#!/usr/bin/env python
"""Benchmark of the sparse-brick simulation step: voxel-steps/s on one B200.

Workload: the large single-simulation scene (three seeded sphere/box emitters, a radial
burst at step 30, turbulence, a sphere and a box collider; 8^3-cell bricks of 2.5 cm), grown
until it holds the target brick count, then stepped K times. A "step" is one full
simulation step: allocation, MacCormack transport, evolution, forces, divergence, one
multigrid V-cycle and projection over every computing brick.

Legs
  value     device time of K steps (CUDA events on the simulation's own stream), inputs
            resident: sum over steps of computing bricks x 512 voxels / time.
  e2e       the same K-step loop through the public C ABI with host frames: each step copies
            its scene and parameters host-to-device and reads its measurement back.
  roofline  per-phase CUDA-event timing (the GpuProfiler analogue) of K more steps; the
            dominant phase's algorithmic bytes per voxel x voxels / its device time.
  cpu_baseline  the oracle's FP32 restatement on the host cores (OpenMP), a bounded sample.

`--impl reference` times the reference algorithm's CPU restatement (the reference itself is
TypeScript/WGSL and cannot run here) on the same scene and metric.
Multi-GPU (torchrun): independent replicas, one per GPU; the timed region is bracketed by
barriers and the time is the max over ranks.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "threejs-fire-pro_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

BRICK_VOXELS = 512
BUDGET = 2 ** 24  # voxels: 32768 slots, ~3.2 GB of pools
TARGET_BRICKS = 4096
MAX_GROW_STEPS = 600
# Steps the large scene grows (untimed) before the warm-up and the timed steps, in every arm:
# past the burst, to about 4.1k computing bricks, then ~4.9k over the timed steps.
GROW_STEPS = 180

# Algorithmic bytes per voxel per phase in FP32: every live field read once and written once
# per kernel that must touch it (velocity 12 B, scalars 16 B, expansion/divergence/pressure
# 4 B). Predictor = advect velocity (24) + advect scalars (44); correct_evolve = correct
# velocity (36) + evolve fields (64); divergence includes the fused first Jacobi iterate's
# write (4); multigrid = (8/7)(12 B x 3 post-sweeps + 9 B restriction + 8.5 B prolongation).
BYTES_PER_VOXEL = {
    "predict": 68.0,
    "correct": 36.0,
    "evolve": 64.0,
    "curl": 28.0,
    "forces": 56.0,
    "divergence": 24.0,
    "multigrid": 8.0 / 7.0 * (12.0 * 3 + 17.5),
    "project": 28.0,
}
STEP_BYTES = sum(BYTES_PER_VOXEL.values())


WORKLOAD = ("large_scene (seed 1): 3 seeded sphere/box emitters, burst at step 30, turbulence 2 m/s, sphere+box "
            "colliders; 8^3 bricks, 2.5 cm voxels, budget 2^24 voxels; grown 180 steps + W warm-up, then K timed; "
            "plain FP32 storage; 1 cold-started V-cycle (reference schedule)")


def workload_config(gpus: int) -> dict:
    """The `config` of both arms: what the workload is, nothing measured (the state it reached
    is reported beside it, under `state`)."""
    return {"workload": WORKLOAD, "grown_steps": GROW_STEPS, "budget_voxels": BUDGET, "brick_size": 8,
            "parallelism": "replicas" if gpus > 1 else "single",
            "l2": "working set > L2: pools of ~4k bricks x 97 KB"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock and throttle-reason samples every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_sample(scene_cls, max_seconds: float, max_steps: int, threads: int, warmup: int = 1):
    """The FP32 oracle on the host cores: voxel-steps/s over a bounded run of the scene, after
    `warmup` untimed steps (the GPU arm's growth and warm-up, so both time the same state)."""
    from oracle import fp_oracle

    fp_oracle.set_threads(threads)
    sc = scene_cls(seed=1)
    o = fp_oracle.OracleSim(sc.grid(budget=BUDGET), real=1)
    o.set_runtime(0.05, BUDGET, True)
    warmup = max(1, warmup)
    for s in range(warmup):
        o.step(sc.frame(s).frame)
    voxels, t0, steps = 0.0, time.perf_counter(), 0
    step_ms = []
    while steps < max_steps and time.perf_counter() - t0 < max_seconds:
        t = time.perf_counter()
        o.step(sc.frame(warmup + steps).frame)
        step_ms.append((time.perf_counter() - t) * 1e3)
        voxels += o.active_bricks * BRICK_VOXELS
        steps += 1
    elapsed = time.perf_counter() - t0
    o.close()
    return voxels / elapsed, steps, voxels / max(steps, 1) / BRICK_VOXELS, step_ms


def percentiles(ms):
    s = sorted(ms)
    if not s:
        return None, None
    return s[len(s) // 2], s[min(len(s) - 1, int(round(0.99 * (len(s) - 1))))]


def run_reference(args, rank, world):
    if rank != 0:
        return
    from firepro import scenes

    threads = os.cpu_count() or 1
    # The GPU arm's workload: the same scene grown the same GROW_STEPS steps and W warm-up
    # steps untimed, then K timed steps (capped at 120 s of CPU time).
    untimed = GROW_STEPS + args.warmup
    value, steps, bricks, step_ms = cpu_sample(scenes.LargeScene, 120.0, args.steps, threads, warmup=untimed)
    p50, p99 = percentiles(step_ms)
    line = {
        "impl": "reference", "metric": "voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": statistics.mean(step_ms) if step_ms else None,
        "p50_ms": p50, "p99_ms": p99, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.gpus),
        "state": {"mean_active_bricks": bricks},
        "cpu_baseline": {"value": value, "unit": "voxel-steps/s", "cores": threads, "kind": "port",
                         "sample": f"oracle FP32 restatement of the step on {threads} threads: the large scene grown "
                                   f"{GROW_STEPS} + {args.warmup} steps untimed, then {steps} timed steps "
                                   f"(mean {bricks:.0f} bricks), capped at 120 s"},
        "e2e": {"value": value, "unit": "voxel-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batched_form(local: int, sims: int = 64, grow: int = 90, steps: int = 60, seed: int = 1) -> dict:
    """The batched workload: `sims` member scenes (brick budgets log-uniform 16-2048, 1-4
    emitters of radius 0.1-0.6 m, rates 0.2-2.0 /s), grown `grow` steps, then `steps` timed
    steps (a) each simulation through its own FluidSimulation, one call after another (the
    plain drop-in; each has its own stream, so their work may overlap on the GPU) and (b) all
    of them through one SimulationBatch (one upload, one graph per step). Both evolve the same
    states bit for bit, so they do the same voxel-steps; wall time of the host loop until the
    GPU is idle, host frames built inside the loop."""
    import torch

    from firepro import scenes
    from firepro.engine import FIXED_DT, FluidSimulation, SimulationBatch, reserved_tiles

    mem = [scenes.MemberScene(seed, k) for k in range(sims)]
    batch = SimulationBatch(8, device=local)
    ids = []
    # Both sides hold tables sized for their budgets, so no step stops to grow them.
    for m in mem:
        i = batch.add(m.grid(budget=m.budget))
        batch.set_runtime(i, 0.05, m.budget, True)
        batch.reserve_tiles(i, reserved_tiles(m.grid(budget=m.budget)))
        ids.append(i)
    plain = []
    for m in mem:
        s = FluidSimulation(m.grid(budget=m.budget), device=local)
        s.set_runtime(0.05, m.budget, True)
        s.reserve_tiles(reserved_tiles(m.grid(budget=m.budget)))
        plain.append(s)
    for st in range(grow):
        fds = [m.frame(st) for m in mem]
        batch.step([(i, fd.frame, FIXED_DT) for i, fd in zip(ids, fds)])
        for s, fd in zip(plain, fds):
            s.step(fd.frame)
    batch.synchronize()
    for s in plain:
        s.synchronize()
    # The frames are the workload's input, built before the timed loops; the voxel-steps come
    # from each simulation's count of bricks stepped, read once before and once after.
    frames = [[m.frame(grow + k) for m in mem] for k in range(steps)]
    stepped_b = lambda: sum(batch.stats(i).bricks_stepped for i in ids)
    stepped_p = lambda: sum(s.stats().bricks_stepped for s in plain)
    # (b) batched: device time on the batch's stream and wall time
    stream = torch.cuda.ExternalStream(batch.stream(), device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    b0 = stepped_b()
    t0 = time.perf_counter()
    ev[0].record(stream)
    for k in range(steps):
        batch.step([(i, fd.frame, FIXED_DT) for i, fd in zip(ids, frames[k])])
        ev[k + 1].record(stream)
    batch.synchronize()
    wall_b = time.perf_counter() - t0
    vox_b = (stepped_b() - b0) * BRICK_VOXELS
    dev_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    # (a) plain: one simulation after another
    p0 = stepped_p()
    t0 = time.perf_counter()
    for k in range(steps):
        for s, fd in zip(plain, frames[k]):
            s.step(fd.frame)
    for s in plain:
        s.synchronize()
    wall_p = time.perf_counter() - t0
    vox_p = (stepped_p() - p0) * BRICK_VOXELS
    same = [s.stats().active_bricks for s in plain] == [batch.stats(i).active_bricks for i in ids] and vox_b == vox_p
    p50, p99 = percentiles(dev_ms)
    out = {
        "workload": f"{sims} member scenes, brick budgets log-uniform 16-2048 (seed {seed}), 1-4 emitters r 0.1-0.6 m, "
                    f"rates 0.2-2.0/s; grown {grow} steps, {steps} timed, frames built before; plain FP32",
        "mean_active_bricks": vox_b / BRICK_VOXELS / steps,
        "batched": {"value": vox_b / wall_b, "device_value": vox_b / (sum(dev_ms) / 1e3), "ms_per_step": 1e3 * wall_b / steps,
                    "device_p50_ms": p50, "device_p99_ms": p99},
        "plain": {"value": vox_p / wall_p, "ms_per_step": 1e3 * wall_p / steps},
        "speedup": wall_p / wall_b,
        "same_final_bricks": same,
        "unit": "voxel-steps/s",
    }
    # The accurate batch: the autotuner picks the solve schedule (FCG or defect correction
    # around Jacobi or red-black V-cycles) that holds post-projection divergence under 1e-4 in
    # the least device time, from the batch's state; then both forms run it for the same steps.
    from firepro.autotune import ScheduleTuner

    k0 = grow + steps
    tframes = [[m.frame(k0 + k) for m in mem] for k in range(3)]
    tuner = ScheduleTuner(batch, device=local, divergence=1e-4, steps=3)
    choice = tuner.tune(ids, [[(i, fd.frame, FIXED_DT) for i, fd in zip(ids, row)] for row in tframes])
    for s in plain:
        s.set_schedule(choice.candidate.schedule)
        s.set_solver(choice.candidate.vcycles, choice.candidate.tolerance)
    acc = min(steps, 20)
    aframes = [[m.frame(k0 + k) for m in mem] for k in range(acc)]
    batch.synchronize()
    b0 = stepped_b()
    t0 = time.perf_counter()
    for k in range(acc):
        batch.step([(i, fd.frame, FIXED_DT) for i, fd in zip(ids, aframes[k])])
    batch.synchronize()
    wall_ab = time.perf_counter() - t0
    vox_ab = (stepped_b() - b0) * BRICK_VOXELS
    worst = max(batch.read_solver(i).divergence for i in ids)
    p0 = stepped_p()
    t0 = time.perf_counter()
    for k in range(acc):
        for s, fd in zip(plain, aframes[k]):
            s.step(fd.frame)
    for s in plain:
        s.synchronize()
    wall_ap = time.perf_counter() - t0
    vox_ap = (stepped_p() - p0) * BRICK_VOXELS
    out["accurate"] = {
        "autotune": {"chosen": choice.candidate.name,
                     "trials": [{"name": t.name, "ms_per_step": t.ms_per_step, "worst_divergence": t.worst_divergence,
                                 "mean_vcycles": t.mean_vcycles} for t in choice.trials]},
        "batched": {"value": vox_ab / wall_ab, "ms_per_step": 1e3 * wall_ab / acc, "worst_divergence_last": worst},
        "plain": {"value": vox_ap / wall_ap, "ms_per_step": 1e3 * wall_ap / acc},
        "speedup": wall_ap / wall_ab,
    }
    batch.dispose()
    for s in plain:
        s.dispose()
    return out


def served_form(local: int, sessions: int = 64, grow: int = 90, ticks: int = 300, seed: int = 1,
                min_bricks: int = 16, max_bricks: int = 2048) -> dict:
    """Serving at `sessions` live sessions: member scenes (brick budgets log-uniform in
    [min_bricks, max_bricks]) opened on one FireServer, grown `grow` steps submitted as fast as
    the server takes them, then `ticks` ticks of a 60 Hz wall clock at which every session
    submits its next step. Latency is submission to completion of the step on the device (the
    server's clock); throughput is the timed steps' voxel-steps over the span from the first
    timed submission to the last completion. Frames are built before the timed loop."""
    from firepro import scenes
    from firepro.engine import FireServer

    mem = [scenes.MemberScene(seed, k, min_bricks, max_bricks) for k in range(sessions)]
    srv = FireServer(150 * (1 << 30), max_sessions=256, device=local)
    ids = [srv.open(m.grid(budget=m.budget)) for m in mem]
    for s in range(grow):
        fds = [m.frame(s) for m in mem]
        for i, fd in zip(ids, fds):
            srv.submit(i, fd.frame)
        srv.drain()
    while srv.poll():
        pass
    frames = [[m.frame(grow + t) for m in mem] for t in range(ticks)]
    first_ticket = None
    t0 = time.perf_counter()
    for t in range(ticks):
        target = t0 + t / 60.0
        delay = target - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        for i, fd in zip(ids, frames[t]):
            k = srv.submit(i, fd.frame)
            if first_ticket is None:
                first_ticket = k
    srv.drain(600000)
    done = []
    while True:
        got = srv.poll()
        if not got:
            break
        done += [c for c in got if c.ticket >= first_ticket]
    st = srv.stats()
    srv.dispose()
    lat = sorted(c.done_ms - c.submit_ms for c in done)
    span_ms = max(c.done_ms for c in done) - min(c.submit_ms for c in done)
    vox = sum(c.active_bricks for c in done) * BRICK_VOXELS
    return {
        "workload": f"{sessions} sessions, member scenes with brick budgets log-uniform {min_bricks}-{max_bricks} "
                    f"(seed {seed}); grown {grow} steps, then {ticks} ticks at 60 Hz, one step request per session "
                    f"per tick; plain FP32",
        "value": vox / (span_ms / 1e3),
        "unit": "voxel-steps/s",
        "latency_p50_ms": lat[len(lat) // 2],
        "latency_p99_ms": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))],
        "mean_active_bricks": sum(c.active_bricks for c in done) / ticks,
        "mean_batch": st.mean_batch,
        "steps": len(done),
    }


# The accurate solve every form that compares at equal accuracy uses: flexible CG around a
# red-black V-cycle on every level (2 + 2 sweeps, 8 at the bottom) with every brick's topology
# rebuilt each step, a fixed number of V-cycles a step: the fewest that hold post-projection
# divergence under 1e-4 of the velocity on the large scene at the benchmark's size, chosen by
# precision_form (which runs first) from CANDIDATE_VCYCLES.
ACCURATE = {"smoother": 1, "levels": 0, "pre": 2, "post": 2, "bottom": 8, "krylov": 1, "topology": 1,
            "vcycles": 6, "tolerance": 0.0}
CANDIDATE_VCYCLES = (4, 5, 6, 8, 10)
DIVERGENCE_GATE = 1e-4


def accurate_schedule():
    from firepro import abi

    a = ACCURATE
    return abi.schedule(a["smoother"], a["levels"], a["pre"], a["post"], a["bottom"], a["krylov"], a["topology"])


def _timed_steps(sim, sc, step, steps, local):
    """Device time of `steps` steps on the simulation's stream, then 10 more read back for the
    solve's accuracy: (ms per step, mean bricks, V-cycles, worst divergence, last residual)."""
    import torch

    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    actives = []
    ev[0].record(stream)
    for k in range(steps):
        sim.step(sc.frame(step + k).frame)
        actives.append(sim.stats().active_bricks)
    ev[1].record(stream)
    sim.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    cycles, div = [], []
    for k in range(10):
        sim.step(sc.frame(step + steps + k).frame)
        sol = sim.read_solver()
        cycles.append(int(sol.vcycles))
        div.append(sol.divergence)
    return ms, sum(actives) / len(actives), cycles, max(div), sol.residual[max(0, sol.vcycles - 1)]


def precision_form(local: int, steps: int = 30) -> dict:
    """The large scene grown GROW_STEPS steps in plain FP32 and saved; from that state each
    candidate V-cycle count of the accurate solve runs 3 + 10 steps and reports its worst
    post-projection divergence (RMS of h (div u - e) / u); the fewest that meet 1e-4 becomes the
    accurate solve of this run. Then, each from the same kind of grown state: FP32 storage and
    FP_PRECISION_MIXED (FP16 scalar state, BF16 coarse multigrid, FP32 finest level and CG) with
    the accurate solve, and the reference's single V-cycle, timed `steps` steps on the
    simulation's stream."""
    from firepro import abi, scenes
    from firepro.engine import FluidSimulation

    out = {"solver": dict(ACCURATE, name="FCG(red-black V-cycle), topology each step")}
    grown = {}
    for name, precision in (("fp32", abi.FP_PRECISION_FP32), ("mixed", abi.FP_PRECISION_MIXED)):
        sc = scenes.LargeScene(seed=1)
        sim = FluidSimulation(sc.grid(budget=BUDGET, precision=precision), device=local)
        sim.set_runtime(0.05, BUDGET, True)
        for step in range(GROW_STEPS):
            sim.step(sc.frame(step).frame)
        grown[name] = (sim, sc, sim.snapshot())
    sim, sc, blob = grown["fp32"]
    calibration = []
    for vc in CANDIDATE_VCYCLES:
        sim.restore(blob)
        sim.set_schedule(accurate_schedule())
        sim.set_solver(vc, 0.0)
        for k in range(3):
            sim.step(sc.frame(GROW_STEPS + k).frame)
        worst = 0.0
        for k in range(10):
            sim.step(sc.frame(GROW_STEPS + 3 + k).frame)
            worst = max(worst, sim.read_solver().divergence)
        calibration.append({"vcycles": vc, "divergence_max": worst})
    ok = [c["vcycles"] for c in calibration if c["divergence_max"] <= DIVERGENCE_GATE]
    ACCURATE["vcycles"] = ok[0] if ok else CANDIDATE_VCYCLES[-1]
    out["solver"]["vcycles"] = ACCURATE["vcycles"]
    out["calibration"] = calibration
    runs = (("fp32", "fp32", True), ("mixed", "mixed", True), ("fp32_reference_vcycle", "fp32", False))
    for name, which, accurate in runs:
        sim, sc, blob = grown[which]
        sim.restore(blob)
        if accurate:
            sim.set_schedule(accurate_schedule())
            sim.set_solver(ACCURATE["vcycles"], ACCURATE["tolerance"])
        else:
            sim.set_schedule(abi.schedule())
            sim.set_solver(1, 1e-30)  # one V-cycle, measured
        step = GROW_STEPS
        for _ in range(3):
            sim.step(sc.frame(step).frame)
            step += 1
        ms, bricks, cycles, worst, residual = _timed_steps(sim, sc, step, steps, local)
        out[name] = {"value": bricks * BRICK_VOXELS / (ms / 1e3), "ms_per_step": ms, "mean_active_bricks": bricks,
                     "vcycles": cycles, "residual_last": residual, "divergence_max": worst,
                     "memory_bytes": sim.stats().memory_bytes}
    for sim, _, _ in grown.values():
        sim.dispose()
    out["speedup_mixed_vs_fp32"] = out["mixed"]["value"] / out["fp32"]["value"]
    out["unit"] = "voxel-steps/s"
    return out


def profile_small_form(local: int, grow: int = 40) -> dict:
    """A small case that runs every kernel family once inside the profiler window (for
    `ncu --profile-from-start off`, one GPU): the force scene (colliders, every force kind) with
    coarse smoke (smoke divisor 2) on 8^3 bricks, budget 2^20 voxels, grown `grow` steps, then
    one step and a half-resolution render at 320x180 inside the window."""
    import torch

    from firepro import render, scenes
    from firepro.engine import FluidSimulation

    sc = scenes.ForceScene()
    grid = sc.grid(budget=2 ** 20)
    grid.smoke_divisor = 2
    sim = FluidSimulation(grid, device=local)
    sim.set_runtime(0.05, 2 ** 20, True)
    for step in range(grow):
        sim.step(sc.frame(step).frame)
    cam = render.look_at((0.0, 1.0, 3.0), (0.0, 0.5, 0.0), 320, 180)
    cam.half_resolution = 1
    rs = render.default_settings(ray_steps=64, shadow_samples=8)
    sim.render(cam, rs)  # the render pools and table, outside the window
    sim.synchronize()
    torch.cuda.profiler.start()
    sim.step(sc.frame(grow).frame)
    image = sim.render(cam, rs)
    sim.synchronize()
    torch.cuda.profiler.stop()
    out = {"workload": f"force scene, 8^3 bricks, smoke divisor 2, budget 2^20 voxels, grown {grow} steps; one step "
                       f"and a 320x180 half-resolution render in the profiler window",
           "active_bricks": int(sim.stats().active_bricks), "covered": float((image[..., 3] > 0.01).mean())}
    sim.dispose()
    return out


def stress_form(local: int, grow: int = 600, steps: int = 20, renders: int = 5) -> dict:
    """The stress workload: the 25 m/s jet scene grown `grow` steps (untimed) at the
    benchmark's budget, its step timed (plain FP32, the 6-level reference V-cycle), and the
    half-resolution camera render at 960x540 with 128 ray steps and 16 shadow samples timed on
    the simulation's stream: ms per render, march samples per second (pixels x ray steps /
    time, an upper bound on the samples the march takes) and the render passes' pool bytes."""
    import numpy as np
    import torch

    from firepro import render, scenes
    from firepro.engine import FluidSimulation

    sc = scenes.StressScene(seed=1)
    sim = FluidSimulation(sc.grid(budget=BUDGET), device=local)
    sim.set_runtime(0.05, BUDGET, True)
    step = 0
    while step < grow:
        sim.step(sc.frame(step).frame)
        step += 1
    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    actives = []
    ev[0].record(stream)
    for _ in range(steps):
        sim.step(sc.frame(step).frame)
        step += 1
        actives.append(sim.stats().active_bricks)
    ev[1].record(stream)
    sim.synchronize()
    step_ms = ev[0].elapsed_time(ev[1]) / steps
    cam = render.look_at((-0.5, 1.2, 3.2), (-0.2, 0.6, 0.0), 960, 540)
    cam.half_resolution = 1
    rs = render.default_settings(ray_steps=128, shadow_samples=16)
    image = torch.empty((540, 960, 4), dtype=torch.float32, device=f"cuda:{local}")
    sim.render_device(cam, rs, image.data_ptr())  # warm-up: pools, table
    sim.synchronize()
    ev[0].record(stream)
    for _ in range(renders):
        sim.render_device(cam, rs, image.data_ptr())
    ev[1].record(stream)
    sim.synchronize()
    render_ms = ev[0].elapsed_time(ev[1]) / renders
    lit = float((image[..., 3] > 0.01).float().mean().item())
    out = {"workload": f"25 m/s jet (box emitter 0.05 m on a wandering path, fuel 1.0, 3 m/s crosswise wind), "
                       f"grown {grow} steps, budget 2^24 voxels; render 960x540 half resolution, 128 ray steps, "
                       f"16 shadow samples, cubic filter",
           "mean_active_bricks": sum(actives) / len(actives), "step_ms": step_ms,
           "value": sum(actives) * BRICK_VOXELS / (step_ms * steps / 1e3), "unit": "voxel-steps/s",
           "render_ms": render_ms, "render_samples_per_s": 960 * 540 * 128 / (render_ms / 1e3),
           "covered_pixel_fraction": lit}
    sim.dispose()
    return out


def default_grid_form(local: int, steps: int = 20) -> dict:
    """The large scene on the reference's default grid (options.ts:460-462: 16^3 bricks,
    velocityDivisor 2, smokeDivisor 2) at the benchmark's budget: grown GROW_STEPS steps
    (untimed), then `steps` steps timed on the simulation's stream, plain FP32, the reference's
    V-cycle. Voxels are field voxels (16^3 a brick)."""
    import torch

    from firepro import scenes
    from firepro.engine import FluidSimulation

    sc = scenes.LargeScene(seed=1)
    sc.brick_size = 16
    sc.velocity_divisor = 2
    grid = sc.grid(budget=BUDGET)
    grid.smoke_divisor = 2
    sim = FluidSimulation(grid, device=local)
    sim.set_runtime(0.05, BUDGET, True)
    step = 0
    while step < GROW_STEPS:
        sim.step(sc.frame(step).frame)
        step += 1
    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    actives = []
    ev[0].record(stream)
    for _ in range(steps):
        sim.step(sc.frame(step).frame)
        step += 1
        actives.append(sim.stats().active_bricks)
    ev[1].record(stream)
    sim.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    # per-phase device time of 10 more steps (fp_sim_set_profiling)
    sim.set_profiling(True)
    for _ in range(10):
        sim.step(sc.frame(step).frame)
        step += 1
    prof = sim.profile()
    sim.set_profiling(False)
    out = {"workload": f"large_scene (seed 1) on 16^3 bricks, velocity divisor 2, smoke divisor 2, 2.5 cm voxels, "
                       f"budget 2^24 voxels; grown {GROW_STEPS} steps, {steps} timed; plain FP32, reference V-cycle",
           "mean_active_bricks": sum(actives) / len(actives), "ms_per_step": ms,
           "value": sum(actives) * 16 ** 3 / (ms * steps / 1e3), "unit": "voxel-steps/s",
           "phases_ms_per_step": {name: t / 10 for name, (n, t, _) in prof.items() if n}}
    sim.dispose()
    return out


def serving_forms(local: int, wall: float = 20.0) -> dict:
    """The serving workload (Poisson arrivals at 20 sessions/s, budgets log-uniform 32-8192
    bricks, lifetimes 5-60 s of simulated time, 60 Hz step requests, at most 256 live sessions,
    150 GB admission cap), every arm with the accurate solve: served + mixed precision, served +
    FP32, and the plain FP32 drop-in (one FluidSimulation per session, one fp_sim_step call
    each). Voxel-steps/s and latency over the second half of `wall` seconds. Then the served +
    mixed capacity sweep: N = 4, 8, 16, ... sessions open from the start (budgets 32-8192), 60 Hz
    each, until p99 passes 16 ms; the capacity is the most voxel-steps/s of a run within it."""
    from firepro import abi, scenes, workloads

    sched, vc, tol = accurate_schedule(), ACCURATE["vcycles"], ACCURATE["tolerance"]
    trace = workloads.serving_trace(seed=1, rate=20.0, duration=wall)
    out = {"workload": f"Poisson arrivals 20/s over {wall:.0f} s ({len(trace)} sessions), budgets log-uniform "
                       f"32-8192 bricks, lifetimes 5-60 s simulated, 60 Hz requests (each after the previous "
                       f"completed), <= 256 live, 150 GB cap; solve FCG(red-black) to 1e-6; window: second half",
           "unit": "voxel-steps/s"}
    arms = (("served_mixed", lambda: workloads.ServerBackend(abi.FP_PRECISION_MIXED, sched, vc, tol, device=local)),
            ("served_fp32", lambda: workloads.ServerBackend(abi.FP_PRECISION_FP32, sched, vc, tol, device=local)),
            ("plain_fp32", lambda: workloads.PlainBackend(abi.FP_PRECISION_FP32, sched, vc, tol, device=local)))
    for name, make in arms:
        be = make()
        out[name] = workloads.run_trace(be, trace, wall)
        be.dispose()
    out["ratio_served_mixed_vs_plain_fp32"] = out["served_mixed"]["value"] / max(1.0, out["plain_fp32"]["value"])
    sweep = []
    for n in (4, 8, 16, 32, 64, 128, 256):
        be = workloads.ServerBackend(abi.FP_PRECISION_MIXED, sched, vc, tol, device=local)
        members = [scenes.MemberScene(2, k, 32, 8192) for k in range(n)]
        r = workloads.run_fixed(be, members, wall=6.0, grow=30)
        be.dispose()
        r["sessions"] = n
        sweep.append(r)
        if r["latency_p99_ms"] is not None and r["latency_p99_ms"] > 16.0:
            break
    ok = [r for r in sweep if r["latency_p99_ms"] is not None and r["latency_p99_ms"] <= 16.0]
    best = max(ok, key=lambda r: r["value"], default=None)
    out["capacity_sweep"] = {"runs": sweep, "capacity_value": best["value"] if best else None,
                             "capacity_sessions": best["sessions"] if best else None}
    return out


FORM_ORDER = ("served_64", "precision", "batched", "stress", "default_grid", "serving")


def run_forms(args) -> dict:
    """Every form in a process of its own (`--form NAME`), so that no form runs in the state an
    earlier one left. The 64-session served form runs first: it keeps the GPU near saturation
    (one launch after another at a 60 Hz request clock), so a few per cent of throughput lost
    after a long batched form (plausibly to the heat it leaves) decides whether its queue drains
    (p99 11 ms measured first, 30-70 ms right after the batched form). The precision form's
    V-cycle calibration of the accurate solve is handed to the forms that use that solve."""
    out = {}
    for name in FORM_ORDER:
        cmd = [sys.executable, str(ROOT / "bench.py"), "--form", name, "--steps", str(args.steps),
               "--accurate-vcycles", str(ACCURATE["vcycles"])]
        r = subprocess.run(cmd, capture_output=True, text=True)
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not lines:
            out[name] = {"error": (r.stderr or r.stdout)[-2000:]}
            continue
        d = json.loads(lines[-1])
        d.pop("form", None)
        out[name] = d
        if name == "precision":
            ACCURATE["vcycles"] = int(d["solver"]["vcycles"])
    return out


def run_ours(args, rank, world, local):
    import torch

    from firepro import scenes
    from firepro.engine import FluidSimulation

    torch.cuda.set_device(local)
    sc = scenes.SCENES[args.scene](seed=1)
    sim = FluidSimulation(sc.grid(budget=BUDGET), device=local)
    sim.set_runtime(0.05, BUDGET, True)
    # Grow the scene (untimed): GROW_STEPS steps, as the reference arm does.
    step = 0
    while step < GROW_STEPS:
        sim.step(sc.frame(step).frame)
        step += 1
    for _ in range(args.warmup):
        sim.step(sc.frame(step).frame)
        step += 1
    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    frames = [sc.frame(step + k) for k in range(args.steps)]

    # --- value: device time of K steps on the simulation's stream
    events = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    st0 = sim.stats()
    launches0 = st0.kernel_launches
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    actives = []
    torch.cuda.profiler.start()  # marks the timed window for `ncu --profile-from-start off`
    events[0].record(stream)
    for k, fd in enumerate(frames):
        sim.step(fd.frame)
        events[k + 1].record(stream)
        actives.append(sim.stats().active_bricks)
    sim.synchronize()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    clock = clocks.stop()
    barrier(world)
    step += args.steps
    st1 = sim.stats()
    launches = st1.kernel_launches - launches0
    host = {"prepare_ms_per_step": (st1.host_prepare_ms - st0.host_prepare_ms) / args.steps,
            "wait_ms_per_step": (st1.host_wait_ms - st0.host_wait_ms) / args.steps}
    total_ms = events[0].elapsed_time(events[-1])
    step_ms = [events[k].elapsed_time(events[k + 1]) for k in range(args.steps)]
    voxels = sum(actives) * BRICK_VOXELS
    total_ms_max = max_over_ranks(total_ms, world)
    voxels_all = sum_over_ranks(voxels, world)
    value = voxels_all / (total_ms_max / 1e3)

    # --- roofline: per-phase device time over K more steps
    sim.set_profiling(True)
    for k in range(args.steps):
        sim.step(sc.frame(step + k).frame)
    step += args.steps
    prof = sim.profile()
    sim.set_profiling(False)
    peak, peak_kind = measured_peaks()
    phases = {}
    for name, (n, ms, vox) in prof.items():
        if n == 0:
            continue
        per = BYTES_PER_VOXEL.get(name)
        phases[name] = {"launches": int(n), "ms": ms, "share": None,
                        "gbs": (per * vox / (ms / 1e3) / 1e9) if per and ms > 0 else None}
    total_prof = sum(p["ms"] for p in phases.values())
    for p in phases.values():
        p["share"] = p["ms"] / total_prof if total_prof else None
    # The dominant kernel: the longest phase that is one kernel (the multigrid phase is ~30
    # launches of several kernels and is reported beside it).
    dominant = max((k for k in phases if k != "multigrid"), key=lambda k: phases[k]["ms"])
    dom = phases[dominant]
    achieved = dom["gbs"]
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": None,
                "peak_kind": peak_kind, "bytes_per_voxel": BYTES_PER_VOXEL.get(dominant),
                "step_gbs": STEP_BYTES * voxels / (total_ms / 1e3) / 1e9, "phases": phases}
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        t = json.loads(traffic_file.read_text()).get(dominant)
        if t:
            # DRAM bytes per voxel from the committed ncu capture, scaled to a launch here.
            roofline["traffic"] = t["dram_bytes_per_voxel"] * (dom["launches"] and prof[dominant][2] / dom["launches"])

    # --- e2e: the public C ABI with host frames, wall clock, measurement read each step
    h2d, d2h, e2e_vox = 0, 0, 0.0
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for k in range(args.steps):
        fd = sc.frame(step + k)  # host buffers built this step
        sim.step(fd.frame)
        st = sim.stats()  # device-to-host read of the step's measurement
        e2e_vox += st.active_bricks * BRICK_VOXELS
        h2d += st.h2d_bytes
        d2h += st.d2h_bytes
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_vox = sum_over_ranks(e2e_vox, world)
    step += args.steps
    sim.dispose()

    if rank != 0:
        return
    p50, p99 = percentiles(step_ms)
    line = {
        "metric": "voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "p50_ms": p50, "p99_ms": p99,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(world),
        "state": {"mean_active_bricks": sum(actives) / len(actives), "live_tiles": int(st.tiles),
                  "tile_capacity": int(st.tile_capacity)},
        "roofline": roofline,
        "e2e": {"value": e2e_vox / e2e_s, "unit": "voxel-steps/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": int(launches),
        "host": host,
        "clocks": clock,
    }
    if world == 1 and not args.no_forms:
        line["forms"] = run_forms(args)
    if world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        untimed = GROW_STEPS + args.warmup
        cv, csteps, cbricks, _ = cpu_sample(scenes.LargeScene, 20.0, args.steps, threads, warmup=untimed)
        line["cpu_baseline"] = {"value": cv, "unit": "voxel-steps/s", "cores": threads, "kind": "port",
                                "sample": f"oracle FP32 restatement on {threads} threads: the large scene grown "
                                          f"{GROW_STEPS} + {args.warmup} steps untimed (as this arm), then {csteps} "
                                          f"timed steps (mean {cbricks:.0f} bricks), capped at 20 s"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and served workloads")
    ap.add_argument("--scene", default="large_scene", help="workload (default: the large single simulation)")
    ap.add_argument("--form", default=None, choices=["batched", "served_64", "precision", "stress", "default_grid",
                                                       "serving", "profile_small"],
                    help="run one of the forms alone on GPU 0 and print its JSON")
    ap.add_argument("--accurate-vcycles", type=int, default=None,
                    help="the accurate solve's V-cycles a step (the precision form calibrates them)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.accurate_vcycles:
        ACCURATE["vcycles"] = args.accurate_vcycles
    if args.form:
        forms = {"batched": lambda: batched_form(0, steps=max(10, min(args.steps, 60))), "served_64": lambda: served_form(0),
                 "precision": lambda: precision_form(0), "stress": lambda: stress_form(0),
                 "default_grid": lambda: default_grid_form(0), "serving": lambda: serving_forms(0),
                 "profile_small": lambda: profile_small_form(0)}
        print(json.dumps({"form": args.form, **forms[args.form]()}), flush=True)
        return
    rank, world, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
