"""Serving workloads: seeded session traces and a paced client loop over a serving backend.

A trace is the serving workload of the benchmark: sessions arriving as a Poisson process,
each with a brick budget drawn log-uniform and a lifetime in simulated seconds; while it
lives a session asks for one step every 1/60 s of wall time (a client that waits for its
previous step before asking for the next, so a saturated server slows its clients instead of
queueing without bound). Two backends run it:

  ServerBackend  the serving front end (fp_server_*): continuous batching of every session's
                 requests into one launch, admission by device-memory budget.
  PlainBackend   the plain drop-in: one FluidSimulation per session, each step its own
                 fp_sim_step on the session's own stream, completion seen through a CUDA event.

`run_trace` drives either and reports latency percentiles and voxel-steps/s over a window.
No dataset is involved: every number derives from the trace's seed.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

from . import abi, scenes
from .engine import FIXED_DT, FireServer, FluidSimulation


@dataclass
class Arrival:
    at: float            # seconds after the start of the trace
    scene: scenes.MemberScene
    steps: int           # lifetime in steps at 60 steps per simulated second


def serving_trace(seed: int = 1, rate: float = 20.0, duration: float = 30.0, min_bricks: int = 32,
                  max_bricks: int = 8192, life=(5.0, 60.0), max_arrivals: int = 100000) -> list:
    """Poisson arrivals at `rate` per second for `duration` seconds: member scenes with brick
    budgets log-uniform in [min_bricks, max_bricks], lifetimes uniform in `life` seconds of
    simulated time."""
    out, t, k = [], 0.0, 0
    while k < max_arrivals:
        u = scenes._hash01(k, seed * 7 + 3)
        t += -math.log(max(1e-12, 1.0 - u)) / rate
        if t >= duration:
            break
        life_s = life[0] + (life[1] - life[0]) * scenes._hash01(k, seed * 7 + 5)
        out.append(Arrival(t, scenes.MemberScene(seed, k, min_bricks, max_bricks), int(round(life_s * 60.0))))
        k += 1
    return out


class ServerBackend:
    """Sessions on one FireServer."""

    def __init__(self, precision: int, schedule=None, vcycles: int = 1, tolerance: float = 0.0,
                 memory_budget: int = 150 << 30, max_sessions: int = 256, device: int = 0):
        self.srv = FireServer(memory_budget, max_sessions=max_sessions, device=device)
        if schedule is not None:
            self.srv.set_solver(schedule, vcycles, tolerance)
        self.precision = precision
        self.tickets = {}

    def open(self, scene) -> int:
        return self.srv.open(scene.grid(budget=scene.budget, precision=self.precision))

    def live(self, handle) -> bool:
        return self.srv.state(handle) == abi.FP_SESSION_LIVE

    def submit(self, handle, frame) -> int:
        return self.srv.submit(handle, frame)

    def poll(self):
        """(ticket, done seconds on the backend's clock, latency seconds, active bricks, status)."""
        return [(c.ticket, c.done_ms / 1e3, (c.done_ms - c.submit_ms) / 1e3, c.active_bricks, c.status)
                for c in self.srv.poll()]

    def now(self) -> float:
        return self.srv.stats().elapsed_ms / 1e3

    def close(self, handle):
        self.srv.close(handle)

    def dispose(self):
        self.srv.dispose()


class PlainBackend:
    """One FluidSimulation per session, stepped one call at a time (the plain drop-in)."""

    def __init__(self, precision: int, schedule=None, vcycles: int = 1, tolerance: float = 0.0, device: int = 0):
        import torch

        self.torch = torch
        self.device = device
        self.precision = precision
        self.schedule, self.vcycles, self.tolerance = schedule, vcycles, tolerance
        self.sims = {}
        self.pending = []  # (ticket, event, handle, submitted at)
        self.next_ticket = 1
        self.next_handle = 0
        self.t0 = time.perf_counter()

    def open(self, scene) -> int:
        sim = FluidSimulation(scene.grid(budget=scene.budget, precision=self.precision), device=self.device)
        sim.set_runtime(0.05, scene.budget, True)
        if self.schedule is not None:
            sim.set_schedule(self.schedule)
            sim.set_solver(self.vcycles, self.tolerance)
        h = self.next_handle
        self.next_handle += 1
        stream = self.torch.cuda.ExternalStream(sim.stream(), device=self.device)
        self.sims[h] = (sim, stream)
        return h

    def live(self, handle) -> bool:
        return handle in self.sims

    def submit(self, handle, frame) -> int:
        sim, stream = self.sims[handle]
        sim.step(frame)
        ev = self.torch.cuda.Event()
        ev.record(stream)
        t = self.next_ticket
        self.next_ticket += 1
        self.pending.append((t, ev, handle, self.now()))
        return t

    def poll(self):
        done, keep = [], []
        now = self.now()
        for t, ev, h, at in self.pending:
            if ev.query():
                done.append((t, now, now - at, self.sims[h][0].stats().active_bricks, abi.FP_OK))
            else:
                keep.append((t, ev, h, at))
        self.pending = keep
        return done

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def close(self, handle):
        sim, _ = self.sims.pop(handle)
        sim.dispose()

    def dispose(self):
        for sim, _ in self.sims.values():
            sim.dispose()
        self.sims.clear()


def run_trace(backend, trace, wall: float, hz: float = 60.0, window=(0.5, 1.0), cells: int = 512,
              max_live: int = 256) -> dict:
    """Drive `backend` with `trace` for `wall` seconds: sessions open at their arrival time (or,
    with `max_live` sessions open, as soon as one leaves) and close after their lifetime's
    steps; each live session submits its next step at its next 1/hz tick once its previous step
    completed. Reports, over the completions in the window (fractions of `wall`), latency
    p50/p99 (submission to completion on the backend's clock) and voxel-steps/s, with the live
    sessions and computing bricks seen."""
    start = time.perf_counter()
    t_backend0 = backend.now()
    sessions = {}  # handle -> dict(scene, steps left, step, due, inflight ticket, frame kept)
    arrivals = list(trace)
    submitted = {}  # ticket -> handle
    records = []    # (done time, latency, active bricks)
    live_samples = []
    failures = 0
    while True:
        now = time.perf_counter() - start
        if now >= wall:
            break
        while arrivals and arrivals[0].at <= now and len(sessions) < max_live:
            a = arrivals.pop(0)
            h = backend.open(a.scene)
            sessions[h] = {"scene": a.scene, "left": a.steps, "step": 0, "due": now, "inflight": None, "keep": None}
        for h, s in list(sessions.items()):
            if s["inflight"] is None and s["left"] <= 0:
                backend.close(h)
                del sessions[h]
                continue
            if s["inflight"] is None and s["due"] <= now and backend.live(h):
                fd = s["scene"].frame(s["step"])
                s["keep"] = fd
                t = backend.submit(h, fd.frame)
                submitted[t] = h
                s["inflight"] = t
                s["step"] += 1
                s["left"] -= 1
                s["due"] = max(s["due"] + 1.0 / hz, now)
        for t, done, latency, bricks, status in backend.poll():
            h = submitted.pop(t)
            if status != abi.FP_OK:
                failures += 1
            records.append((done - t_backend0, latency, bricks))
            if h in sessions:
                sessions[h]["inflight"] = None
        live_samples.append(len(sessions))
        time.sleep(0.0005)
    lo, hi = window[0] * wall, window[1] * wall
    sel = [r for r in records if lo <= r[0] < hi]
    lat = sorted(r[1] * 1e3 for r in sel)
    span = hi - lo
    for h in list(sessions):
        backend.close(h)
    return {
        "steps": len(sel),
        "value": sum(r[2] for r in sel) * cells / span if span > 0 else 0.0,
        "latency_p50_ms": lat[len(lat) // 2] if lat else None,
        "latency_p99_ms": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))] if lat else None,
        "mean_live_sessions": sum(live_samples) / max(1, len(live_samples)),
        "mean_active_bricks_per_step": sum(r[2] for r in sel) / max(1, len(sel)),
        "failed_steps": failures,
        "window_s": [lo, hi],
    }


def run_fixed(backend, members, wall: float, hz: float = 60.0, grow: int = 60, cells: int = 512) -> dict:
    """`members` sessions open from the start, grown `grow` steps, then paced at `hz` (each
    waiting for its previous step) for `wall` seconds: latency p50/p99 and voxel-steps/s."""
    handles = [backend.open(m) for m in members]
    t0 = time.perf_counter()
    while not all(backend.live(h) for h in handles):
        if time.perf_counter() - t0 > 60:
            raise RuntimeError("sessions were not admitted")
        time.sleep(0.001)
    keep = []
    pend = set()
    for s in range(grow):
        for h, m in zip(handles, members):
            fd = m.frame(s)
            keep.append(fd)
            pend.add(backend.submit(h, fd.frame))
        while pend:
            for t, *_ in backend.poll():
                pend.discard(t)
        keep.clear()
    out = _paced(backend, handles, members, grow, wall, hz, cells)
    for h in handles:
        backend.close(h)
    return out


def _paced(backend, handles, members, first_step, wall, hz, cells):
    start = time.perf_counter()
    t_backend0 = backend.now()
    state = {h: {"step": first_step, "due": 0.0, "inflight": None, "keep": None} for h in handles}
    submitted = {}
    records = []
    by_handle = dict(zip(handles, members))
    while True:
        now = time.perf_counter() - start
        if now >= wall:
            break
        for h, s in state.items():
            if s["inflight"] is None and s["due"] <= now:
                fd = by_handle[h].frame(s["step"])
                s["keep"] = fd
                t = backend.submit(h, fd.frame)
                submitted[t] = h
                s["inflight"] = t
                s["step"] += 1
                s["due"] = max(s["due"] + 1.0 / hz, now)
        for t, done, latency, bricks, status in backend.poll():
            h = submitted.pop(t)
            records.append((done - t_backend0, latency, bricks))
            state[h]["inflight"] = None
        time.sleep(0.0005)
    # drain what is in flight (not counted)
    t1 = time.perf_counter()
    while submitted and time.perf_counter() - t1 < 30:
        for t, *_ in backend.poll():
            submitted.pop(t, None)
        time.sleep(0.001)
    lo, hi = 0.2 * wall, wall
    sel = [r for r in records if lo <= r[0] < hi]
    lat = sorted(r[1] * 1e3 for r in sel)
    return {
        "steps": len(sel),
        "value": sum(r[2] for r in sel) * cells / (hi - lo),
        "latency_p50_ms": lat[len(lat) // 2] if lat else None,
        "latency_p99_ms": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))] if lat else None,
        "mean_active_bricks_per_step": sum(r[2] for r in sel) / max(1, len(sel)),
    }
