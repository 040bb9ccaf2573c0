"""Autotuner of the pressure solve's schedule for a batch of simulations.

A batch launch runs one solve schedule for all its simulations (fp_batch_set_schedule). Which
schedule reaches the accuracy gate fastest depends on the simulations' sizes and shapes: the
reference's Jacobi V-cycle needs more cycles than a red-black one, CG around either converges in
fewer, deeper hierarchies pay off on larger grids. The tuner measures instead of guessing:

  1. every simulation of the batch is saved (fp_batch_snapshot);
  2. for each candidate schedule the batch steps a few frames from that state, timed with CUDA
     events on the batch's stream, and each simulation's post-projection divergence is read;
  3. the state is put back (fp_batch_restore) before the next candidate, so every candidate
     starts from the same state and sees the same frames;
  4. the fastest candidate whose worst divergence meets the gate wins (else the most accurate).

Choices are cached by a bucket of the batch's computing bricks (a power of two), so a batch that
grows retunes only when it crosses into a new bucket. No reference counterpart: the reference
runs one fixed V-cycle.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import abi


@dataclass
class Candidate:
    name: str
    schedule: abi.fp_solver_schedule
    vcycles: int
    tolerance: float


def default_candidates() -> list:
    """CG around Jacobi or red-black V-cycles with every brick's topology rebuilt each step (the
    solve then sees the solids the projection sees), fixed V-cycle counts."""
    RB, J, FCG = abi.FP_SMOOTHER_REDBLACK, abi.FP_SMOOTHER_JACOBI, abi.FP_KRYLOV_FCG
    out = []
    for vc in (4, 5, 6, 8):
        out.append(Candidate(f"fcg(rb 2/2/8) x{vc}", abi.schedule(RB, 0, 2, 2, 8, FCG, 1), vc, 0.0))
    for vc in (6, 8):
        out.append(Candidate(f"fcg(jacobi) x{vc}", abi.schedule(J, krylov=FCG, topology=1), vc, 0.0))
    out.append(Candidate("fcg(rb 1/1/4) x8", abi.schedule(RB, 0, 1, 1, 4, FCG, 1), 8, 0.0))
    out.append(Candidate("fcg(rb 4 levels 2/2/16) x6", abi.schedule(RB, 4, 2, 2, 16, FCG, 1), 6, 0.0))
    return out


@dataclass
class Trial:
    name: str
    ms_per_step: float
    worst_divergence: float
    mean_vcycles: float


@dataclass
class Choice:
    candidate: Candidate
    trials: list = field(default_factory=list)


class ScheduleTuner:
    """Tunes and applies the solve schedule of a SimulationBatch."""

    def __init__(self, batch, device: int = 0, candidates=None, divergence: float = 1e-4, steps: int = 3):
        self.batch = batch
        self.device = device
        self.candidates = candidates or default_candidates()
        self.divergence = divergence
        self.steps = steps
        self.cache = {}  # bucket -> Choice

    @staticmethod
    def bucket(bricks: int) -> int:
        return 0 if bricks <= 0 else int(math.log2(bricks))

    def apply(self, ids, candidate: Candidate):
        for i in ids:
            self.batch.set_schedule(i, candidate.schedule)
            self.batch.set_solver(i, candidate.vcycles, candidate.tolerance)

    def tune(self, ids, frames) -> Choice:
        """`frames[k]` is the list of (id, frame, dt) of trial step k (at least `steps` of them).
        Returns the choice, applied to the batch, and caches it by the batch's brick bucket."""
        import torch

        b = self.batch
        bricks = sum(b.stats(i).active_bricks for i in ids)
        key = self.bucket(bricks)
        if key in self.cache:
            self.apply(ids, self.cache[key].candidate)
            return self.cache[key]
        saved = {i: b.snapshot(i) for i in ids}
        stream = torch.cuda.ExternalStream(b.stream(), device=self.device)
        trials = []
        for c in self.candidates:
            self.apply(ids, c)
            b.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            worst, cycles = 0.0, []
            for k in range(self.steps):
                b.step(frames[k])
            ev[1].record(stream)
            b.synchronize()
            for i in ids:
                sol = b.read_solver(i)
                worst = max(worst, sol.divergence if sol.divergence >= 0 else math.inf)
                cycles.append(sol.vcycles)
            trials.append(Trial(c.name, ev[0].elapsed_time(ev[1]) / self.steps, worst, sum(cycles) / len(cycles)))
            for i in ids:
                b.restore(i, saved[i])
        ok = [(t, c) for t, c in zip(trials, self.candidates) if t.worst_divergence <= self.divergence]
        if ok:
            best = min(ok, key=lambda tc: tc[0].ms_per_step)[1]
        else:
            best = min(zip(trials, self.candidates), key=lambda tc: tc[0].worst_divergence)[1]
        choice = Choice(best, trials)
        self.cache[key] = choice
        self.apply(ids, best)
        return choice
