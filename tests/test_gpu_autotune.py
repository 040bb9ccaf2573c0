"""The schedule autotuner (firepro/autotune.py) on a batch: every candidate starts from the same
saved state, the state after tuning is the state before it, the choice meets the divergence
gate, and a batch in the same brick bucket reuses the cached choice."""
import numpy as np
import pytest

from firepro import abi, scenes
from firepro.autotune import ScheduleTuner
from firepro.engine import FIXED_DT, SimulationBatch

pytestmark = pytest.mark.gpu


def test_tuner_restores_state_and_meets_the_gate():
    members = [scenes.MemberScene(5, k, 64, 1024) for k in range(6)]
    batch = SimulationBatch(8)
    ids = []
    for m in members:
        i = batch.add(m.grid(budget=m.budget))
        batch.set_runtime(i, 0.05, m.budget, True)
        ids.append(i)
    for s in range(24):
        batch.step([(i, m.frame(s).frame, FIXED_DT) for i, m in zip(ids, members)])
    before = {i: batch.field(i, abi.FP_FIELD_VELOCITY) for i in ids}
    keep = [[m.frame(24 + k) for m in members] for k in range(3)]
    frames = [[(i, fd.frame, FIXED_DT) for i, fd in zip(ids, row)] for row in keep]
    tuner = ScheduleTuner(batch, divergence=1e-4, steps=3)
    choice = tuner.tune(ids, frames)
    print("autotune:", [(t.name, round(t.ms_per_step, 3), f"{t.worst_divergence:.2e}", t.mean_vcycles)
                        for t in choice.trials], "->", choice.candidate.name)
    assert len(choice.trials) == len(tuner.candidates)
    for i in ids:
        assert np.array_equal(batch.field(i, abi.FP_FIELD_VELOCITY), before[i]), "tuning changed the state"
    best = [t for t in choice.trials if t.name == choice.candidate.name][0]
    assert best.worst_divergence <= 1e-4
    # the choice is applied: the next step meets the gate
    batch.step(frames[0])
    assert max(batch.read_solver(i).divergence for i in ids) <= 1e-4
    # same bucket: cached, nothing re-measured
    again = tuner.tune(ids, frames)
    assert again is choice
    batch.dispose()
