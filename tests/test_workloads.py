"""CPU tests of the serving workload's trace (Poisson arrivals at 20 a second, brick budgets
log-uniform in [32, 8192], lifetimes of 5-60 simulated seconds, the same trace for the same
seed) and of the autotuner's brick-count buckets."""
import math

import numpy as np

from firepro import workloads
from firepro.autotune import ScheduleTuner


def test_serving_trace_statistics():
    rate, duration = 20.0, 200.0
    trace = workloads.serving_trace(seed=1, rate=rate, duration=duration)
    at = np.array([a.at for a in trace])
    bricks = np.array([a.scene.bricks for a in trace])
    steps = np.array([a.steps for a in trace])
    expected = rate * duration
    assert abs(len(trace) - expected) < 4 * math.sqrt(expected)  # a Poisson count
    gaps = np.diff(at)
    assert np.all(gaps > 0) and at[0] > 0 and at[-1] < duration
    # Exponential gaps: mean and standard deviation both 1 / rate.
    assert abs(gaps.mean() * rate - 1.0) < 0.05
    assert abs(gaps.std() * rate - 1.0) < 0.1
    # Log-uniform budgets: equal counts in equal bins of log(bricks).
    assert bricks.min() >= 32 and bricks.max() <= 8192
    u = (np.log(bricks) - math.log(32)) / (math.log(8192) - math.log(32))
    counts = np.histogram(u, bins=5, range=(0.0, 1.0))[0]
    assert np.all(np.abs(counts - len(trace) / 5) < 4 * math.sqrt(len(trace) / 5)), counts
    # Lifetimes of 5-60 s at 60 steps a second, spread over the whole range.
    assert steps.min() >= 300 and steps.max() <= 3600
    assert steps.min() < 400 and steps.max() > 3500


def test_serving_trace_is_seeded():
    a = workloads.serving_trace(seed=3, duration=10.0)
    b = workloads.serving_trace(seed=3, duration=10.0)
    c = workloads.serving_trace(seed=4, duration=10.0)
    key = lambda tr: [(x.at, x.scene.bricks, x.steps, len(x.scene.emitters)) for x in tr]
    assert key(a) == key(b)
    assert key(a) != key(c)
    assert workloads.serving_trace(seed=3, duration=10.0, max_arrivals=7)[-1].at == a[6].at


def test_member_scene_budget_covers_its_bricks():
    for index in range(50):
        s = workloads.scenes.MemberScene(seed=2, index=index, min_bricks=32, max_bricks=8192)
        assert 32 <= s.bricks <= 8192
        assert s.budget == s.bricks * s.brick_size ** 3
        assert 1 <= len(s.emitters) <= 4


def test_autotune_buckets_are_powers_of_two():
    assert ScheduleTuner.bucket(0) == 0 and ScheduleTuner.bucket(1) == 0
    for k in range(1, 20):
        assert ScheduleTuner.bucket(2 ** k) == k
        assert ScheduleTuner.bucket(2 ** k - 1) == k - 1
