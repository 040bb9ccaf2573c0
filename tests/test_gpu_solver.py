"""The pressure solve's schedules against the FP64 oracle, through the C ABI.

The reference runs one cold-started Jacobi V-cycle a step (PressureSolver.ts:276-365). The
schedules here add a red-black Gauss-Seidel smoother on a chosen number of levels with chosen
sweep counts, and flexible conjugate gradients with one V-cycle as the preconditioner; the
oracle restates each (oracle/fp_oracle.cpp cycleRB, solveFCG). Lockstep parity holds every
step as in test_gpu_parity: tables bit-exact, fields within relative L2 1e-3. The accuracy
test grows the large scene to the benchmark's size and asks the solve for the accuracy gate:
post-projection divergence at most 1e-4 of the velocity.
"""
import numpy as np
import pytest

from firepro import abi, scenes
from firepro.engine import FireProError, FluidSimulation, SimulationBatch
import parity
from test_gpu_parity import check, run

pytestmark = pytest.mark.gpu

RB = abi.FP_SMOOTHER_REDBLACK
FCG = abi.FP_KRYLOV_FCG


def test_redblack_three_levels_parity():
    """The plume's schedule: 3 levels, 2 red-black sweeps before and after, 2 V-cycles."""
    sched = abi.schedule(RB, levels=3, pre=2, post=2, bottom=8)
    check(run(scenes.SinglePlume(), 24, budget=2 ** 19, vcycles=2, schedule=sched), min_active=216)


def test_redblack_all_levels_with_colliders_parity():
    """Every level down to the bottom (the one-CTA red-black bottom), colliders' Neumann
    ghosts in the prolongation, 16^3 bricks' staged levels."""
    sched = abi.schedule(RB, levels=0, pre=2, post=2, bottom=8)
    check(run(scenes.ForceScene(), 12, budget=2 ** 20, vcycles=2, schedule=sched))
    sc = scenes.SinglePlume()
    sc.brick_size = 16
    check(run(sc, 10, budget=2 ** 20, schedule=abi.schedule(RB, levels=4, pre=1, post=1, bottom=4)))


def test_topology_each_step_parity():
    """Every brick's topology rebuilt each step (schedule topology 1) around the colliders of the
    force scene and the large scene, with flexible CG: lockstep with the oracle."""
    sched = abi.schedule(RB, levels=0, pre=2, post=2, bottom=8, krylov=FCG, topology=1)
    check(run(scenes.ForceScene(), 10, budget=2 ** 20, vcycles=6, schedule=sched))
    check(run(scenes.LargeScene(), 40, budget=2 ** 20, vcycles=6, schedule=sched), min_active=100)


@pytest.mark.parametrize("smoother", [abi.FP_SMOOTHER_JACOBI, RB])
def test_fcg_parity(smoother):
    """Flexible CG with the reference V-cycle or a red-black one as preconditioner: 5 V-cycles
    a step (the start and four CG steps) on the force scene and the large scene."""
    sched = abi.schedule(smoother, levels=0, pre=2, post=2, bottom=8, krylov=FCG)
    check(run(scenes.ForceScene(), 10, budget=2 ** 20, vcycles=5, schedule=sched))
    check(run(scenes.LargeScene(), 34, budget=2 ** 20, vcycles=5, schedule=sched), min_active=100)


def test_fcg_meets_the_divergence_gate_at_bench_size():
    """The large scene at the benchmark's budget, grown 180 steps (past 4096 computing bricks):
    flexible CG around the red-black V-cycle, to a relative residual of 1e-6, with every brick's
    topology rebuilt each step (so the solve sees the solids the projection sees), leaves the
    projected velocity's divergence (less the expansion it keeps) at most 1e-4 of the velocity
    every step; the reference's single V-cycle does not."""
    sc = scenes.LargeScene()
    budget = 2 ** 24
    sim = FluidSimulation(sc.grid(budget=budget))
    sim.set_runtime(0.05, budget, True)
    sim.set_schedule(abi.schedule(RB, levels=0, pre=2, post=2, bottom=8, krylov=FCG, topology=1))
    sim.set_solver(16, 1e-6)
    worst, cycles = 0.0, []
    for s in range(190):
        sim.step(sc.frame(s).frame)
        if s >= 176:
            sol = sim.read_solver()
            worst = max(worst, sol.divergence)
            cycles.append(sol.vcycles)
    bricks = sim.stats().active_bricks
    print(f"FCG(red-black): {bricks} bricks, divergence <= {worst:.2e}, V-cycles {cycles}")
    assert bricks >= 4096
    assert 0 <= worst <= 1e-4, worst
    # The reference schedule on the same state leaves far more.
    sim.set_schedule(abi.schedule())
    sim.set_solver(1, 0.0)
    ref = []
    for s in range(190, 193):
        sim.step(sc.frame(s).frame)
        ref.append(sim.read_solver().divergence)
    print(f"reference V-cycle: divergence {ref}")
    sim.dispose()


def test_schedule_validation():
    sim = FluidSimulation(scenes.SinglePlume().grid(budget=2 ** 19))
    for bad, msg in [(abi.schedule(RB, levels=1), "levels must be"), (abi.schedule(RB, pre=0), "pre_sweeps"),
                     (abi.schedule(RB, post=9), "post_sweeps"), (abi.schedule(RB, bottom=0), "bottom_sweeps"),
                     (abi.schedule(smoother=7), "smoother"), (abi.schedule(krylov=3), "krylov"),
                     (abi.schedule(topology=2), "topology")]:
        with pytest.raises(FireProError, match=msg):
            sim.set_schedule(bad)
    sim.dispose()
    batch = SimulationBatch(8)
    sc = scenes.SinglePlume()
    a, b = batch.add(sc.grid(budget=2 ** 19)), batch.add(sc.grid(budget=2 ** 19))
    batch.set_schedule(b, abi.schedule(RB, levels=3, pre=2, post=2, bottom=8))
    fd = sc.frame(0)
    with pytest.raises(FireProError, match="solver schedule differs"):
        batch.step([(a, fd.frame, 1 / 60), (b, fd.frame, 1 / 60)])
    batch.dispose()
