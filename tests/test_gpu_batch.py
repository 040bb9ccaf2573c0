"""Batched stepping through the C ABI: simulations stepped together in one launch give the
same tables and fields, bit for bit, as each stepped alone."""
import numpy as np
import pytest

from firepro import abi, scenes
from firepro.engine import FIXED_DT, FireProError, FluidSimulation, SimulationBatch

pytestmark = pytest.mark.gpu

FIELDS = [abi.FP_FIELD_VELOCITY, abi.FP_FIELD_SCALARS, abi.FP_FIELD_EXPANSION, abi.FP_FIELD_PRESSURE,
          abi.FP_FIELD_DIVERGENCE]
TABLES = [abi.FP_TABLE_ENTRIES, abi.FP_TABLE_PAGES, abi.FP_TABLE_ACTIVITY, abi.FP_TABLE_RECORDS,
          abi.FP_TABLE_FREE, abi.FP_TABLE_ACTIVE, abi.FP_TABLE_SOLIDS, abi.FP_TABLE_TILES]


def members():
    """Uneven simulations: a plume, two large scenes of other seeds and budgets, the force scene
    (colliders, every force kind), and a plume of another voxel size."""
    plume2 = scenes.SinglePlume(seed=5)
    plume2.voxel_size = 0.03
    return [
        (scenes.SinglePlume(seed=1), 2 ** 19),
        (scenes.LargeScene(seed=2), 2 ** 20),
        (scenes.ForceScene(), 2 ** 20),
        (scenes.LargeScene(seed=7, dissipation=0.5), 200 * 512),
        (plume2, 2 ** 18),
    ]


def dts(k):
    return [FIXED_DT, FIXED_DT, 1.0 / 50.0, FIXED_DT, 1.0 / 45.0][k]


def snapshot(get_field, get_table):
    out = {}
    for f in FIELDS:
        out[("f", f)] = get_field(f)
    for t in TABLES:
        out[("t", t)] = get_table(t)
    return out


def assert_same(a, b, label):
    for k in a:
        if k == ("t", abi.FP_TABLE_ACTIVE):
            # the active list is ascending on both sides
            assert np.array_equal(a[k], b[k]), f"{label}: active lists differ"
            continue
        assert a[k].shape == b[k].shape, f"{label}: {k} shapes differ"
        assert np.array_equal(a[k], b[k]), f"{label}: {k} differs in {np.count_nonzero(a[k] != b[k])} values"


def run_alone(scene, budget, steps, dt, schedule=None):
    sim = FluidSimulation(scene.grid(budget=budget))
    sim.set_runtime(0.05, budget, True)
    for s in range(steps):
        if schedule is None or schedule(s):
            fd = scene.frame(s)
            sim.step(fd.frame, dt)
    snap = snapshot(sim.field, sim.table)
    st = sim.stats()
    sim.dispose()
    return snap, st


def test_batch_matches_alone():
    steps = 24
    mem = members()
    batch = SimulationBatch(8)
    ids = []
    for sc, budget in mem:
        i = batch.add(sc.grid(budget=budget))
        batch.set_runtime(i, 0.05, budget, True)
        ids.append(i)
    for s in range(steps):
        fds = [sc.frame(s) for sc, _ in mem]
        batch.step([(ids[k], fds[k].frame, dts(k)) for k in range(len(mem))])
    for k, (sc, budget) in enumerate(mem):
        got = snapshot(lambda f: batch.field(ids[k], f), lambda t: batch.table(ids[k], t))
        want, st = run_alone(sc, budget, steps, dts(k))
        assert st.active_bricks > 0
        assert_same(got, want, f"simulation {k}")
        assert batch.stats(ids[k]).active_bricks == st.active_bricks
    batch.dispose()


def test_batch_subsets_and_churn():
    """Simulations step at different rates, one leaves and a new one takes its id."""
    steps = 16
    a, b, c = scenes.SinglePlume(seed=1), scenes.LargeScene(seed=3), scenes.SinglePlume(seed=9)
    batch = SimulationBatch(8)
    ia = batch.add(a.grid(budget=2 ** 19))
    ib = batch.add(b.grid(budget=2 ** 20))
    for i, bud in ((ia, 2 ** 19), (ib, 2 ** 20)):
        batch.set_runtime(i, 0.05, bud, True)
    na = nb = 0
    ic = None
    nc = 0
    for s in range(steps):
        items = []
        keep = []
        fa = a.frame(na)
        keep.append(fa)
        items.append((ia, fa.frame, FIXED_DT))
        na += 1
        if ib is not None and s % 2 == 0:
            fb = b.frame(nb)
            keep.append(fb)
            items.append((ib, fb.frame, FIXED_DT))
            nb += 1
        if ic is not None:
            fc = c.frame(nc)
            keep.append(fc)
            items.append((ic, fc.frame, FIXED_DT))
            nc += 1
        batch.step(items)
        if s == 9:
            got_b = snapshot(lambda f: batch.field(ib, f), lambda t: batch.table(ib, t))
            batch.remove(ib)
            old = ib
            ib = None
            ic = batch.add(c.grid(budget=2 ** 18))
            batch.set_runtime(ic, 0.05, 2 ** 18, True)
            assert ic == old, "a freed id is reused"
    want_a, _ = run_alone(a, 2 ** 19, na, FIXED_DT)
    want_b, _ = run_alone(b, 2 ** 20, nb, FIXED_DT)
    want_c, _ = run_alone(c, 2 ** 18, nc, FIXED_DT)
    assert_same(snapshot(lambda f: batch.field(ia, f), lambda t: batch.table(ia, t)), want_a, "a")
    assert_same(got_b, want_b, "b")
    assert_same(snapshot(lambda f: batch.field(ic, f), lambda t: batch.table(ic, t)), want_c, "c")
    batch.dispose()


def test_batch_validation_changes_nothing():
    """A bad dt in one simulation fails the whole step before any simulation changes."""
    batch = SimulationBatch(8)
    sc = scenes.SinglePlume()
    i = batch.add(sc.grid(budget=2 ** 18))
    j = batch.add(sc.grid(budget=2 ** 18))
    f0, f1 = sc.frame(0), sc.frame(0)
    batch.step([(i, f0.frame, FIXED_DT), (j, f1.frame, FIXED_DT)])
    with pytest.raises(FireProError) as err:
        batch.step([(i, f0.frame, FIXED_DT), (j, f1.frame, 0.5)])
    assert "simulation 1" in str(err.value) and "(0, 1/30]" in str(err.value)
    assert batch.stats(i).steps == 1 and batch.stats(j).steps == 1
    with pytest.raises(FireProError):
        batch.step([(i, f0.frame, FIXED_DT), (i, f0.frame, FIXED_DT)])
    with pytest.raises(FireProError):
        batch.add(_grid16())  # brick size differs from the batch's
    batch.dispose()


def _grid16():
    g = scenes.SinglePlume().grid(budget=2 ** 18)
    g.brick_size = 16
    return g


def test_reserved_tiles_change_storage_only():
    """A simulation whose tables are reserved for its budget gives the same fields and the same
    tables over the tile slots both hold, and no more tile slots in use."""
    sc = scenes.LargeScene(seed=2)
    budget = 2 ** 20
    want, st = run_alone(sc, budget, 20, FIXED_DT)
    sim = FluidSimulation(sc.grid(budget=budget))
    sim.set_runtime(0.05, budget, True)
    sim.reserve_tiles(4096)
    assert sim.stats().tile_capacity == 4096
    for s in range(20):
        fd = sc.frame(s)
        sim.step(fd.frame)
    got = snapshot(sim.field, sim.table)
    for f in FIELDS:
        assert np.array_equal(got[("f", f)], want[("f", f)])
    cap = st.tile_capacity
    per_id = {abi.FP_TABLE_ENTRIES: 1, abi.FP_TABLE_PAGES: 1, abi.FP_TABLE_RECORDS: 28}
    for t, w in per_id.items():
        a, b = got[("t", t)], want[("t", t)]
        assert np.array_equal(a[: cap * 64 * w], b), f"table {t} differs"
        if t != abi.FP_TABLE_RECORDS:
            assert np.all(a[cap * 64 * w:].view(np.int32) == -1)
    assert np.array_equal(got[("t", abi.FP_TABLE_ACTIVE)], want[("t", abi.FP_TABLE_ACTIVE)])
    assert np.array_equal(got[("t", abi.FP_TABLE_FREE)], want[("t", abi.FP_TABLE_FREE)])
    sim.dispose()
