"""Session snapshot and restore through the C ABI: a simulation's whole state between steps as
one blob, put back into another simulation of the same grid (or the same one, rewound), steps
on bit for bit as the original; a server evicts a session (snapshot, close) and brings it back
(open, restore) with the same result as never leaving."""
import numpy as np
import pytest

from firepro import abi, scenes
from firepro.engine import FireProError, FireServer, FluidSimulation

pytestmark = pytest.mark.gpu

FIELDS = [abi.FP_FIELD_VELOCITY, abi.FP_FIELD_SCALARS, abi.FP_FIELD_PRESSURE, abi.FP_FIELD_EXPANSION]
TABLES = [abi.FP_TABLE_ENTRIES, abi.FP_TABLE_ACTIVE, abi.FP_TABLE_FREE, abi.FP_TABLE_RECORDS, abi.FP_TABLE_TILES]


def state(sim):
    return ({f: sim.field(f) for f in FIELDS}, {t: sim.table(t) for t in TABLES}, sim.stats().steps)


def same(a, b):
    for f in FIELDS:
        assert np.array_equal(a[0][f], b[0][f]), f"field {f} differs"
    for t in TABLES:
        assert np.array_equal(a[1][t], b[1][t]), f"table {t} differs"
    assert a[2] == b[2]


def _sim(sc, budget, schedule=None):
    sim = FluidSimulation(sc.grid(budget=budget))
    sim.set_runtime(0.05, budget, True)
    if schedule is not None:
        sim.set_schedule(schedule)
        sim.set_solver(4, 0.0)
    return sim


@pytest.mark.parametrize("name", ["plume", "force", "mesh_fcg"])
def test_restore_steps_on_bit_for_bit(name):
    sc, budget, sched = {
        "plume": (scenes.SinglePlume(), 2 ** 19, None),
        "force": (scenes.ForceScene(), 2 ** 20, None),
        "mesh_fcg": (scenes.MeshTargetScene(), 2 ** 20,
                     abi.schedule(abi.FP_SMOOTHER_REDBLACK, 0, 2, 2, 8, abi.FP_KRYLOV_FCG)),
    }[name]
    a = _sim(sc, budget, sched)
    for s in range(12):
        a.step(sc.frame(s).frame)
    blob = a.snapshot()
    for s in range(12, 20):
        a.step(sc.frame(s).frame)
    want = state(a)
    # into another simulation of the same grid
    b = _sim(sc, budget)
    b.step(scenes.EmptyScene().frame(0).frame)  # some unrelated state to overwrite
    b.restore(blob)
    for s in range(12, 20):
        b.step(sc.frame(s).frame)
    same(state(b), want)
    # into the same simulation, rewound
    a.restore(blob)
    for s in range(12, 20):
        a.step(sc.frame(s).frame)
    same(state(a), want)
    a.dispose()
    b.dispose()


def test_restore_refuses_other_grids_and_truncation():
    sc = scenes.SinglePlume()
    a = _sim(sc, 2 ** 19)
    for s in range(3):
        a.step(sc.frame(s).frame)
    blob = a.snapshot()
    g = sc.grid(budget=2 ** 19)
    g.brick_size = 16
    other = FluidSimulation(g)
    with pytest.raises(FireProError, match="another grid"):
        other.restore(blob)
    other.dispose()
    with pytest.raises(FireProError, match="truncated|do not match"):
        a.restore(blob[: len(blob) // 2])
    with pytest.raises(FireProError, match="not a snapshot"):
        a.restore(b"nonsense" * 8)
    before = a.stats().steps
    a.step(sc.frame(3).frame)  # the failed restores changed nothing
    assert a.stats().steps == before + 1
    a.dispose()


def test_server_evicts_and_restores_a_session():
    sc = scenes.SinglePlume(seed=2)
    srv = FireServer(8 << 30)
    sa = srv.open(sc.grid(budget=2 ** 19))
    keep = []
    for s in range(10):
        fd = sc.frame(s)
        keep.append(fd)
        srv.submit(sa, fd.frame)
    srv.drain()
    blob = srv.snapshot(sa)
    srv.close(sa)
    sb = srv.open(sc.grid(budget=2 ** 19))
    import time

    t = time.time()
    while srv.state(sb) != abi.FP_SESSION_LIVE:
        assert time.time() - t < 30
        time.sleep(0.005)
    srv.restore(sb, blob)
    for s in range(10, 16):
        fd = sc.frame(s)
        keep.append(fd)
        srv.submit(sb, fd.frame)
    srv.drain()
    served = {f: srv.field(sb, f) for f in FIELDS}
    srv.dispose()
    plain = _sim(sc, 2 ** 19)
    for s in range(16):
        plain.step(sc.frame(s).frame)
    for f in FIELDS:
        assert np.array_equal(served[f], plain.field(f)), f"field {f}: evicted and restored differs"
    plain.dispose()
