"""The serving front end through the C ABI: admission by memory budget, continuous batching,
and results that are the same alone and among other sessions (bit for bit)."""
import time

import numpy as np
import pytest

from firepro import abi, scenes
from firepro.engine import FIXED_DT, FireProError, FireServer, FluidSimulation, grid_memory_bytes

pytestmark = pytest.mark.gpu

FIELDS = [abi.FP_FIELD_VELOCITY, abi.FP_FIELD_SCALARS, abi.FP_FIELD_PRESSURE]
GB = 1 << 30


def wait_state(server, session, state, timeout=30.0):
    t = time.time()
    while server.state(session) != state:
        assert time.time() - t < timeout, f"session {session} never reached state {state}"
        time.sleep(0.005)


def test_server_alone_and_in_the_mix():
    steps = 12
    a = scenes.SinglePlume(seed=1)
    others = [scenes.MemberScene(4, k) for k in range(5)]
    # alone: the only session
    srv = FireServer(8 * GB)
    sa = srv.open(a.grid(budget=2 ** 19))
    keep = []
    for s in range(steps):
        fd = a.frame(s)
        keep.append(fd)
        srv.submit(sa, fd.frame)
    srv.drain()
    alone = {f: srv.field(sa, f) for f in FIELDS}
    done = []
    while True:
        got = srv.poll()
        if not got:
            break
        done += got
    assert [c.ticket for c in done] == list(range(1, steps + 1))
    assert all(c.status == abi.FP_OK and c.done_ms >= c.submit_ms for c in done)
    srv.dispose()
    # in the mix: other sessions open and submit at their own pace, interleaved
    srv = FireServer(8 * GB)
    ids = [srv.open(m.grid(budget=m.budget)) for m in others]
    sa = srv.open(a.grid(budget=2 ** 19))
    keep = []
    for s in range(steps):
        for k, (i, m) in enumerate(zip(ids, others)):
            if (s + k) % 2 == 0:
                fd = m.frame(s)
                keep.append(fd)
                srv.submit(i, fd.frame)
        fd = a.frame(s)
        keep.append(fd)
        srv.submit(sa, fd.frame)
        if s % 3 == 0:
            time.sleep(0.002)
    srv.drain()
    mixed = {f: srv.field(sa, f) for f in FIELDS}
    st = srv.stats()
    assert st.steps_done >= steps + 5 and st.mean_batch > 1.0
    srv.dispose()
    # and the plain simulation
    sim = FluidSimulation(a.grid(budget=2 ** 19))
    sim.set_runtime(0.05, 2 ** 19, True)
    for s in range(steps):
        fd = a.frame(s)
        sim.step(fd.frame)
    plain = {f: sim.field(f) for f in FIELDS}
    sim.dispose()
    for f in FIELDS:
        assert np.array_equal(alone[f], mixed[f]), f"field {f}: alone and mixed differ"
        assert np.array_equal(alone[f], plain[f]), f"field {f}: served and plain differ"


def test_admission_waits_for_memory():
    a, b = scenes.SinglePlume(seed=1), scenes.SinglePlume(seed=2)
    ga, gb = a.grid(budget=2 ** 19), b.grid(budget=2 ** 19)
    need = grid_memory_bytes(ga)
    srv = FireServer(need + need // 2)  # room for one of the two
    sa = srv.open(ga)
    sb = srv.open(gb)
    wait_state(srv, sa, abi.FP_SESSION_LIVE)
    assert srv.state(sb) == abi.FP_SESSION_WAITING
    keep = [a.frame(0), b.frame(0)]
    srv.submit(sa, keep[0].frame)
    srv.submit(sb, keep[1].frame)  # queued while it waits
    time.sleep(0.2)
    assert srv.state(sb) == abi.FP_SESSION_WAITING
    srv.close(sa)
    wait_state(srv, sb, abi.FP_SESSION_LIVE)
    srv.drain()
    assert srv.state(sa) == abi.FP_SESSION_CLOSED
    st = srv.stats()
    assert st.steps_done == 2 and st.live == 1 and st.waiting == 0
    assert st.memory_bytes == need
    with pytest.raises(FireProError):
        srv.submit(sa, keep[0].frame)
    with pytest.raises(FireProError) as err:
        srv.open(scenes.SinglePlume().grid(budget=2 ** 26))
    assert err.value.code == abi.FP_ELIMIT
    srv.dispose()


def test_session_limit_and_statistics():
    srv = FireServer(16 * GB, max_sessions=2)
    ms = [scenes.MemberScene(2, k) for k in range(3)]
    ids = [srv.open(m.grid(budget=m.budget)) for m in ms]
    wait_state(srv, ids[0], abi.FP_SESSION_LIVE)
    wait_state(srv, ids[1], abi.FP_SESSION_LIVE)
    assert srv.state(ids[2]) == abi.FP_SESSION_WAITING
    keep = []
    for s in range(6):
        for i, m in zip(ids[:2], ms):
            fd = m.frame(s)
            keep.append(fd)
            srv.submit(i, fd.frame)
    srv.drain()
    done = srv.poll()
    assert len(done) == 12
    st = srv.stats()
    assert st.latency_p50_ms > 0 and st.latency_p99_ms >= st.latency_p50_ms
    assert st.voxel_steps == sum(c.active_bricks for c in done) * 512
    for i in ids[:2]:
        tickets = [c.ticket for c in done if c.session == i]
        assert tickets == sorted(tickets) and [c.step for c in done if c.session == i] == list(range(1, 7))
    srv.close(ids[0])
    wait_state(srv, ids[2], abi.FP_SESSION_LIVE)
    srv.dispose()


def _plain_fields(scene, grid, frames):
    sim = FluidSimulation(grid)
    sim.set_runtime(0.05, grid.voxel_budget, True)
    for fd in frames:
        sim.step(fd.frame)
    out = {f: sim.field(f) for f in FIELDS}
    sim.dispose()
    return out


def test_server_copies_mesh_frames():
    """Mesh emission records, mesh target cells and their ranges are copied at submission: the
    caller's arrays are overwritten right after each submit, and the served fields still equal
    fp_sim_step's on the intact frames."""
    import ctypes as C

    scs = [scenes.MeshEmitterScene(), scenes.MeshTargetScene()]
    steps = 8
    srv = FireServer(8 * GB)
    ids = [srv.open(sc.grid(budget=2 ** 20)) for sc in scs]
    for s in range(steps):
        for i, sc in zip(ids, scs):
            fd = sc.frame(s)
            srv.submit(i, fd.frame)
            for a in fd.keep:  # the caller reuses its memory
                C.memset(C.addressof(a), 0xFF, C.sizeof(a))
    srv.drain()
    done = []
    while True:
        got = srv.poll()
        if not got:
            break
        done += got
    assert len(done) == 2 * steps and all(c.status == abi.FP_OK for c in done)
    served = [{f: srv.field(i, f) for f in FIELDS} for i in ids]
    srv.dispose()
    for sc, got in zip(scs, served):
        plain = _plain_fields(sc, sc.grid(budget=2 ** 20), [sc.frame(s) for s in range(steps)])
        for f in FIELDS:
            assert np.array_equal(got[f], plain[f]), f"{sc.name} field {f}: served and plain differ"


def test_server_isolates_an_invalid_frame():
    """One session among eight submits a frame whose flame ramp is invalid: that step alone
    fails, with the reference's message, and the other sessions' fields are bit-identical to
    stepping each alone (a session that raises mid-batch harms no other)."""
    ms = [scenes.MemberScene(3, k, max_bricks=256) for k in range(8)]
    steps, bad_session, bad_step = 6, 3, 2
    srv = FireServer(16 * GB)
    ids = [srv.open(m.grid(budget=m.budget)) for m in ms]
    keep = []
    for s in range(steps):
        for k, (i, m) in enumerate(zip(ids, ms)):
            fd = m.frame(s)
            if k == bad_session and s == bad_step:
                fd.frame.combustion.ramps[2].knots[0][0] = 0.1
            keep.append(fd)
            srv.submit(i, fd.frame)
    srv.drain()
    done = []
    while True:
        got = srv.poll()
        if not got:
            break
        done += got
    failed = [c for c in done if c.status != abi.FP_OK]
    assert len(failed) == 1 and failed[0].session == ids[bad_session]
    assert failed[0].status == abi.FP_EINVAL
    assert "expansion ramp must span lifetime 0–1." in srv.lib.fp_server_last_error(srv.h).decode()
    assert sum(1 for c in done if c.status == abi.FP_OK) == 8 * steps - 1
    served = {i: {f: srv.field(i, f) for f in FIELDS} for i in ids}
    srv.dispose()
    for k, (i, m) in enumerate(zip(ids, ms)):
        frames = [m.frame(s) for s in range(steps) if not (k == bad_session and s == bad_step)]
        plain = _plain_fields(m, m.grid(budget=m.budget), frames)
        for f in FIELDS:
            assert np.array_equal(served[i][f], plain[f]), f"session {k} field {f}: served and alone differ"


def test_server_refuses_another_velocity_divisor():
    srv = FireServer(8 * GB)
    a = scenes.SinglePlume()
    srv.open(a.grid(budget=2 ** 19))
    g = a.grid(budget=2 ** 19)
    g.velocity_divisor = 2
    with pytest.raises(FireProError, match="velocityDivisor 2 differs"):
        srv.open(g)
    srv.dispose()
