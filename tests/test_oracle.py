"""CPU tests of the oracle: numeric helpers pinned to numpy, allocation invariants, pool
exhaustion, the reference's validation messages, tile lifecycle, determinism, projection, and
invariance of the whole step under a translation by one tile."""
import ctypes as C

import numpy as np
import pytest

from firepro import abi, scenes
from oracle.fp_oracle import OracleSim
import parity

BUDGET = 2 ** 19


def _sim(scene, real=1, budget=BUDGET, cutoff=0.05, ground=True, **grid):
    o = OracleSim(scene.grid(budget=budget, **grid), real=real)
    o.set_runtime(cutoff, budget, ground)
    return o


def test_round_f16_matches_numpy(oracle_lib):
    L = oracle_lib
    L.or_round_f16.restype = C.c_double
    L.or_round_f16.argtypes = [C.c_double]
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.normal(0, 10, 2000), rng.normal(0, 1e-5, 500), [0.0, 65504.0, 1e-8, -3.1e-7, 2049.0, 2051.0]])
    for x in xs.astype(np.float32):
        assert L.or_round_f16(float(x)) == float(np.float16(x)), x


def test_round_bf16_and_truncate(oracle_lib):
    L = oracle_lib
    for fn in (L.or_round_bf16, L.or_truncate_half):
        fn.restype = C.c_double
        fn.argtypes = [C.c_double]
    rng = np.random.default_rng(1)
    for x in rng.normal(0, 5, 500).astype(np.float32):
        u = np.array([x], np.float32).view(np.uint32)[0]
        rounded = ((int(u) + 0x7FFF + ((int(u) >> 16) & 1)) & 0xFFFF0000)
        assert L.or_round_bf16(float(x)) == float(np.array([rounded], np.uint32).view(np.float32)[0])
        t = L.or_truncate_half(float(x))
        # Toward zero with ten mantissa bits: |t| <= |x| and within one half ulp.
        assert abs(t) <= abs(x) and abs(x - t) <= abs(x) * 2 ** -10
        assert float(np.float16(t)) == t


def test_plume_allocation_invariants(oracle_lib):
    o = _sim(scenes.SinglePlume())
    sc = scenes.SinglePlume()
    for s in range(3):
        o.step(sc.frame(s).frame)
    entries = o.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    pages = o.table(abi.FP_TABLE_PAGES).view(np.int32)
    active = o.table(abi.FP_TABLE_ACTIVE)
    free = o.table(abi.FP_TABLE_FREE)
    n = int(active[0])
    ids = active[1:1 + n]
    # The starting block is exactly 6x6x6 bricks.
    assert n == 216
    assert np.all(np.diff(ids.astype(np.int64)) > 0), "computing bricks are listed in ascending id order"
    slots = pages[ids]
    assert np.all(slots >= 0) and len(np.unique(slots)) == n, "each computing brick owns a distinct slot"
    assert np.all((entries[ids] & 0xFFFFFF) == slots)
    assert np.all(entries[pages < 0] == -1)
    # Every slot is either on the free stack or owned.
    assert int(free[0]) + n == o.slots
    stack = free[2:2 + int(free[0])]
    assert len(np.intersect1d(stack, slots)) == 0
    # Slots are handed out lowest first.
    assert sorted(slots.tolist()) == list(range(n))


def test_plume_first_step_fresh_flags(oracle_lib):
    o = _sim(scenes.SinglePlume())
    sc = scenes.SinglePlume()
    o.step(sc.frame(0).frame)
    e = o.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    live = e[e >= 0]
    assert np.all(live & 0x2000000), "slots granted this step are fresh"
    o.step(sc.frame(1).frame)
    e = o.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    assert not np.any(e[e >= 0] & 0x2000000), "kept slots are not fresh"


def test_records_match_entries(oracle_lib):
    sc = scenes.SinglePlume()
    o = _sim(sc)
    for s in range(2):
        o.step(sc.frame(s).frame)
    e = o.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    rec = o.table(abi.FP_TABLE_RECORDS).view(np.int32).reshape(-1, 28)
    tiles = o.table(abi.FP_TABLE_TILES).view(np.int32).reshape(-1, 4)
    coord = {}
    for t, (x, y, z, st) in enumerate(tiles):
        if st:
            coord[(x, y, z)] = t

    def brick_id(b):
        t = coord.get((b[0] >> 2, b[1] >> 2, b[2] >> 2))
        return -1 if t is None else t * 64 + ((b[2] & 3) * 4 + (b[1] & 3)) * 4 + (b[0] & 3)

    for bid in np.nonzero(e >= 0)[0][:50]:
        t, l = bid // 64, bid % 64
        x, y, z, _ = tiles[t]
        b = (x * 4 + (l & 3), y * 4 + ((l >> 2) & 3), z * 4 + (l >> 4))
        for k in range(27):
            d = (k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1)
            nb = brick_id((b[0] + d[0], b[1] + d[1], b[2] + d[2]))
            assert rec[bid, k] == (e[nb] if nb >= 0 else -1)


def test_step_validation_messages(oracle_lib):
    sc = scenes.SinglePlume()
    o = _sim(sc)
    fd = sc.frame(0)
    for dt in (0.0, -1.0, 1 / 29, float("nan")):
        with pytest.raises(ValueError, match=r"Simulation step must be in \(0, 1/30\]"):
            o.step(fd.frame, dt)
    fd.frame.combustion.ramps[0].count = 1
    with pytest.raises(ValueError, match="smoke ramp needs 2–8 knots"):
        o.step(fd.frame)
    fd = sc.frame(0)
    fd.frame.combustion.ramps[1].knots[1][0] = 1.5
    with pytest.raises(ValueError, match="heat knots must increase in f32 with coordinates in \\[0,1\\]"):
        o.step(fd.frame)
    fd = sc.frame(0)
    fd.frame.combustion.lifespan = 0.0
    with pytest.raises(ValueError, match="Flame timestep and lifespan must be positive in f32"):
        o.step(fd.frame)


def test_empty_scene_holds_nothing(oracle_lib):
    sc = scenes.EmptyScene()
    o = _sim(sc)
    for s in range(3):
        o.step(sc.frame(s).frame)
    assert o.active_bricks == 0
    assert o.info(8) == 0, "no tile without a source or content"


@pytest.mark.parametrize("slots", [100, 150])
def test_pool_exhaustion_conserves_demand(oracle_lib, slots):
    # The plume's starting block wants 216 bricks; a budget of fewer slots grants every slot,
    # counts the rest as failures and flags the pool as limited (poolLimited), step after step.
    sc = scenes.SinglePlume()
    o = _sim(sc, budget=slots * 512)
    for s in range(3):
        o.step(sc.frame(s).frame)
        assert o.slots == slots and o.info(5) == slots, "every slot granted"
        assert o.active_bricks == slots
        assert o.info(5) + o.info(7) == 216, "granted + failed = wanted"
        assert o.info(6) == 1
    free = o.table(abi.FP_TABLE_FREE)
    assert free[0] == 0 and free[1] == 216 - slots, "an empty free stack and the failure count"
    active = o.table(abi.FP_TABLE_ACTIVE)
    pages = o.table(abi.FP_TABLE_PAGES).view(np.int32)
    ids = active[1:1 + int(active[0])]
    assert np.array_equal(np.sort(pages[ids]), np.arange(slots)), "each slot held by one computing brick"


def test_deterministic(oracle_lib):
    sc = scenes.SinglePlume()
    a, b = _sim(sc), _sim(sc)
    for s in range(4):
        a.step(sc.frame(s).frame)
        b.step(sc.frame(s).frame)
    assert np.array_equal(a.field(abi.FP_FIELD_VELOCITY), b.field(abi.FP_FIELD_VELOCITY))
    assert np.array_equal(a.field(abi.FP_FIELD_SCALARS), b.field(abi.FP_FIELD_SCALARS))


def test_fp32_tracks_fp64(oracle_lib):
    sc = scenes.SinglePlume()
    a, b = _sim(sc, real=0), _sim(sc, real=1)
    for s in range(5):
        a.step(sc.frame(s).frame)
        b.step(sc.frame(s).frame)
    for fid in (abi.FP_FIELD_VELOCITY, abi.FP_FIELD_SCALARS):
        x, y = a.field(fid, f64=True), b.field(fid)
        assert np.linalg.norm(x - y) <= 1e-5 * np.linalg.norm(x)


def test_tiles_linger_then_close(oracle_lib):
    """A source that stops leaves its tiles for LINGER_STEPS (60), then they close and go."""
    class Burst(scenes.Scene):
        def frame(self, step):
            src = [scenes.source(1, "sphere", (0, 0.5, 0), (0.1, 0.1, 0.1))] if step == 0 else []
            return scenes.make_frame(scenes.settings(), scenes.combustion(), False, src)

    sc = Burst()
    o = _sim(sc)
    o.step(sc.frame(0).frame)
    tiles0 = o.info(8)
    assert tiles0 > 0
    for s in range(1, 62):
        o.step(sc.frame(s).frame)
    assert o.info(8) == tiles0, "tiles linger 60 steps"
    o.step(sc.frame(62).frame)
    states = o.table(abi.FP_TABLE_TILES).view(np.int32).reshape(-1, 4)[:, 3]
    assert np.all(states[states != 0] == 2), "then close"
    o.step(sc.frame(63).frame)
    assert o.info(8) == 0, "and are removed a step later"


def test_projection_reduces_divergence(oracle_lib):
    sc = scenes.SinglePlume()
    o = _sim(sc, real=0)
    for s in range(40):
        o.step(sc.frame(s).frame)
    div = o.field(abi.FP_FIELD_DIVERGENCE, f64=True)  # h^2 (div u - expansion) before projection
    v = o.field(abi.FP_FIELD_VELOCITY, f64=True)
    e = o.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    slots = np.unique(e[e >= 0] & 0xFFFFFF)
    # Interior divergence of the projected velocity within each brick.
    B = 8
    u = v[slots].reshape(len(slots), 3, B, B, B)  # [s, c, z, y, x]
    d = (u[:, 0, 1:, 1:, 1:] - u[:, 0, 1:, 1:, :-1]) + (u[:, 1, 1:, 1:, 1:] - u[:, 1, 1:, :-1, 1:]) + \
        (u[:, 2, 1:, 1:, 1:] - u[:, 2, :-1, 1:, 1:])
    h = 0.025
    expn = o.field(abi.FP_FIELD_EXPANSION, f64=True)[slots].reshape(len(slots), B, B, B)[:, 1:, 1:, 1:]
    after = np.linalg.norm(d / h - expn)
    before = np.linalg.norm(div[slots].reshape(len(slots), B, B, B)[:, 1:, 1:, 1:]) / h ** 2
    assert after < 0.5 * before, (after, before)


def test_scene_light_sums(oracle_lib):
    """collectLights in the oracle: every computing brick's emission goes to exactly one
    anchor, so the luminance and RGB totals over anchors do not depend on the anchors; a single
    anchor gathers them all, and its offset sum is the luminance-weighted centroid's."""
    from firepro import render
    sc = scenes.ForceScene()
    o = _sim(sc, real=1, budget=2 ** 20)
    for s in range(4):
        o.step(sc.frame(s).frame)
    st = render.default_settings()
    one = o.collect_lights(st, [[0.0, 0.0, 0.0]])
    three = o.collect_lights(st, [[0.0, 0.2, 0.0], [1.0, 0.2, 0.0], [-1.0, 0.5, 0.3]])
    assert one[0, 0] > 0
    for k in (0, 4, 5, 6):
        assert three[:, k].sum() == pytest.approx(one[0, k], rel=1e-12)
    centroid = one[0, 1:4] / one[0, 0]
    assert 0.0 < centroid[1] < 1.5 and abs(centroid[0]) < 0.5 and abs(centroid[2]) < 0.5
    far = o.collect_lights(st, [[0.0, 0.0, 0.0], [50.0, 0.0, 0.0]])
    assert far[1, 0] == 0 and far[0, 0] == pytest.approx(one[0, 0], rel=1e-12)
    o.close()


def test_solver_schedules_converge():
    """The oracle's pressure solves (the checker of the CUDA schedules): on the plume, the
    reference's Jacobi V-cycles, the red-black V-cycle and flexible CG around either. Each
    residual norm is the FP64 sum of squares of rhs + A x over the unknowns after a V-cycle;
    the red-black cycles converge at least as fast as the reference's, and CG reduces the
    residual 100-fold in 8 V-cycles where the reference's V-cycle iteration does not."""
    sc = scenes.SinglePlume()
    out = {}
    for name, sched in [("jacobi", abi.schedule()),
                        ("redblack", abi.schedule(abi.FP_SMOOTHER_REDBLACK, 0, 2, 2, 8)),
                        ("fcg", abi.schedule(krylov=abi.FP_KRYLOV_FCG)),
                        ("fcg_redblack", abi.schedule(abi.FP_SMOOTHER_REDBLACK, 0, 2, 2, 8, abi.FP_KRYLOV_FCG))]:
        o = _sim(sc, real=0)
        o.set_solver(8)
        o.set_schedule(sched)
        for s in range(6):
            o.step(sc.frame(s).frame)
        r = np.sqrt(o.cg_residuals())
        assert r.size == 8 and np.all(np.isfinite(r)) and r[0] > 0
        out[name] = r / r[0]
        o.close()
    assert out["redblack"][-1] <= out["jacobi"][-1]
    assert out["fcg"][-1] < 1e-2 and out["fcg_redblack"][-1] < 1e-2
    assert out["jacobi"][-1] > 1e-3
    # CG never lets the residual grow much, step to step.
    for name in ("fcg", "fcg_redblack"):
        assert np.all(out[name][1:] <= 1.5 * out[name][:-1]), out[name]


def _cube(half):
    v = np.array([[x, y, z] for z in (-half, half) for y in (-half, half) for x in (-half, half)], np.float32)
    # outward-wound faces of the cube (corner index = x + 2y + 4z)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tris = []
    for a, b, c, d in quads:
        tris += [(a, b, c), (a, c, d)]
    return v, np.array(tris, np.uint32)


def test_mesh_voxelize_cube_is_cell_centre_inclusion():
    """The oracle's MeshCollider.voxelize on a box: a cell is solid exactly when its centre lies
    inside the box (faces placed off the cell centres)."""
    from oracle import fp_oracle

    pos, idx = _cube(0.113)
    M = np.eye(4)
    M[:3, 3] = [0.31, 0.52, -0.07]
    h = 0.025
    lo, dims, words = fp_oracle.mesh_voxelize(pos, idx, M, h)
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")[: int(np.prod(dims))].reshape(dims[2], dims[1], dims[0])
    z, y, x = np.meshgrid(*[(np.arange(dims[a]) + lo[a] + 0.5) * h for a in (2, 1, 0)], indexing="ij")
    inside = (np.abs(x - 0.31) < 0.113) & (np.abs(y - 0.52) < 0.113) & (np.abs(z + 0.07) < 0.113)
    assert inside.sum() > 500 and np.array_equal(bits.astype(bool), inside)


def test_mesh_splat_single_sample():
    """The oracle's MeshSourceRasterizer: one sample splats weight x area / mean face area over
    its 8 cells trilinearly; coverage caps at 1 and scales the rates."""
    from firepro.mesh import MeshEmitter
    from oracle import fp_oracle

    h = 0.1
    e = MeshEmitter([[0.125, 0.26, 0.375]], [1.0], 0.01 * 3, flame=0.5, heat=2.0, smoke=1.0, fuel=0.25,
                    velocity=(0, 1, 0), response=60.0)
    recs = fp_oracle.mesh_splat([e], h)
    assert len(recs) == 8
    g = np.array([0.125, 0.26, 0.375]) / h - 0.5
    base, f = np.floor(g), g - np.floor(g)
    for r in recs:
        off = np.array(r.cell[:3]) - base
        w = np.prod(np.where(off == 1, f, 1 - f))
        cover = min(1.0, w * 0.03 / (h * h))
        assert r.scalar[1] == pytest.approx(2.0 * cover, rel=1e-6)
        assert r.scalar[0] == pytest.approx(0.5 * cover, rel=1e-6)
        assert r.motion[1] == pytest.approx(60.0 * cover, rel=1e-6) and r.motion[3] == pytest.approx(60.0 * cover, rel=1e-6)


def test_translation_by_a_tile_is_invariant(oracle_lib):
    # The force scene (colliders of every kind, wind, vortex, targeted radial force, a burst,
    # an emitter that stops) spans negative and positive brick coordinates; moved by one tile
    # (4 bricks) in x and z, every integer table is the same (brick ids and slots follow the
    # tile slots, not the coordinates), the tiles' coordinates move by one, and the fields of
    # each brick match its moved twin. The scene's positions are FP32, so the moved scene's
    # positions round differently: fields agree to ~1e-7, not to FP64 rounding.
    sc = scenes.ForceScene()
    budget = 2 ** 20
    a, b = _sim(sc, real=0, budget=budget), _sim(sc, real=0, budget=budget)
    metres, cells = 4 * sc.brick_size * sc.voxel_size, 4 * sc.brick_size
    for s in range(24):
        a.step(parity.shift_frame(sc.frame(s), 0.0, 0.0, 0).frame)
        b.step(parity.shift_frame(sc.frame(s), metres, metres, cells).frame)
        sa, sb = parity.brick_slots(a), parity.brick_slots(b)
        assert {(x + 4, y, z + 4): v for (x, y, z), v in sa.items()} == sb, f"step {s}: bricks and slots"
        keys = sorted(sa)
        for fid in (abi.FP_FIELD_VELOCITY, abi.FP_FIELD_SCALARS, abi.FP_FIELD_EXPANSION, abi.FP_FIELD_PRESSURE,
                    abi.FP_FIELD_DIVERGENCE):
            fa, fb = a.field(fid, f64=True), b.field(fid, f64=True)
            x = np.stack([fa[sa[k]] for k in keys])
            y = np.stack([fb[sb[(k[0] + 4, k[1], k[2] + 4)]] for k in keys])
            assert np.linalg.norm(x - y) <= 1e-5 * np.linalg.norm(x), (s, fid)
    assert min(len(sa), a.active_bricks) > 100 and any(k[0] < 0 for k in sa), "the scene grew across x = 0"
    for tid in (abi.FP_TABLE_ENTRIES, abi.FP_TABLE_PAGES, abi.FP_TABLE_STATE, abi.FP_TABLE_ACTIVITY,
                abi.FP_TABLE_RECORDS, abi.FP_TABLE_FREE, abi.FP_TABLE_ACTIVE, abi.FP_TABLE_SOLIDS):
        assert np.array_equal(a.table(tid), b.table(tid)), tid
    ta = a.table(abi.FP_TABLE_TILES).view(np.int32).reshape(-1, 4)
    tb = b.table(abi.FP_TABLE_TILES).view(np.int32).reshape(-1, 4)
    live = ta[:, 3] != 0
    assert np.array_equal(ta[:, 3], tb[:, 3]) and np.array_equal(ta[live, :3] + [1, 0, 1], tb[live, :3])
