"""Seeded synthetic scenes that drive the step through the C ABI.

Each scene yields one `fp_frame` per step, built the way `FireSimulation.step` builds its
`SimulationFrame` (src/library/FireSimulation.ts:455-519): settings, combustion, fuel,
sources, forces and colliders as they are at that step. No dataset is involved; every
number derives from the scene's seed.

Scenes
  single_plume  — one sphere emitter (r = 0.25 m at y = 0.2 m) injecting heat 1.0/s and fuel
                  0.8/s with a 3-octave value-noise jitter of its rates, over a 6x6x6-brick
                  block held by a zero-rate box source; buoyancy 1.5, vorticity 0.3,
                  combustion on; 8^3-cell bricks of 2.5 cm voxels.
  large_scene   — three seeded sphere/box emitters, a radial burst at step 30 (r = 0.5 m,
                  outward 20 m/s), 2 m/s turbulence, one sphere and one box collider; grows
                  to thousands of bricks.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

from . import abi

# DEFAULT_FLAME_SETTINGS ramps (src/engine/flame.ts:16-40).
DEFAULT_RAMPS = {
    "smoke": [(0.0, 0.0), (0.2, 1.0), (0.5, 0.0), (1.0, 0.0)],
    "heat": [(0.0, 0.0), (0.2, 1.0), (1.0, 1.0)],
    "expansion": [(0.0, 0.0), (0.5, 0.0), (0.75, 1.0), (1.0, 1.0)],
}


def combustion(lifespan=1.2, smoke_rate=2.0, heat_rate=4.0, expansion_rate=1.0, ramps=None) -> abi.fp_combustion:
    """`FlameSettings` with the reference's default ramps (flame.ts:16-40)."""
    c = abi.fp_combustion()
    c.lifespan, c.smoke_rate, c.heat_rate, c.expansion_rate = lifespan, smoke_rate, heat_rate, expansion_rate
    ramps = ramps or DEFAULT_RAMPS
    for i, name in enumerate(("smoke", "heat", "expansion")):
        knots = ramps[name]
        c.ramps[i].count = len(knots)
        for k, (x, y) in enumerate(knots):
            c.ramps[i].knots[k][0] = x
            c.ramps[i].knots[k][1] = y
    return c


def settings(buoyancy=1.6, smoke_weight=0.12, damping=0.1, cooling=0.62, dissipation=0.35, vorticity=3.2, seed=1):
    """`SimulationSettings` with the library defaults (src/library/options.ts:324-361)."""
    s = abi.fp_settings()
    s.buoyancy, s.smoke_weight, s.velocity_damping = buoyancy, smoke_weight, damping
    s.cooling, s.dissipation, s.vorticity, s.seed = cooling, dissipation, vorticity, seed
    return s


def source(id, shape="sphere", position=(0, 0, 0), size=(0.3, 0.3, 0.3), flame=0.0, heat=0.0, smoke=0.0, fuel=0.0,
           velocity=(0, 0, 0), response=0.0, outward=0.0, variation=None) -> abi.fp_source:
    s = abi.fp_source()
    s.id = id
    s.shape = {"sphere": abi.FP_SHAPE_SPHERE, "box": abi.FP_SHAPE_BOX, "mesh": abi.FP_SHAPE_MESH}[shape]
    s.position[:] = position
    s.size[:] = size
    s.flame, s.heat_rate, s.smoke_rate, s.fuel_rate = flame, heat, smoke, fuel
    s.velocity[:] = velocity
    s.velocity_response = response
    s.outward_speed = outward
    if variation is not None:
        s.has_variation = 1
        s.variation_period, s.variation_strength = variation
    return s


def force(kind, vector=(0, 1, 0), center=(0, 0, 0), strength=1.0, scale=1.0, lift=0.0, inward=0.0,
          targeted=False, first_target=0, target_count=0) -> abi.fp_force:
    f = abi.fp_force()
    f.type = {"wind": 0, "turbulence": 1, "vortex": 2, "radial": 3}[kind]
    f.vector[:] = vector
    f.center[:] = center
    f.strength, f.scale, f.lift, f.inward = strength, scale, lift, inward
    f.targeted = int(targeted)
    f.first_target, f.target_count = first_target, target_count
    return f


def collider(shape, position=(0, 0, 0), size=(0.2, 0.2, 0.2), axes=((1, 0, 0), (0, 1, 0), (0, 0, 1))):
    c = abi.fp_collider()
    c.shape = {"sphere": abi.FP_SHAPE_SPHERE, "box": abi.FP_SHAPE_BOX}[shape]
    c.position[:] = position
    c.size[:] = size
    for a in range(3):
        c.axes[a][:] = axes[a]
    return c


def _hash01(i: int, seed: int) -> float:
    h = (i * 374761393 + seed * 668265263) & 0xFFFFFFFF
    h = ((h ^ (h >> 13)) * 1274126177) & 0xFFFFFFFF
    h ^= h >> 16
    return (h & 0xFFFFFF) / float(1 << 24)


def value_noise_1d(t: float, seed: int, octaves: int = 3) -> float:
    """Seeded fractal value noise in [-1, 1]: `octaves` octaves, gain 0.5, lacunarity 2."""
    total, norm, amp, freq = 0.0, 0.0, 1.0, 1.0
    for o in range(octaves):
        x = t * freq
        i = math.floor(x)
        f = x - i
        s = f * f * (3 - 2 * f)
        a = _hash01(i, seed + 101 * o)
        b = _hash01(i + 1, seed + 101 * o)
        total += amp * (2.0 * (a + (b - a) * s) - 1.0)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


@dataclass
class FrameData:
    """One step's frame and the ctypes arrays it points into (kept alive with it)."""

    frame: abi.fp_frame
    keep: list = field(default_factory=list)


def make_frame(sim_settings, comb, fuel_enabled, sources, forces=(), targets=(), colliders=(), masks=(),
               ignition=0.5, burn_rate=4.0, mesh_sources=(), target_cells=()) -> FrameData:
    """`target_cells`: per force target, the lattice cells a mesh target covers (empty for the
    analytic ones)."""
    f = abi.fp_frame()
    f.simulation = sim_settings
    f.combustion = comb
    f.fuel.enabled = int(fuel_enabled)
    f.fuel.ignition_heat = ignition
    f.fuel.burn_rate = burn_rate
    keep = []

    def arr(typ, items):
        a = (typ * max(1, len(items)))(*items)
        keep.append(a)
        return C.cast(a, C.POINTER(typ)), len(items)

    f.sources, f.source_count = arr(abi.fp_source, list(sources))
    f.forces, f.force_count = arr(abi.fp_force, list(forces))
    f.force_targets, f.force_target_count = arr(abi.fp_source, list(targets))
    f.colliders, f.collider_count = arr(abi.fp_collider, list(colliders))
    f.collider_masks, f.collider_mask_words = arr(C.c_uint32, list(masks))
    f.mesh_sources, f.mesh_source_count = arr(abi.fp_mesh_source, list(mesh_sources))
    words, ranges = [], []
    for t in range(len(targets)):
        cells = list(target_cells[t]) if t < len(target_cells) else []
        ranges += [len(words) // 3, len(cells)]
        for c in cells:
            words += list(c)
    f.target_cells, _ = arr(C.c_int32, words)
    f.target_cell_count = len(words) // 3
    f.target_cell_ranges, _ = arr(C.c_uint32, ranges)
    return FrameData(f, keep)


class Scene:
    """A seeded scene: `grid()` for creation, `frame(step)` for every step."""

    name = "scene"
    voxel_size = 0.025
    brick_size = 8
    velocity_divisor = 1
    steps = 120

    def grid(self, precision=abi.FP_PRECISION_FP32, budget=8e6, maccormack=True) -> abi.fp_grid:
        g = abi.fp_grid()
        g.voxel_size = self.voxel_size
        g.velocity_divisor = self.velocity_divisor
        g.brick_size = self.brick_size
        g.smoke_divisor = 1
        g.scalar_maccormack = int(maccormack)
        g.precision = precision
        g.voxel_budget = budget
        return g

    def frame(self, step: int) -> FrameData:
        raise NotImplementedError


class SinglePlume(Scene):
    """The single-simulation plume: 6x6x6-brick starting block around one jittered emitter."""

    name = "single_plume"
    steps = 120

    def __init__(self, seed: int = 1):
        self.seed = seed
        self.settings = settings(buoyancy=1.5, vorticity=0.3, seed=seed)
        self.comb = combustion()

    def frame(self, step: int) -> FrameData:
        j = 1.0 + 0.25 * value_noise_1d(step / 12.0, self.seed)
        plume = source(1, "sphere", (0.0, 0.2, 0.0), (0.25, 0.25, 0.25), flame=0.0, heat=1.0 * j, fuel=0.8 * j)
        # A zero-rate box whose allocation reach (sourceNear: extent + 2 voxels) covers exactly
        # bricks -3..2 in x and z and 0..5 in y: the 6x6x6-brick starting block.
        block = source(2, "box", (0.0, 0.6, 0.0), (0.45, 0.45, 0.45))
        return make_frame(self.settings, self.comb, True, [plume, block])


class LargeScene(Scene):
    """Three seeded emitters, a burst at step 30, turbulence and two colliders."""

    name = "large_scene"
    steps = 600

    def __init__(self, seed: int = 1, smoke: float = 1.5, dissipation: float = 0.75, cooling: float = 0.62,
                 flame_smoke: float = 2.0):
        self.seed = seed
        self.smoke = smoke
        self.settings = settings(buoyancy=1.6, vorticity=1.0, seed=seed, dissipation=dissipation, cooling=cooling)
        self.comb = combustion(smoke_rate=flame_smoke)
        rng = [_hash01(k, seed) for k in range(32)]
        self.emitters = []
        for e in range(3):
            x = -1.2 + 1.2 * e + 0.3 * (rng[3 * e] - 0.5)
            z = 0.4 * (rng[3 * e + 1] - 0.5)
            r = 0.2 + 0.2 * rng[3 * e + 2]
            shape = "box" if e == 1 else "sphere"
            self.emitters.append((shape, (x, 0.25, z), (r, r, r)))

    def frame(self, step: int) -> FrameData:
        srcs = []
        for i, (shape, pos, size) in enumerate(self.emitters):
            j = 1.0 + 0.25 * value_noise_1d(step / 12.0, self.seed + 17 * i)
            srcs.append(source(10 + i, shape, pos, size, flame=0.8, heat=2.0 * j, smoke=self.smoke * j, fuel=0.6 * j,
                               velocity=(0.0, 1.0, 0.0), response=60.0))
        if step == 30:
            # Explosion burst (FireSimulation.ts:471-493): charge / FIXED_DT for one step.
            srcs.append(source(1000, "sphere", (0.0, 1.0, 0.0), (0.5, 0.5, 0.5), flame=1.0, heat=2.0 * 60,
                               smoke=0.5 * 60, fuel=0.0, response=60.0, outward=20.0, variation=(0.5, 0.3)))
        forces = [force("turbulence", strength=2.0, scale=1.0)]
        cols = [collider("sphere", (0.6, 1.3, 0.0), (0.3, 0.3, 0.3)),
                collider("box", (-0.6, 1.6, 0.2), (0.35, 0.1, 0.35))]
        return make_frame(self.settings, self.comb, True, srcs, forces, (), cols)


class ForceScene(Scene):
    """Every force kind (wind, turbulence, vortex, targeted radial), a rotated box and a
    sphere collider, a mesh-mask collider, smoke and flame emitters with velocity
    coupling, a one-step burst with Perlin variation at step 6, and an emitter that stops at
    step 12 so its tiles linger and close."""

    name = "force_scene"
    steps = 80

    def __init__(self, seed: int = 3):
        self.seed = seed
        self.settings = settings(buoyancy=1.6, smoke_weight=0.3, damping=0.2, vorticity=2.0, seed=seed)
        self.comb = combustion()
        # A 10x4x10-cell mesh occupancy mask: a slab with a hole.
        self.mask_lo, self.mask_dims = (-14, 20, -6), (10, 4, 10)
        bits = []
        for z in range(10):
            for y in range(4):
                for x in range(10):
                    bits.append(0 if (3 <= x <= 6 and 3 <= z <= 6) else 1)
        words = [0] * ((len(bits) + 31) // 32)
        for i, b in enumerate(bits):
            if b:
                words[i >> 5] |= 1 << (i & 31)
        self.mask_words = words

    def frame(self, step: int) -> FrameData:
        c, s = math.cos(0.4), math.sin(0.4)
        srcs = [
            source(1, "sphere", (0.05, 0.25, 0.0), (0.2, 0.2, 0.2), flame=1.0, heat=1.5, smoke=0.5,
                   velocity=(0.0, 1.4, 0.0), response=60.0),
            source(2, "box", (-0.5, 0.3, 0.3), (0.12, 0.12, 0.12), flame=0.0, heat=0.85, smoke=4.0,
                   velocity=(0.3, 1.2, 0.0), response=60.0),
        ]
        if step < 12:
            srcs.append(source(3, "sphere", (0.6, 0.2, -0.4), (0.1, 0.1, 0.1), heat=2.0, fuel=1.0))
        if step == 6:
            srcs.append(source(99, "sphere", (0.0, 0.5, 0.0), (0.3, 0.3, 0.3), flame=1.0, heat=2.0 * 60, smoke=0.2 * 60,
                               response=60.0, outward=8.0, variation=(0.5, 0.6)))
        targets = [source(1, "sphere", (0.05, 0.25, 0.0), (0.2, 0.2, 0.2))]
        forces = [force("wind", vector=(1.0, 0.0, 0.0), strength=0.8),
                  force("turbulence", strength=1.5, scale=2.0),
                  force("vortex", vector=(0.0, 1.0, 0.0), center=(0.0, 0.5, 0.0), strength=3.0, scale=0.5, lift=1.0,
                        inward=0.5),
                  force("radial", center=(0.05, 0.4, 0.0), strength=-2.0, scale=0.4, targeted=True, first_target=0,
                        target_count=1)]
        mesh = abi.fp_collider()
        mesh.shape = abi.FP_SHAPE_MESH
        mesh.lo[:] = self.mask_lo
        mesh.dims[:] = self.mask_dims
        mesh.mask_offset = 0
        cols = [collider("box", (0.2, 0.9, 0.1), (0.25, 0.05, 0.2), axes=((c, s, 0), (-s, c, 0), (0, 0, 1))),
                collider("sphere", (-0.4, 0.8, 0.3), (0.12, 0.12, 0.12)), mesh]
        return make_frame(self.settings, self.comb, True, srcs, forces, targets, cols, self.mask_words)


class MeshEmitterScene(Scene):
    """Mesh emission: a disc of lattice cells (the records a mesh source's surface samples
    splat to, MeshSourceRasterizer's output) burning with upward velocity coupling, stepping one
    cell in x every 5 steps so the tables are rebuilt; one sphere emitter beside it."""

    name = "mesh_emitter"
    steps = 40

    def __init__(self, seed: int = 1, radius_cells: int = 6):
        self.seed = seed
        self.radius = radius_cells
        self.settings = settings(buoyancy=1.5, vorticity=0.3, seed=seed)
        self.comb = combustion()

    def records(self, step: int):
        shift = step // 5
        out = []
        r = self.radius
        for dz in range(-r, r + 1):
            for dx in range(-r, r + 1):
                if dx * dx + dz * dz > r * r:
                    continue
                m = abi.fp_mesh_source()
                m.cell[:] = (dx + shift, 4, dz, 0)
                w = 1.0 - (dx * dx + dz * dz) / float((r + 1) * (r + 1))
                m.scalar[:] = (0.9 * w, 2.0 * w, 1.2 * w, 0.5 * w)  # flame, heat, smoke, fuel
                m.motion[:] = (0.0, 1.5 * 4.0 * w, 0.0, 4.0 * w)     # velocity x response, response
                out.append(m)
        return out

    def frame(self, step: int) -> FrameData:
        recs = self.records(step)
        h = self.voxel_size
        lo = [min(m.cell[a] for m in recs) * h + 0.5 * h for a in range(3)]
        hi = [max(m.cell[a] for m in recs) * h + 0.5 * h for a in range(3)]
        mesh = source(3, "mesh", lo, hi, flame=0.9, heat=2.0, smoke=1.2, fuel=0.5)
        ball = source(4, "sphere", (0.6, 0.2, 0.0), (0.15, 0.15, 0.15), heat=1.0, smoke=0.8)
        return make_frame(self.settings, self.comb, True, [mesh, ball], mesh_sources=recs)


class MeshTargetScene(MeshEmitterScene):
    """Mesh force targets: the burning disc plus a targeted wind whose targets are a mesh (a
    column of cells above the disc, the velocity cells its samples reach, following the disc)
    and a sphere around the side emitter, so coverage comes from the cell bits in one place and
    the analytic region in the other; an untargeted vortex beside them."""

    name = "mesh_target"

    def target_cells(self, step: int):
        shift = step // 5
        return [(dx + shift, y, dz) for y in range(5, 14) for dz in range(-3, 4) for dx in range(-3, 4)]

    def frame(self, step: int) -> FrameData:
        recs = self.records(step)
        h = self.voxel_size
        lo = [min(m.cell[a] for m in recs) * h + 0.5 * h for a in range(3)]
        hi = [max(m.cell[a] for m in recs) * h + 0.5 * h for a in range(3)]
        mesh = source(3, "mesh", lo, hi, flame=0.9, heat=2.0, smoke=1.2, fuel=0.5)
        ball = source(4, "sphere", (0.6, 0.2, 0.0), (0.15, 0.15, 0.15), heat=1.0, smoke=0.8)
        cells = self.target_cells(step)
        tlo = [min(c[a] for c in cells) * h + 0.5 * h for a in range(3)]
        thi = [max(c[a] for c in cells) * h + 0.5 * h for a in range(3)]
        targets = [source(5, "mesh", tlo, thi), source(4, "sphere", (0.6, 0.2, 0.0), (0.15, 0.15, 0.15))]
        forces = [force("wind", vector=(1.0, 0.0, 0.4), strength=2.5, targeted=True, first_target=0, target_count=2),
                  force("vortex", vector=(0.0, 1.0, 0.0), center=(0.0, 0.5, 0.0), strength=1.5, scale=0.5,
                        lift=0.5, inward=0.3)]
        return make_frame(self.settings, self.comb, True, [mesh, ball], forces, targets, mesh_sources=recs,
                          target_cells=[cells, []])


class StressScene(Scene):
    """A flamethrower-like jet: a 5 cm box emitter wandering on a smooth path (the editor's
    wanderPosition-style motion, editor/scenes/motion.ts), pushing 25 m/s of fuel-rich flame
    along +x (CFL up to 4 in 2.5 cm voxels at 60 Hz), combustion with fuel 1.0, a 3 m/s
    crosswise wind; grows to thousands of bricks."""

    name = "stress"
    steps = 300

    def __init__(self, seed: int = 1, speed: float = 25.0):
        self.seed = seed
        self.speed = speed
        self.settings = settings(buoyancy=1.6, vorticity=1.5, seed=seed, dissipation=0.02, cooling=0.2, damping=0.02)
        self.comb = combustion(smoke_rate=1.5)

    def position(self, step: int):
        t = step / 60.0
        return (-1.5 + 0.15 * math.sin(1.3 * t + self.seed), 0.4 + 0.1 * math.sin(0.9 * t),
                0.2 * math.sin(0.7 * t + 2.0 * self.seed))

    def frame(self, step: int) -> FrameData:
        j = 1.0 + 0.2 * value_noise_1d(step / 12.0, self.seed)
        jet = source(1, "box", self.position(step), (0.05, 0.05, 0.05), flame=1.0, heat=30.0 * j, smoke=40.0 * j,
                     fuel=1.0 * j, velocity=(self.speed, 2.0, 0.0), response=60.0)
        wind = force("wind", vector=(0.0, 0.0, 1.0), strength=3.0)
        return make_frame(self.settings, self.comb, True, [jet], [wind])


class EmptyScene(Scene):
    """No sources, forces or colliders: nothing computes."""

    name = "empty"

    def __init__(self, seed: int = 1):
        self.settings = settings(seed=seed)
        self.comb = combustion()

    def frame(self, step: int) -> FrameData:
        return make_frame(self.settings, self.comb, False, [])


class MemberScene(Scene):
    """One simulation of a batch or a serving session, drawn from `(seed, index)`: 1-4 sphere or
    box emitters of radius 0.1-0.6 m with heat, smoke and fuel rates 0.2-2.0 /s each, within
    a metre of the origin, combustion on; its brick budget is drawn log-uniform from
    [min_bricks, max_bricks] and caps its growth."""

    name = "member"

    def __init__(self, seed: int = 1, index: int = 0, min_bricks: int = 16, max_bricks: int = 2048):
        self.seed = seed
        self.index = index
        r = [_hash01(index * 64 + k, seed) for k in range(64)]
        self.bricks = int(round(math.exp(math.log(min_bricks) + r[0] * (math.log(max_bricks) - math.log(min_bricks)))))
        self.settings = settings(buoyancy=1.5, vorticity=0.3 + 1.5 * r[1], seed=seed * 1000 + index)
        self.comb = combustion()
        self.emitters = []
        count = 1 + int(r[2] * 4) if r[2] < 1.0 else 4
        for e in range(count):
            q = r[3 + 8 * e: 11 + 8 * e]
            radius = 0.1 + 0.5 * q[0]
            pos = (1.6 * (q[1] - 0.5), 0.1 + radius * 0.5 + 0.3 * q[2], 1.6 * (q[3] - 0.5))
            rates = [0.2 + 1.8 * q[k] for k in (4, 5, 6)]
            shape = "box" if q[7] < 0.3 else "sphere"
            self.emitters.append((shape, pos, (radius, radius, radius), rates))

    @property
    def budget(self) -> float:
        return float(self.bricks * self.brick_size ** 3)

    def frame(self, step: int) -> FrameData:
        srcs = []
        for i, (shape, pos, size, (heat, smoke, fuel)) in enumerate(self.emitters):
            j = 1.0 + 0.25 * value_noise_1d(step / 12.0, self.seed * 7919 + self.index * 31 + i)
            srcs.append(source(i + 1, shape, pos, size, flame=0.0, heat=heat * j, smoke=smoke * j, fuel=fuel * j))
        return make_frame(self.settings, self.comb, True, srcs)


SCENES = {"single_plume": SinglePlume, "large_scene": LargeScene, "force_scene": ForceScene, "stress": StressScene,
          "empty": EmptyScene}
