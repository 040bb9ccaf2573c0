"""Lockstep parity harness: the CUDA step against the FP64 oracle from identical state.

Each step both run the same frame from the same state. Integer tables must match bit for
bit; each field must match within the relative-L2 tolerance. The CUDA fields and activity
flags are then copied into the oracle (teacher forcing), so per-step differences never
compound through the flow's chaos.
"""
from __future__ import annotations

import numpy as np

from firepro import abi
from oracle.fp_oracle import OracleSim

# The parity tolerance: relative L2 <= 1e-3 against the FP64 oracle per field per step.
REL_L2_TOL = 1e-3

CHECK_FIELDS = {
    "velocity": abi.FP_FIELD_VELOCITY,
    "scalars": abi.FP_FIELD_SCALARS,
    "expansion": abi.FP_FIELD_EXPANSION,
    "pressure": abi.FP_FIELD_PRESSURE,
    "divergence": abi.FP_FIELD_DIVERGENCE,
}


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    num = float(np.linalg.norm((a.astype(np.float64) - b).ravel()))
    den = float(np.linalg.norm(b.ravel()))
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den


def active_slots(entries: np.ndarray) -> np.ndarray:
    e = entries.view(np.int32)
    return np.unique(e[e >= 0] & 0xFFFFFF)


def compare_tables(gpu, orc) -> dict:
    """Bit-exact comparison of the allocation's integer tables. Returns mismatch counts."""
    out = {}
    for name, tid in (("entries", abi.FP_TABLE_ENTRIES), ("pages", abi.FP_TABLE_PAGES),
                      ("state", abi.FP_TABLE_STATE), ("active", abi.FP_TABLE_ACTIVE),
                      ("free", abi.FP_TABLE_FREE), ("tiles", abi.FP_TABLE_TILES)):
        a, b = gpu.table(tid), orc.table(tid)
        if name == "state":
            a, b = a & 1, b & 1  # the persistent bit; the rank bits are scratch
        out[name] = int(np.count_nonzero(a != b)) if a.shape == b.shape else -1
    ea = gpu.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    ra = gpu.table(abi.FP_TABLE_RECORDS).reshape(-1, 28)
    rb = orc.table(abi.FP_TABLE_RECORDS).reshape(-1, 28)
    live = ea >= 0
    out["records"] = int(np.count_nonzero(ra[live] != rb[live])) if ra.shape == rb.shape else -1
    act_a = gpu.table(abi.FP_TABLE_ACTIVITY)
    act_b = orc.table(abi.FP_TABLE_ACTIVITY)
    out["activity"] = int(np.count_nonzero(act_a != act_b)) if act_a.shape == act_b.shape else -1
    if gpu.table(abi.FP_TABLE_SOLIDS).shape == orc.table(abi.FP_TABLE_SOLIDS).shape:
        slots = active_slots(ea)
        sa = gpu.table(abi.FP_TABLE_SOLIDS).reshape(gpu_slots(gpu), -1)[slots]
        sb = orc.table(abi.FP_TABLE_SOLIDS).reshape(orc.slots, -1)[slots]
        out["solids"] = int(np.count_nonzero(sa != sb))
    return out


def gpu_slots(gpu) -> int:
    return int(gpu.stats().pool_slots)


# A MacCormack limiter test whose corrected value lies within FP32 rounding of the donors'
# bound may go the other way in the FP64 oracle; that face then keeps the predicted instead of
# the corrected value (or the reverse), which moves the face and the divergence of its two
# cells by up to the correction. Like the activity flags, a few such isolated flips are
# allowed per step: without the FLIP_CELLS(n) largest pointwise differences a field must be
# within the tolerance, and with them within FLIP_BOUND times it.
FLIP_BOUND = 10.0


def flip_cells(bricks: int) -> int:
    return 2 * max(2, bricks // 500)


def trimmed_rel_l2(a: np.ndarray, b: np.ndarray, k: int) -> float:
    """rel_l2 without the k largest pointwise differences (the denominator keeps them)."""
    d = np.abs(a.astype(np.float64) - b).ravel()
    if 0 < k < d.size:
        d = np.partition(d, d.size - k)[: d.size - k]
    den = float(np.linalg.norm(b.ravel()))
    num = float(np.linalg.norm(d))
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den


def compare_fields(gpu, orc, slots: np.ndarray) -> dict:
    """Per field (scalars per channel): relative L2, and under name + "@trim" the same without
    the flip_cells(len(slots)) largest pointwise differences."""
    out = {}
    k = flip_cells(len(slots))
    for name, fid in CHECK_FIELDS.items():
        a = gpu.field(fid)[slots]
        b = orc.field(fid, f64=orc.real == 0)[slots]
        if fid == abi.FP_FIELD_SCALARS:
            for c, ch in enumerate(("smoke", "heat", "lifetime", "fuel")):
                out[ch] = rel_l2(a[:, c], b[:, c])
                out[ch + "@trim"] = trimmed_rel_l2(a[:, c], b[:, c], k)
        else:
            out[name] = rel_l2(a, b)
            out[name + "@trim"] = trimmed_rel_l2(a, b, k)
    if getattr(gpu, "smoke_cells", 0):  # the coarse smoke grid (smoke_divisor > 1)
        a = gpu.field(abi.FP_FIELD_SMOKE)[slots]
        b = orc.field(abi.FP_FIELD_SMOKE, f64=orc.real == 0)[slots]
        out["coarse_smoke"] = rel_l2(a, b)
        out["coarse_smoke@trim"] = trimmed_rel_l2(a, b, k)
    return out


def field_within(fields: dict, name: str, tol: float) -> bool:
    """The acceptance rule above for one field of a compare_fields report."""
    v = fields[name]
    return v <= tol or (fields[name + "@trim"] <= tol and v <= FLIP_BOUND * tol)


def force(gpu, orc):
    """Copy the CUDA state that carries into the next step into the oracle."""
    for fid in (abi.FP_FIELD_VELOCITY, abi.FP_FIELD_SCALARS, abi.FP_FIELD_EXPANSION):
        orc.write_field(fid, gpu.field(fid))
    if getattr(gpu, "smoke_cells", 0):
        orc.write_field(abi.FP_FIELD_SMOKE, gpu.field(abi.FP_FIELD_SMOKE))
    orc.write_activity(gpu.table(abi.FP_TABLE_ACTIVITY))


def lockstep(scene, steps: int, gpu_factory, cutoff=0.05, budget=8e6, ground=True, start=0, log=None, grid=None,
             before_step=None, vcycles=1, after=None, schedule=None):
    """Run `steps` steps in lockstep; returns per-step (tables, fields) reports.
    `before_step(step, gpu, oracle)` may change runtime settings on both. `vcycles` V-cycles
    a step on both sides (tolerance 0: all of them run), with the pressure-solve `schedule`
    (an abi.fp_solver_schedule; None: the reference's)."""
    grid = grid if grid is not None else scene.grid(budget=budget)
    gpu = gpu_factory(grid)
    orc = OracleSim(grid, real=0)
    gpu.set_runtime(cutoff, budget, ground)
    orc.set_runtime(cutoff, budget, ground)
    if vcycles != 1:
        gpu.set_solver(vcycles, 0.0)
        orc.set_solver(vcycles)
    if schedule is not None:
        gpu.set_schedule(schedule)
        orc.set_schedule(schedule)
    reports = []
    for s in range(start, start + steps):
        if before_step:
            before_step(s, gpu, orc)
        fd = scene.frame(s)
        gpu.step(fd.frame)
        orc.step(fd.frame)
        tables = compare_tables(gpu, orc)
        slots = active_slots(gpu.table(abi.FP_TABLE_ENTRIES))
        fields = compare_fields(gpu, orc, slots)
        reports.append((s, tables, fields, len(slots)))
        if log:
            log(s, tables, fields, len(slots))
        force(gpu, orc)
    if after:
        after(gpu, orc)  # both hold the same state here
    gpu.dispose()
    orc.close()
    return reports


def brick_slots(sim) -> dict:
    """World brick coordinates -> slot of every brick with one."""
    entries = sim.table(abi.FP_TABLE_ENTRIES).view(np.int32)
    tiles = sim.table(abi.FP_TABLE_TILES).view(np.int32).reshape(-1, 4)
    ids = np.nonzero(entries >= 0)[0]
    t, l = tiles[ids >> 6], ids & 63
    coords = np.stack([t[:, 0] * 4 + (l & 3), t[:, 1] * 4 + ((l >> 2) & 3), t[:, 2] * 4 + (l >> 4)], 1)
    return {tuple(int(v) for v in c): int(entries[i] & 0xFFFFFF) for i, c in zip(ids, coords)}


def shift_frame(fd, dx: float, dz: float, cells: int):
    """The frame's scene moved by (dx, 0, dz) metres (`cells` field cells for mesh-mask
    colliders), with turbulence off: its noise is sampled at world positions."""
    f = fd.frame
    for k in range(f.force_count):
        if f.forces[k].type == 1:
            f.forces[k].strength = 0.0
        f.forces[k].center[0] += dx
        f.forces[k].center[2] += dz
    for rows, n in ((f.sources, f.source_count), (f.force_targets, f.force_target_count)):
        for k in range(n):
            rows[k].position[0] += dx
            rows[k].position[2] += dz
    for k in range(f.collider_count):
        c = f.colliders[k]
        if c.shape == abi.FP_SHAPE_MESH:
            c.lo[0] += cells
            c.lo[2] += cells
        else:
            c.position[0] += dx
            c.position[2] += dz
    return fd

