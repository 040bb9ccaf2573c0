"""`FluidSimulation`-shaped wrapper of the C ABI (src/engine/FluidSimulation.ts).

One object per simulation; every call goes through libfirepro.so. A non-zero status raises
`FireProError` with the library's message, which follows the reference's Error text.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class Snapshot:
    """A state blob the library allocated (fp_*_snapshot), kept in host memory without a copy
    (states of large budgets take gigabytes) and released with fp_snapshot_free. `bytes(blob)`
    copies it; restore() takes either."""

    def __init__(self, lib, ptr: C.c_void_p, size: int):
        self.lib, self.ptr, self.size = lib, ptr, size

    def __len__(self) -> int:
        return self.size

    def __bytes__(self) -> bytes:
        out = bytearray(self.size)
        C.memmove((C.c_char * self.size).from_buffer(out), self.ptr, self.size)
        return bytes(out)

    def __getitem__(self, key):
        return bytes(self)[key]

    def __del__(self):
        if getattr(self, "ptr", None):
            self.lib.fp_snapshot_free(self.ptr)
            self.ptr = None


def _blob(blob):
    """(pointer, size) of a Snapshot or a bytes-like blob."""
    if isinstance(blob, Snapshot):
        return blob.ptr, blob.size
    return blob, len(blob)


class FireProError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


FIXED_DT = 1.0 / 60.0


class FluidSimulation:
    def __init__(self, grid: abi.fp_grid, device: int = 0):
        self.lib = abi.load_library()
        self.grid = grid
        h = C.c_void_p()
        rc = self.lib.fp_sim_create(C.byref(grid), device, C.byref(h))
        if rc != abi.FP_OK:
            raise FireProError(rc, self.lib.fp_last_error(None).decode())
        self.h = h
        self.cells = grid.brick_size ** 3
        # cells a slot of the velocity lattice (velocity, pressure, divergence, curl)
        self.velocity_cells = self.cells // max(1, grid.velocity_divisor) ** 3
        # cells a slot of the coarse smoke grid (FP_FIELD_SMOKE), smoke_divisor > 1 only
        self.smoke_cells = self.cells // grid.smoke_divisor ** 3 if grid.smoke_divisor > 1 else 0

    def _check(self, rc: int):
        if rc != abi.FP_OK:
            raise FireProError(rc, self.lib.fp_last_error(self.h).decode())

    def dispose(self):
        if getattr(self, "h", None):
            self.lib.fp_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    def set_runtime(self, cutoff: float, voxel_budget: float, ground: bool):
        self._check(self.lib.fp_sim_set_runtime(self.h, cutoff, voxel_budget, int(ground)))

    def step(self, frame: abi.fp_frame, dt: float = FIXED_DT):
        self._check(self.lib.fp_sim_step(self.h, C.byref(frame), dt))

    def reserve_tiles(self, tiles: int):
        self._check(self.lib.fp_sim_reserve_tiles(self.h, tiles))

    def set_solver(self, vcycles: int, tolerance: float = 0.0):
        """Up to `vcycles` V-cycles a step, stopping at relative residual `tolerance` (0: all)."""
        self._check(self.lib.fp_sim_set_solver(self.h, vcycles, tolerance))

    def set_schedule(self, schedule: abi.fp_solver_schedule):
        """The pressure solve's smoother, levels, sweeps and Krylov wrapper (fp_sim_set_schedule)."""
        self._check(self.lib.fp_sim_set_schedule(self.h, C.byref(schedule)))

    def snapshot(self) -> Snapshot:
        """The whole state between steps (fp_sim_snapshot)."""
        p, n = C.c_void_p(), C.c_size_t()
        self._check(self.lib.fp_sim_snapshot(self.h, C.byref(p), C.byref(n)))
        return Snapshot(self.lib, p, n.value)

    def restore(self, blob):
        """Put a snapshot of a simulation of the same grid back (fp_sim_restore)."""
        self._check(self.lib.fp_sim_restore(self.h, *_blob(blob)))

    def render(self, camera: abi.fp_camera, settings: abi.fp_render_settings) -> np.ndarray:
        """The latest state rendered: (height, width, 4) linear radiance and opacity."""
        out = np.zeros((camera.height, camera.width, 4), np.float32)
        self._check(self.lib.fp_sim_render(self.h, C.byref(camera), C.byref(settings), out.ctypes.data))
        return out

    def render_device(self, camera: abi.fp_camera, settings: abi.fp_render_settings, image_ptr: int):
        """Render into device memory at `image_ptr` (width x height x 4 floats), enqueued."""
        self._check(self.lib.fp_sim_render_device(self.h, C.byref(camera), C.byref(settings), image_ptr))

    def collect_lights(self, settings: abi.fp_render_settings, anchors) -> np.ndarray:
        """Scene-light sums of the latest state (SceneLights.sample's GPU pass): (anchors, 8)
        floats, the luminance, its weighted offset from the anchor and the RGB of the flames
        nearest each anchor."""
        a = np.ascontiguousarray(np.asarray(anchors, np.float32).reshape(-1, 3))
        out = np.zeros((len(a), 8), np.float32)
        self._check(self.lib.fp_sim_collect_lights(self.h, C.byref(settings), a.ctypes.data, len(a), out.ctypes.data))
        return out

    def read_solver(self) -> abi.fp_solver_stats:
        """The latest step's pressure solve (waits for the step)."""
        s = abi.fp_solver_stats()
        self._check(self.lib.fp_sim_read_solver(self.h, C.byref(s)))
        return s

    def read_bounds(self) -> abi.fp_bounds:
        """The bounds-checked build's record (checked 0 in the release build)."""
        b = abi.fp_bounds()
        self._check(self.lib.fp_sim_read_bounds(self.h, C.byref(b)))
        return b

    def reset(self):
        self._check(self.lib.fp_sim_reset(self.h))

    def synchronize(self):
        self._check(self.lib.fp_sim_synchronize(self.h))

    def stats(self) -> abi.fp_stats:
        s = abi.fp_stats()
        self._check(self.lib.fp_sim_stats(self.h, C.byref(s)))
        return s

    def field(self, fid: int) -> np.ndarray:
        s = self.stats()
        ch = abi.FIELD_CHANNELS[fid]
        cells = self.smoke_cells if fid == abi.FP_FIELD_SMOKE else (
            self.velocity_cells if fid in abi.VELOCITY_FIELDS else self.cells)
        out = np.empty((s.pool_slots, ch, cells), np.float32)
        self._check(self.lib.fp_sim_read_field(self.h, fid, out.ctypes.data_as(C.POINTER(C.c_float)), out.nbytes))
        return out

    def table(self, tid: int) -> np.ndarray:
        n = C.c_size_t(0)
        self.lib.fp_sim_read_table(self.h, tid, None, C.byref(n))
        out = np.empty(max(1, n.value // 4), np.uint32)
        n2 = C.c_size_t(out.nbytes)
        self._check(self.lib.fp_sim_read_table(self.h, tid, out.ctypes.data, C.byref(n2)))
        return out[: n2.value // 4]

    def stream(self) -> int:
        """The cudaStream_t the simulation enqueues on, as an integer handle."""
        out = C.c_void_p()
        self._check(self.lib.fp_sim_stream(self.h, C.byref(out)))
        return out.value or 0

    def set_profiling(self, on: bool):
        self._check(self.lib.fp_sim_set_profiling(self.h, int(on)))

    def profile(self) -> dict:
        """Per-phase device time since profiling started: {name: (launches, ms, voxels)}."""
        arr = (abi.fp_phase * 16)()
        n = C.c_uint32(16)
        self._check(self.lib.fp_sim_read_profile(self.h, arr, C.byref(n)))
        return {arr[i].name.decode(): (arr[i].launches, arr[i].ms, arr[i].voxels) for i in range(n.value)}

    def read_bricks(self) -> np.ndarray:
        n = C.c_uint32(0)
        self.lib.fp_sim_read_bricks(self.h, None, C.byref(n))
        out = np.empty((max(1, n.value), 6), np.float32)
        cnt = C.c_uint32(n.value)
        self._check(self.lib.fp_sim_read_bricks(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(cnt)))
        return out[: cnt.value]


class SimulationBatch:
    """Many simulations stepped by one launch (fp_batch_* of the C ABI).

    `add` returns an id; `step` takes a list of (id, frame, dt) and steps them together. Each
    simulation's results are the same as stepping it alone with `FluidSimulation`.
    """

    def __init__(self, brick_size: int = 8, device: int = 0):
        self.lib = abi.load_library()
        h = C.c_void_p()
        rc = self.lib.fp_batch_create(device, brick_size, C.byref(h))
        if rc != abi.FP_OK:
            raise FireProError(rc, self.lib.fp_last_error(None).decode())
        self.h = h
        self.cells = brick_size ** 3
        self._divisors = {}  # per simulation: its velocity divisor (velocity-lattice field sizes)
        self._frames = None

    def _check(self, rc: int):
        if rc != abi.FP_OK:
            raise FireProError(rc, self.lib.fp_batch_last_error(self.h).decode())

    def dispose(self):
        if getattr(self, "h", None):
            self.lib.fp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    def add(self, grid: abi.fp_grid) -> int:
        out = C.c_uint32()
        self._check(self.lib.fp_batch_add(self.h, C.byref(grid), C.byref(out)))
        self._divisors[out.value] = max(1, grid.velocity_divisor)
        return out.value

    def remove(self, sim: int):
        self._check(self.lib.fp_batch_remove(self.h, sim))

    def reset(self, sim: int):
        self._check(self.lib.fp_batch_reset(self.h, sim))

    def set_runtime(self, sim: int, cutoff: float, voxel_budget: float, ground: bool):
        self._check(self.lib.fp_batch_set_runtime(self.h, sim, cutoff, voxel_budget, int(ground)))

    def reserve_tiles(self, sim: int, tiles: int):
        self._check(self.lib.fp_batch_reserve_tiles(self.h, sim, tiles))

    def set_solver(self, sim: int, vcycles: int, tolerance: float = 0.0):
        self._check(self.lib.fp_batch_set_solver(self.h, sim, vcycles, tolerance))

    def set_schedule(self, sim: int, schedule: abi.fp_solver_schedule):
        self._check(self.lib.fp_batch_set_schedule(self.h, sim, C.byref(schedule)))

    def snapshot(self, sim: int) -> Snapshot:
        p, n = C.c_void_p(), C.c_size_t()
        self._check(self.lib.fp_batch_snapshot(self.h, sim, C.byref(p), C.byref(n)))
        return Snapshot(self.lib, p, n.value)

    def restore(self, sim: int, blob):
        self._check(self.lib.fp_batch_restore(self.h, sim, *_blob(blob)))

    def read_solver(self, sim: int) -> abi.fp_solver_stats:
        s = abi.fp_solver_stats()
        self._check(self.lib.fp_batch_read_solver(self.h, sim, C.byref(s)))
        return s

    def step(self, items):
        """Step [(id, fp_frame, dt), ...] in one launch."""
        n = len(items)
        ids = (C.c_uint32 * n)(*[i for i, _, _ in items])
        frames = (abi.fp_frame * n)(*[f for _, f, _ in items])
        dts = (C.c_float * n)(*[d for _, _, d in items])
        self._frames = frames  # the frames' arrays stay alive with their owners
        self._check(self.lib.fp_batch_step(self.h, ids, frames, dts, n))

    def synchronize(self):
        self._check(self.lib.fp_batch_synchronize(self.h))

    def stats(self, sim: int) -> abi.fp_stats:
        s = abi.fp_stats()
        self._check(self.lib.fp_batch_stats(self.h, sim, C.byref(s)))
        return s

    def field(self, sim: int, fid: int) -> np.ndarray:
        s = self.stats(sim)
        ch = abi.FIELD_CHANNELS[fid]
        cells = self.cells // self._divisors.get(sim, 1) ** 3 if fid in abi.VELOCITY_FIELDS else self.cells
        out = np.empty((s.pool_slots, ch, cells), np.float32)
        self._check(self.lib.fp_batch_read_field(self.h, sim, fid, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                 out.nbytes))
        return out

    def table(self, sim: int, tid: int) -> np.ndarray:
        n = C.c_size_t(0)
        self.lib.fp_batch_read_table(self.h, sim, tid, None, C.byref(n))
        out = np.empty(max(1, n.value // 4), np.uint32)
        n2 = C.c_size_t(out.nbytes)
        self._check(self.lib.fp_batch_read_table(self.h, sim, tid, out.ctypes.data, C.byref(n2)))
        return out[: n2.value // 4]

    def stream(self) -> int:
        out = C.c_void_p()
        self._check(self.lib.fp_batch_stream(self.h, C.byref(out)))
        return out.value or 0

    def set_profiling(self, on: bool):
        self._check(self.lib.fp_batch_set_profiling(self.h, int(on)))

    def profile(self) -> dict:
        arr = (abi.fp_phase * 16)()
        n = C.c_uint32(16)
        self._check(self.lib.fp_batch_read_profile(self.h, arr, C.byref(n)))
        return {arr[i].name.decode(): (arr[i].launches, arr[i].ms, arr[i].voxels) for i in range(n.value)}


def reserved_tiles(grid: abi.fp_grid) -> int:
    """The tile reservation a server gives a session of `grid`."""
    lib = abi.load_library()
    out = C.c_uint32()
    rc = lib.fp_grid_reserved_tiles(C.byref(grid), C.byref(out))
    if rc != abi.FP_OK:
        raise FireProError(rc, lib.fp_last_error(None).decode())
    return out.value


def grid_memory_bytes(grid: abi.fp_grid) -> int:
    """Device bytes a simulation of `grid` holds once created (the admission estimate)."""
    lib = abi.load_library()
    out = C.c_uint64()
    rc = lib.fp_grid_memory_bytes(C.byref(grid), C.byref(out))
    if rc != abi.FP_OK:
        raise FireProError(rc, lib.fp_last_error(None).decode())
    return out.value


class FireServer:
    """Serving front end (fp_server_* of the C ABI): sessions admitted by device-memory
    budget, their step requests batched by a scheduler thread as they arrive."""

    def __init__(self, memory_budget: int, max_sessions: int = 256, brick_size: int = 8, device: int = 0):
        self.lib = abi.load_library()
        cfg = abi.fp_server_config(device, brick_size, int(memory_budget), max_sessions)
        h = C.c_void_p()
        rc = self.lib.fp_server_create(C.byref(cfg), C.byref(h))
        if rc != abi.FP_OK:
            raise FireProError(rc, self.lib.fp_last_error(None).decode())
        self.h = h
        self.cells = brick_size ** 3
        self._buf = (abi.fp_completion * 1024)()

    def _check(self, rc: int):
        if rc != abi.FP_OK:
            raise FireProError(rc, self.lib.fp_server_last_error(self.h).decode())

    def dispose(self):
        if getattr(self, "h", None):
            self.lib.fp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    def open(self, grid: abi.fp_grid, cutoff: float = 0.05, ground: bool = True) -> int:
        out = C.c_uint32()
        self._check(self.lib.fp_server_open(self.h, C.byref(grid), cutoff, int(ground), C.byref(out)))
        return out.value

    def snapshot(self, session: int) -> Snapshot:
        """A live, idle session's state (fp_server_snapshot)."""
        p, n = C.c_void_p(), C.c_size_t()
        self._check(self.lib.fp_server_snapshot(self.h, session, C.byref(p), C.byref(n)))
        return Snapshot(self.lib, p, n.value)

    def restore(self, session: int, blob):
        self._check(self.lib.fp_server_restore(self.h, session, *_blob(blob)))

    def set_solver(self, schedule: abi.fp_solver_schedule, vcycles: int = 1, tolerance: float = 0.0):
        """The pressure solve of the sessions opened from now on (fp_server_set_solver)."""
        self._check(self.lib.fp_server_set_solver(self.h, C.byref(schedule), vcycles, tolerance))

    def close(self, session: int):
        self._check(self.lib.fp_server_close(self.h, session))

    def state(self, session: int) -> int:
        out = C.c_int()
        self._check(self.lib.fp_server_session_state(self.h, session, C.byref(out)))
        return out.value

    def submit(self, session: int, frame: abi.fp_frame, dt: float = FIXED_DT) -> int:
        t = C.c_uint64()
        self._check(self.lib.fp_server_submit(self.h, session, C.byref(frame), dt, C.byref(t)))
        return t.value

    def poll(self, wait_ms: int = 0) -> list:
        n = C.c_uint32()
        self._check(self.lib.fp_server_poll(self.h, self._buf, len(self._buf), C.byref(n), wait_ms))
        return [abi.fp_completion.from_buffer_copy(self._buf[i]) for i in range(n.value)]

    def drain(self, wait_ms: int = 60000):
        self._check(self.lib.fp_server_drain(self.h, wait_ms))

    def stats(self) -> abi.fp_server_stats:
        s = abi.fp_server_stats()
        self._check(self.lib.fp_server_read_stats(self.h, C.byref(s)))
        return s

    def session_stats(self, session: int) -> abi.fp_stats:
        s = abi.fp_stats()
        self._check(self.lib.fp_server_session_stats(self.h, session, C.byref(s)))
        return s

    def field(self, session: int, fid: int) -> np.ndarray:
        ch = abi.FIELD_CHANNELS[fid]
        out = np.empty((self.session_stats(session).pool_slots, ch, self.cells), np.float32)
        self._check(self.lib.fp_server_read_field(self.h, session, fid, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                  out.nbytes))
        return out
