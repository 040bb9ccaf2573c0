"""TEST INFRASTRUCTURE — ctypes wrapper of the CPU oracle (oracle/_ref/libfp_oracle.so).

Only tests/, bench.py's `cpu_baseline` leg and __graft_entry__.smoke() may use this. The
oracle restates the reference's step on the CPU: real=0 is the FP64 error oracle, real=1
the FP32 CPU baseline. Parity unpinned: the reference has no tests or runnable CPU path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libfp_oracle.so"


def build() -> Path:
    subprocess.run(["make", "-C", str(HERE)], check=True, stdout=subprocess.DEVNULL)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_set_runtime.argtypes = [C.c_void_p, C.c_float, C.c_double, C.c_int]
        L.or_set_solver.argtypes = [C.c_void_p, C.c_int]
        L.or_set_schedule.argtypes = [C.c_void_p, C.c_void_p, C.c_float]
        L.or_mesh_voxelize.restype = C.c_int64
        L.or_mesh_voxelize.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_double,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64]
        L.or_mesh_splat.restype = C.c_int64
        L.or_mesh_splat.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_void_p, C.c_uint64]
        L.or_read_cg.restype = C.c_int
        L.or_read_cg.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.or_step.restype = C.c_int
        L.or_step.argtypes = [C.c_void_p, C.c_void_p, C.c_float]
        L.or_render.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_collect_lights.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.or_blackbody_table.argtypes = [C.c_void_p]
        L.or_error.restype = C.c_char_p
        L.or_error.argtypes = [C.c_void_p]
        L.or_info.restype = C.c_int64
        L.or_info.argtypes = [C.c_void_p, C.c_int]
        L.or_read_field.restype = C.c_int
        L.or_read_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        L.or_write_field.restype = C.c_int
        L.or_write_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        L.or_read_field64.restype = C.c_int
        L.or_read_field64.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        L.or_read_table.restype = C.c_int64
        L.or_read_table.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        L.or_write_activity.restype = C.c_int
        L.or_write_activity.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        _lib = L
    return _lib


CHANNELS = {0: 3, 1: 4, 2: 1, 3: 1, 4: 1, 5: 4, 6: 1}
SMOKE_FIELD = 6  # the coarse smoke grid: (B / smoke_divisor)^3 cells a slot
VELOCITY_FIELDS = (0, 3, 4, 5)  # the velocity lattice: (B / velocity_divisor)^3 cells a slot


class OracleSim:
    """One oracle simulation. `real`: 0 FP64, 1 FP32. `mode`: 0 the grid's precision,
    2 the reference's half-precision storage."""

    def __init__(self, grid, real: int = 0, mode: int = 0):
        self.L = lib()
        self.h = self.L.or_create(C.byref(grid), real, mode)
        if not self.h:
            raise ValueError("oracle rejected the grid")
        self.real = real

    def render(self, camera, settings) -> np.ndarray:
        """The render of the current state: (height, width, 4) linear radiance and opacity."""
        out = np.zeros((camera.height, camera.width, 4), np.float32)
        self.L.or_render(self.h, C.byref(camera), C.byref(settings), out.ctypes.data)
        return out

    def collect_lights(self, settings, anchors) -> np.ndarray:
        """The scene-light sums (count, 8) of the current state, FP64."""
        a = np.ascontiguousarray(np.asarray(anchors, np.float32).reshape(-1, 3))
        out = np.zeros((len(a), 8), np.float64)
        self.L.or_collect_lights(self.h, C.byref(settings), a.ctypes.data, len(a), out.ctypes.data)
        return out

    def close(self):
        if self.h:
            self.L.or_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_runtime(self, cutoff: float, budget: float, ground: bool):
        self.L.or_set_runtime(self.h, cutoff, budget, int(ground))

    def set_solver(self, vcycles: int):
        """V-cycles of each later step's pressure solve (defect corrections after the first)."""
        self.L.or_set_solver(self.h, vcycles)

    def set_schedule(self, schedule, tolerance: float = 0.0):
        """The pressure solve's schedule (an abi.fp_solver_schedule) for later steps."""
        self.L.or_set_schedule(self.h, C.byref(schedule), tolerance)

    def cg_residuals(self) -> np.ndarray:
        """The latest CG solve's residual sums of squares, one per V-cycle it ran."""
        out = np.zeros(16, np.float64)
        n = self.L.or_read_cg(self.h, out.ctypes.data, 16)
        return out[:n]

    def step(self, frame, dt: float = 1.0 / 60.0):
        if self.L.or_step(self.h, C.byref(frame), dt) != 0:
            raise ValueError(self.L.or_error(self.h).decode())

    def info(self, what: int) -> int:
        return int(self.L.or_info(self.h, what))

    @property
    def slots(self):
        return self.info(0)

    @property
    def capacity(self):
        return self.info(1)

    @property
    def cells(self):
        return self.info(2)

    @property
    def active_bricks(self):
        return self.info(3)

    def field(self, fid: int, f64: bool = False) -> np.ndarray:
        cells = self.info(9) if fid == SMOKE_FIELD else (self.info(10) if fid in VELOCITY_FIELDS else self.cells)
        n = self.slots * CHANNELS[fid] * cells
        if f64:
            out = np.empty(n, np.float64)
            assert self.L.or_read_field64(self.h, fid, out.ctypes.data, n) == 0
        else:
            out = np.empty(n, np.float32)
            assert self.L.or_read_field(self.h, fid, out.ctypes.data, n) == 0
        return out.reshape(self.slots, CHANNELS[fid], cells)

    def write_field(self, fid: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, np.float32).ravel()
        assert self.L.or_write_field(self.h, fid, a.ctypes.data, a.size) == 0

    def table(self, tid: int) -> np.ndarray:
        n = self.L.or_read_table(self.h, tid, None, 0)
        out = np.empty(max(n, 1), np.uint32)
        self.L.or_read_table(self.h, tid, out.ctypes.data, out.nbytes)
        return out[:n]

    def write_activity(self, arr: np.ndarray):
        a = np.ascontiguousarray(arr, np.uint32)
        assert self.L.or_write_activity(self.h, a.ctypes.data, a.size) == 0


def blackbody_table() -> np.ndarray:
    """The oracle's blackbody table: (512, 4) RGB peak-normalised and log2 radiance, 500-10000 K."""
    out = np.zeros((512, 4), np.float32)
    lib().or_blackbody_table(out.ctypes.data)
    return out


def set_threads(n: int):
    lib().or_set_threads(n)


def mesh_voxelize(positions, indices, world, spacing: float):
    """The oracle's Collider.meshMask + MeshCollider.voxelize: (lo, dims, words)."""
    L = lib()
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    idx = None if indices is None else np.ascontiguousarray(indices, dtype=np.uint32).ravel()
    w = np.ascontiguousarray(np.asarray(world, dtype=np.float64).ravel(order="F"))
    lo, dims = np.zeros(3, np.int32), np.zeros(3, np.int32)
    L.or_mesh_voxelize(pos.ctypes.data, len(pos), None if idx is None else idx.ctypes.data,
                       0 if idx is None else len(idx), w.ctypes.data, spacing, lo.ctypes.data, dims.ctypes.data, None, 0)
    words = np.zeros((int(np.prod(dims.astype(np.int64))) + 31) // 32, np.uint32)
    n = L.or_mesh_voxelize(pos.ctypes.data, len(pos), None if idx is None else idx.ctypes.data,
                           0 if idx is None else len(idx), w.ctypes.data, spacing, lo.ctypes.data, dims.ctypes.data,
                           words.ctypes.data, len(words))
    assert n == len(words)
    return lo, dims, words


def mesh_splat(emitters, spacing: float) -> np.ndarray:
    """The oracle's MeshSourceRasterizer.prepare: records (n, 12) as int32/float32 words in a
    structured view (cell xyzw int32, then 8 float32), ascending by cell."""
    from firepro import abi

    L = lib()
    arr = (abi.fp_mesh_emitter * max(1, len(emitters)))(*[e.struct() for e in emitters])
    n = L.or_mesh_splat(C.addressof(arr), len(emitters), spacing, None, 0)
    if n < 0:
        n = 1 << 22
    out = (abi.fp_mesh_source * max(1, n))()
    got = L.or_mesh_splat(C.addressof(arr), len(emitters), spacing, C.addressof(out), n)
    return list(out[:got])
