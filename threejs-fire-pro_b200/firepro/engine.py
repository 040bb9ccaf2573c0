"""`FluidSimulation`-shaped wrapper of the C ABI (src/engine/FluidSimulation.ts).

One object per simulation; every call goes through libfirepro.so. A non-zero status raises
`FireProError` with the library's message, which follows the reference's Error text.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


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
        out = np.empty((s.pool_slots, ch, self.cells), np.float32)
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
