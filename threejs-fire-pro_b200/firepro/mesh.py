"""Mesh colliders and mesh emitters: the GPU passes (fp_mesh_voxelize, fp_mesh_splat) and the
host-side setup the reference keeps on the host (MeshSurface's samples).

`voxelize` gives an fp_collider of shape FP_SHAPE_MESH and its occupancy words, as
Collider.frame gives a mesh collider (src/library/handles.ts:299-330); `splat` gives the frame's
mesh-source records, as MeshSourceRasterizer.prepare does (src/engine/MeshSourceRasterizer.ts);
`surface_samples` restates MeshSurface (src/library/MeshSurface.ts:25-103): deterministic,
triangle-area-weighted samples lifted three quarters of a cell off the surface.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi
from .engine import FireProError


def _mesh(positions: np.ndarray, indices) -> tuple:
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    m = abi.fp_mesh()
    m.positions = pos.ctypes.data_as(C.POINTER(C.c_float))
    m.vertex_count = len(pos)
    keep = [pos]
    if indices is not None:
        idx = np.ascontiguousarray(indices, dtype=np.uint32).ravel()
        m.indices = idx.ctypes.data_as(C.POINTER(C.c_uint32))
        m.index_count = len(idx)
        keep.append(idx)
    return m, keep


def voxelize(positions, indices, world, spacing: float, device: int = 0):
    """(fp_collider, words): the mesh's occupancy of lattice cells of `spacing` under the 4x4
    column-major `world` transform, computed on the GPU."""
    lib = abi.load_library()
    m, keep = _mesh(positions, indices)
    w = (C.c_double * 16)(*[float(v) for v in np.asarray(world, dtype=np.float64).ravel(order="F")])
    lo, dims = (C.c_int32 * 3)(), (C.c_int32 * 3)()
    n = C.c_uint32(0)
    rc = lib.fp_mesh_voxelize(device, C.byref(m), w, float(spacing), lo, dims, None, C.byref(n))
    if rc != abi.FP_OK:
        raise FireProError(rc, lib.fp_last_error(None).decode())
    words = np.zeros(n.value, np.uint32)
    rc = lib.fp_mesh_voxelize(device, C.byref(m), w, float(spacing), lo, dims,
                              words.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(n))
    if rc != abi.FP_OK:
        raise FireProError(rc, lib.fp_last_error(None).decode())
    col = abi.fp_collider()
    col.shape = abi.FP_SHAPE_MESH
    col.lo[:] = list(lo)
    col.dims[:] = list(dims)
    col.mask_offset = 0
    return col, words


class MeshEmitter:
    """A mesh emitter's samples (world positions, weights), surface area and rates."""

    def __init__(self, samples, weights, surface_area, flame=0.0, heat=0.0, smoke=0.0, fuel=0.0,
                 velocity=(0.0, 0.0, 0.0), response=0.0):
        self.samples = np.ascontiguousarray(samples, dtype=np.float64).reshape(-1, 3)
        self.weights = np.ascontiguousarray(weights, dtype=np.float64).ravel()
        self.surface_area = float(surface_area)
        self.rates = (flame, heat, smoke, fuel)
        self.velocity = tuple(velocity)
        self.response = response

    def struct(self) -> abi.fp_mesh_emitter:
        e = abi.fp_mesh_emitter()
        e.samples = self.samples.ctypes.data_as(C.POINTER(C.c_double))
        e.weights = self.weights.ctypes.data_as(C.POINTER(C.c_double))
        e.sample_count = len(self.weights)
        e.surface_area = self.surface_area
        e.flame, e.heat_rate, e.smoke_rate, e.fuel_rate = self.rates
        e.velocity[:] = self.velocity
        e.velocity_response = self.response
        return e


def splat(emitters, spacing: float, device: int = 0) -> list:
    """The frame's mesh-source records of `emitters` (MeshEmitter), on the GPU, ascending by cell."""
    lib = abi.load_library()
    arr = (abi.fp_mesh_emitter * max(1, len(emitters)))(*[e.struct() for e in emitters])
    n = C.c_uint32(0)
    rc = lib.fp_mesh_splat(device, arr, len(emitters), float(spacing), None, C.byref(n))
    if rc != abi.FP_OK:
        raise FireProError(rc, lib.fp_last_error(None).decode())
    out = (abi.fp_mesh_source * max(1, n.value))()
    cap = C.c_uint32(n.value)
    rc = lib.fp_mesh_splat(device, arr, len(emitters), float(spacing), out, C.byref(cap))
    if rc != abi.FP_OK:
        raise FireProError(rc, lib.fp_last_error(None).decode())
    return list(out[: cap.value])


def icosphere(subdivisions: int = 2, radius: float = 1.0):
    """A closed, consistently wound (outward) icosphere: (positions float32 (n, 3), indices)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache, nf = {}, []

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    pos = (np.array(verts) * radius).astype(np.float32)
    return pos, np.array(faces, dtype=np.uint32)


def surface_samples(positions, indices, cell_size: float, seed: int = 1):
    """MeshSurface (MeshSurface.ts:25-103): (local sample positions (n, 3) float64, weights,
    surface area). Samples fall at evenly spaced points of the cumulative triangle area, each at a
    seeded random point of its triangle (an LCG as the reference's), lifted 0.75 cell along the
    triangle's normal."""
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    idx = np.asarray(indices, dtype=np.int64).reshape(-1, 3) if indices is not None else np.arange(len(pos)).reshape(-1, 3)
    tri = pos[idx]
    normals = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    areas = np.linalg.norm(normals, axis=1) * 0.5
    cumulative = np.cumsum(np.where(areas > 1e-12, areas, 0.0))
    area = float(cumulative[-1])
    count = min(8192, max(256, math.ceil(area / cell_size ** 2 * 8)))
    state = seed & 0xFFFFFFFF

    def random():
        nonlocal state
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        return state / 4294967296.0

    out = np.zeros((count, 3))
    k = 0
    for i in range(count):
        target = (i + 0.5) / count * area
        while cumulative[k] < target:
            k += 1
        n = normals[k] / np.linalg.norm(normals[k])
        root, along = math.sqrt(random()), random()
        a, b, c = tri[k]
        out[i] = a * (1 - root) + b * (root * (1 - along)) + c * (root * along) + n * (cell_size * 0.75)
    return out, np.full(count, 1.0 / count), area


def place(samples, world) -> np.ndarray:
    """Local sample positions through the 4x4 column-major `world` (applyMatrix4)."""
    m = np.asarray(world, dtype=np.float64)
    h = np.c_[samples, np.ones(len(samples))] @ m.T
    return h[:, :3] / h[:, 3:4]
