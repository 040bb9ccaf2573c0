"""Mesh colliders and mesh emitters on the GPU against the oracle: the voxelization
(MeshCollider.voxelize with Collider.meshMask) bit for bit, the surface splat
(MeshSourceRasterizer.prepare) cell for cell with values within FP64 summation order, and a
simulation whose mesh collider and mesh emitter come from the GPU passes every step, in lockstep
with the FP64 oracle."""
import math

import numpy as np
import pytest

from firepro import abi, mesh, scenes
from firepro.engine import FireProError
from oracle import fp_oracle
from test_gpu_parity import check, run

pytestmark = pytest.mark.gpu


def rotation(ax, ay, az):
    cx, sx, cy, sy, cz, sz = math.cos(ax), math.sin(ax), math.cos(ay), math.sin(ay), math.cos(az), math.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def world(t=(0, 0, 0), r=(0, 0, 0), s=(1, 1, 1)):
    M = np.eye(4)
    M[:3, :3] = rotation(*r) @ np.diag(s)
    M[:3, 3] = t
    return M


@pytest.mark.parametrize("case", ["sphere", "ellipsoid_rotated", "hollow_shell", "cube_soup"])
def test_voxelize_matches_oracle_bit_for_bit(case):
    if case == "sphere":
        pos, idx = mesh.icosphere(3, 0.31)
        M = world((0.1, 0.45, -0.05))
    elif case == "ellipsoid_rotated":
        pos, idx = mesh.icosphere(2, 0.2)
        M = world((-0.3, 0.6, 0.2), (0.3, 0.7, -0.4), (1.6, 0.7, 1.1))
    elif case == "hollow_shell":  # outer shell outward, inner shell inward: the cavity stays empty
        po, io = mesh.icosphere(3, 0.35)
        pi, ii = mesh.icosphere(3, 0.2)
        pos = np.concatenate([po, pi])
        idx = np.concatenate([io, ii[:, ::-1] + len(po)])
        M = world((0.0, 0.5, 0.0), (0.2, 0.1, 0.0))
    else:  # a triangle soup without indices, faces on cell centres' planes
        v = np.array([[x, y, z] for z in (-0.1, 0.1) for y in (-0.1, 0.1) for x in (-0.1, 0.1)], np.float32)
        quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
        tris = [t for a, b, c, d in quads for t in ((a, b, c), (a, c, d))]
        pos, idx = v[np.array(tris).ravel()], None
        M = world((0.0125, 0.3125, 0.0125))
    col, words = mesh.voxelize(pos, idx, M, 0.025)
    lo, dims, want = fp_oracle.mesh_voxelize(pos, idx, M, 0.025)
    assert list(col.lo) == list(lo) and list(col.dims) == list(dims)
    assert np.array_equal(words, want), f"{np.count_nonzero(words != want)} words differ"
    assert np.count_nonzero(words) > 0


def test_splat_matches_oracle():
    pos, idx = mesh.icosphere(2, 0.25)
    local, weights, area = mesh.surface_samples(pos, idx, 0.025, seed=7)
    e1 = mesh.MeshEmitter(mesh.place(local, world((0.2, 0.4, 0.0), (0.3, 0.0, 0.2))), weights, area, flame=0.9,
                          heat=2.0, smoke=1.2, fuel=0.5, velocity=(0, 1.5, 0), response=60.0)
    e2 = mesh.MeshEmitter(mesh.place(local, world((0.35, 0.45, 0.1))), weights, area, flame=0.4, heat=1.0,
                          smoke=0.5, velocity=(0.5, 0, 0), response=30.0)
    got = mesh.splat([e1, e2], 0.025)
    want = fp_oracle.mesh_splat([e1, e2], 0.025)
    assert len(got) == len(want) > 100
    for g, w in zip(got, want):
        assert list(g.cell) == list(w.cell)
        for a, b in zip(list(g.scalar) + list(g.motion), list(w.scalar) + list(w.motion)):
            assert a == pytest.approx(b, rel=1e-6, abs=1e-12)


def test_splat_limits():
    e = mesh.MeshEmitter(np.zeros((300000, 3)), np.ones(300000), 1.0, heat=1.0)
    with pytest.raises(FireProError, match="two million cell visits"):
        mesh.splat([e], 0.025)
    e = mesh.MeshEmitter(np.zeros((4, 3)), np.ones(4), 0.0, heat=1.0)
    with pytest.raises(FireProError, match="positive surface area"):
        mesh.splat([e], 0.025)


class DeviceMeshScene(scenes.Scene):
    """A mesh collider (an ellipsoid, turning and sliding) voxelized on the GPU every step, and a
    mesh emitter (an icosphere's surface samples, rising) splatted on the GPU every step."""

    name = "device_mesh"

    def __init__(self):
        self.settings = scenes.settings(buoyancy=1.5, vorticity=0.5, seed=4)
        self.comb = scenes.combustion()
        self.collider = mesh.icosphere(2, 0.15)
        pos, idx = mesh.icosphere(2, 0.12)
        self.samples = mesh.surface_samples(pos, idx, self.voxel_size, seed=3)

    def frame(self, step):
        col, words = mesh.voxelize(*self.collider, world((0.05 + 0.004 * step, 0.75, 0.0), (0.0, 0.05 * step, 0.3),
                                                         (1.5, 0.6, 1.0)), self.voxel_size)
        local, weights, area = self.samples
        at = world((0.0, 0.2 + 0.002 * step, 0.0), (0.0, 0.1 * step, 0.0))
        em = mesh.MeshEmitter(mesh.place(local, at), weights, area, flame=0.9, heat=2.0, smoke=1.2, fuel=0.5,
                              velocity=(0, 1.5, 0), response=60.0)
        recs = mesh.splat([em], self.voxel_size)
        h = self.voxel_size
        lo = [min(r.cell[a] for r in recs) * h + 0.5 * h for a in range(3)]
        hi = [max(r.cell[a] for r in recs) * h + 0.5 * h for a in range(3)]
        src = scenes.source(3, "mesh", lo, hi, flame=0.9, heat=2.0, smoke=1.2, fuel=0.5)
        fd = scenes.make_frame(self.settings, self.comb, True, [src], colliders=[col], masks=list(words),
                               mesh_sources=recs)
        return fd


def test_simulation_with_gpu_mesh_passes_parity():
    check(run(DeviceMeshScene(), 16, budget=2 ** 20), min_active=30)
