"""The headless volume render through the C ABI against the oracle's FP64 restatement.

Both render the same state: the lockstep parity run forces the CUDA fields into the oracle
each step, so after the last step they hold identical fields and directories. The images
(linear radiance and opacity) must agree within relative L2 RENDER_TOL: the march is the
same arithmetic in FP32 and FP64, with the same jitter, occupancy skips and thresholds.
"""
import ctypes as C

import numpy as np
import pytest

from firepro import abi, render, scenes
from firepro.engine import FluidSimulation
import parity

pytestmark = pytest.mark.gpu

RENDER_TOL = 2e-3


def render_pair(scene, steps, budget, camera, settings):
    out = {}

    def after(gpu, orc):
        out["gpu"] = gpu.render(camera, settings)
        out["orc"] = orc.render(camera, settings)

    parity.lockstep(scene, steps, lambda g: FluidSimulation(g), budget=budget, after=after)
    return out["gpu"], out["orc"]


@pytest.mark.parametrize("filter_mode", [0, 1, 2])
def test_flame_render_parity(filter_mode):
    """Smoke and flame emitters, colliders, every force: each reconstruction filter."""
    cam = render.look_at((1.4, 1.0, 2.0), (0.0, 0.45, 0.0), 64, 48, time=0.5)
    st = render.default_settings(filter_mode=filter_mode, ray_steps=128)
    gpu, orc = render_pair(scenes.ForceScene(), 12, 2 ** 20, cam, st)
    assert np.isfinite(gpu).all()
    assert orc[..., 3].max() > 0.05, "the flames and smoke should be visible"
    err = parity.rel_l2(gpu, orc.astype(np.float64))
    print(f"flames filter {filter_mode}: relative L2 {err:.2e}, opacity max {orc[..., 3].max():.3f}")
    assert err <= RENDER_TOL


@pytest.mark.parametrize("divisor,velocity", [(2, 1), (4, 2)])
def test_coarse_smoke_render_parity(divisor, velocity):
    """Coarse smoke (smokeDivisor 2 and 4): the smoke smoothed on its own lattice
    (smoothCoarseSmoke), sampled once per march step and light sample (renderSmokeAt), the
    fields as the simulation holds them, and the occupancy's conservative bound over coarse
    donors (cachedSmokeCell); with a velocity divisor too."""
    cam = render.look_at((1.4, 1.0, 2.0), (0.0, 0.45, 0.0), 64, 48, time=0.5)
    st = render.default_settings(ray_steps=128)
    sc = scenes.ForceScene()
    sc.velocity_divisor = velocity
    g = sc.grid(budget=2 ** 20)
    g.smoke_divisor = divisor
    out = {}

    def after(gpu, orc):
        out["gpu"] = gpu.render(cam, st)
        out["orc"] = orc.render(cam, st)

    parity.lockstep(sc, 12, lambda gr: FluidSimulation(gr), budget=2 ** 20, grid=g, after=after)
    gpu, orc = out["gpu"], out["orc"]
    assert np.isfinite(gpu).all()
    assert orc[..., 3].max() > 0.05, "the smoke should be visible"
    err = parity.rel_l2(gpu, orc.astype(np.float64))
    print(f"coarse smoke /{divisor}: relative L2 {err:.2e}, opacity max {orc[..., 3].max():.3f}")
    assert err <= RENDER_TOL


def test_large_scene_render_parity():
    """Colliders, turbulence, three emitters; lighting at divisor 2."""
    cam = render.look_at((2.5, 1.6, 3.2), (0.0, 0.8, 0.0), 64, 40, time=1.0)
    st = render.default_settings(ray_steps=128, lighting_divisor=2)
    gpu, orc = render_pair(scenes.LargeScene(), 24, 2 ** 20, cam, st)
    err = parity.rel_l2(gpu, orc.astype(np.float64))
    print(f"large: relative L2 {err:.2e}, opacity max {orc[..., 3].max():.3f}")
    assert orc[..., 3].max() > 0.05
    assert err <= RENDER_TOL


def test_empty_render_is_clear():
    sc = scenes.EmptyScene()
    sim = FluidSimulation(sc.grid(budget=2 ** 18))
    for s in range(3):
        fd = sc.frame(s)
        sim.step(fd.frame)
    img = sim.render(render.look_at((1, 1, 1), (0, 0, 0), 16, 16), render.default_settings())
    assert not img.any()
    sim.dispose()


def test_render_validation():
    sc = scenes.SinglePlume()
    sim = FluidSimulation(sc.grid(budget=2 ** 18))
    st = render.default_settings()
    st.lighting_divisor = 3
    from firepro.engine import FireProError
    with pytest.raises(FireProError):
        sim.render(render.look_at((1, 1, 1), (0, 0, 0), 8, 8), st)
    sim.dispose()


@pytest.mark.parametrize("smoke_divisor", [1, 2])
def test_scene_lights_parity(smoke_divisor):
    """collectLights (scene-lights.wgsl:37-106) against the oracle on the same state: each
    anchor's luminance, luminance-weighted offset and RGB sums; the totals over anchors do not
    depend on where the anchors are; `measure_lights` places each light inside the flames. With
    coarse smoke each sample's density comes from the coarse grid."""
    st = render.default_settings()
    sc = scenes.ForceScene()
    grid = sc.grid(budget=2 ** 20)
    grid.smoke_divisor = smoke_divisor
    anchors = np.array([[0.05, 0.25, 0.0], [-0.5, 0.3, 0.3], [0.6, 0.2, -0.4], [0.0, 0.5, 0.0]], np.float32)
    moved = np.array([[3.0, 0.0, 3.0], [-0.1, 0.9, 0.2]], np.float32)
    out = {}

    def after(gpu, orc):
        out["gpu"], out["orc"] = gpu.collect_lights(st, anchors), orc.collect_lights(st, anchors)
        out["gpu_moved"], out["orc_moved"] = gpu.collect_lights(st, moved), orc.collect_lights(st, moved)
        out["none"] = gpu.collect_lights(st, np.zeros((0, 3), np.float32))

    parity.lockstep(sc, 10, lambda g: FluidSimulation(g), budget=2 ** 20, grid=grid, after=after)
    gpu, orc = out["gpu"].astype(np.float64), out["orc"]
    assert orc[:, 0].sum() > 0, "the flames should emit"
    assert out["none"].shape == (0, 8)
    for name, g, o in (("anchors", gpu, orc), ("moved", out["gpu_moved"].astype(np.float64), out["orc_moved"])):
        scale = o[:, 0].sum()
        for k in range(7):
            # the offsets cancel: their tolerance is the mass times a brick's width
            tol = 1e-4 * (np.abs(o[:, k]) + (scale * 0.2 if 1 <= k <= 3 else 0.0)) + 1e-9
            assert np.all(np.abs(g[:, k] - o[:, k]) <= tol), (name, k, g[:, k], o[:, k])
        assert np.all(g[:, 7] == 0)
    for k in (0, 4, 5, 6):
        assert abs(gpu[:, k].sum() - out["gpu_moved"][:, k].astype(np.float64).sum()) <= 1e-5 * gpu[:, k].sum()
    lights = render.measure_lights(gpu, anchors, 8, sc.voxel_size)
    for (position, rgb, intensity), row in zip(lights, gpu):
        if row[0] > 0:
            assert 0 < intensity <= 400 and rgb.max() <= 1.0 + 1e-6
            if row[4:7].max() >= 1e-8:  # dimmer colours are divided by 1e-8, as the reference does
                assert rgb.max() == pytest.approx(1.0)
            assert position[1] >= 0.0


@pytest.mark.parametrize("half", [0, 1])
def test_scene_depth_and_half_resolution(half):
    """fireProSceneDistance (volume-march.wgsl:76-89): a depth buffer ends the rays at a tilted
    plane through the flames; with `half_resolution` the half-resolution pass records eight
    depths (buildSlices) and each pixel resumes from the last one in front of the scene."""
    w, hgt = 64, 48
    cam = render.look_at((1.4, 1.0, 2.0), (0.0, 0.45, 0.0), w, hgt, time=0.5)
    # clip z of a plane 2.35 m + 0.4 (u - .5) m from the eye along each pixel's ray: from the
    # projection's depth mapping, z_clip = (far (d - near)) / (d (far - near)) for eye depth d
    near, far = 0.05, 50.0
    u = (np.arange(w) + 0.5) / w
    d = 2.35 + 0.4 * (u[None, :] - 0.5) + np.zeros((hgt, 1))
    depth = np.ascontiguousarray((far * (d - near) / (d * (far - near))).astype(np.float32))
    depth[:, : w // 8] = 1.0  # a band with nothing in front
    cam.scene_depth = depth.ctypes.data_as(C.POINTER(C.c_float))
    cam.half_resolution = half
    st = render.default_settings(ray_steps=128)
    out = {}

    def after(gpu, orc):
        out["gpu"] = gpu.render(cam, st)
        out["orc"] = orc.render(cam, st)
        cam.scene_depth = None
        out["open"] = orc.render(cam, st)

    parity.lockstep(scenes.ForceScene(), 12, lambda g: FluidSimulation(g), budget=2 ** 20, after=after)
    gpu, orc = out["gpu"], out["orc"]
    assert np.isfinite(gpu).all()
    assert orc[..., 3].max() > 0.05
    err = parity.rel_l2(gpu, orc.astype(np.float64))
    print(f"depth, half {half}: relative L2 {err:.2e}")
    assert err <= RENDER_TOL
    # the depth clipped something, and nothing where the band is open
    assert np.abs(out["open"] - orc).max() > 1e-3
    assert np.allclose(out["open"][:, : w // 8], orc[:, : w // 8], atol=1e-5) or half


class TwoFires(scenes.Scene):
    """Two burning emitters 4.4 m apart: their tiles form two clusters, so the render marches two
    boxes (TileDirectory.clusters, FluidSimulation.updateBoxes) and a ray between them crosses
    empty space that no box holds."""

    name = "two_fires"

    def __init__(self):
        self.settings = scenes.settings(buoyancy=1.5, vorticity=0.5, seed=9)
        self.comb = scenes.combustion()

    def frame(self, step):
        srcs = [scenes.source(1, "sphere", (-2.2, 0.25, 0.0), (0.2, 0.2, 0.2), flame=0.9, heat=2.0, smoke=1.5, fuel=0.6),
                scenes.source(2, "box", (2.2, 0.25, 0.1), (0.15, 0.15, 0.15), flame=0.7, heat=1.5, smoke=2.0, fuel=0.4)]
        return scenes.make_frame(self.settings, self.comb, True, srcs)


@pytest.mark.parametrize("half", [0, 1])
def test_two_cluster_render_parity(half):
    """One render box per cluster of tiles: the passes clamp and page within each brick's own
    box, the march crosses the boxes in order (span, step and slices over all of them)."""
    cam = render.look_at((0.0, 1.2, 6.5), (0.0, 0.5, 0.0), 96, 48, time=0.25)
    cam.half_resolution = half
    st = render.default_settings(ray_steps=128)
    gpu, orc = render_pair(TwoFires(), 14, 2 ** 21, cam, st)
    assert np.isfinite(gpu).all()
    left, right = orc[:, :48, 3].max(), orc[:, 48:, 3].max()
    assert left > 0.02 and right > 0.02, (left, right)
    err = parity.rel_l2(gpu, orc.astype(np.float64))
    print(f"two clusters (half {half}): relative L2 {err:.2e}")
    assert err <= RENDER_TOL
