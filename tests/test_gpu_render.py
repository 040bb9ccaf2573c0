"""The headless volume render through the C ABI against the oracle's FP64 restatement.

Both render the same state: the lockstep parity run forces the CUDA fields into the oracle
each step, so after the last step they hold identical fields and directories. The images
(linear radiance and opacity) must agree within relative L2 RENDER_TOL: the march is the
same arithmetic in FP32 and FP64, with the same jitter, occupancy skips and thresholds.
"""
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
