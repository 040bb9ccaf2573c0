"""Cameras and render settings for `fp_sim_render` (the headless volume render).

`look_at` builds the clip-to-world matrix the march reads (column-major, as the reference's
WGSL mat4x4f). `default_settings` fills the render uniform with the library's option defaults
where they map one to one (src/library/options.ts:341-364: smoke density 2.5, shadow density
3.5, flame brightness 1.4 and opacity 0.55, temperature 3200 K, soot glow 1, cubic filter,
256 ray steps, lighting divisor 4; 32 shadow samples, types.ts:7), with a white sun.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi


def look_at(eye, target, width: int, height: int, fov_deg: float = 45.0, near: float = 0.05, far: float = 50.0,
            time: float = 0.0) -> abi.fp_camera:
    eye, target = np.asarray(eye, np.float64), np.asarray(target, np.float64)
    f = target - eye
    f /= np.linalg.norm(f)
    up = np.array([0.0, 1.0, 0.0])
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = s, u, -f
    view[:3, 3] = -view[:3, :3] @ eye
    aspect = width / height
    t = 1.0 / math.tan(math.radians(fov_deg) / 2)
    # WebGPU clip space: depth in [0, 1].
    proj = np.zeros((4, 4))
    proj[0, 0], proj[1, 1] = t / aspect, t
    proj[2, 2], proj[2, 3] = far / (near - far), near * far / (near - far)
    proj[3, 2] = -1.0
    inv = np.linalg.inv(proj @ view)
    cam = abi.fp_camera()
    cam.inverse_view_projection[:] = [float(v) for v in inv.T.reshape(-1)]  # column-major
    cam.width, cam.height, cam.time = width, height, time
    return cam


def default_settings(filter_mode: int = 2, ray_steps: int = 256, lighting_divisor: int = 4,
                     shadow_samples: int = 32) -> abi.fp_render_settings:
    s = abi.fp_render_settings()
    s.optical[:] = [2.5, 1.4, 3.5, 0.38]
    s.light[:] = [0.35, 1.0, 0.25, 1.0]
    s.smoke[:] = [0.145, 0.161, 0.180, 1.0]
    s.fire[:] = [1.0, 1.0, 1.0, 3200.0]
    s.scene_light[:] = [1.0, 1.0, 1.0]
    s.ambient_light[:] = [0.15, 0.15, 0.15]
    s.flame_opacity = 0.55
    s.shadow_samples = shadow_samples
    s.ray_steps = ray_steps
    s.filter = filter_mode
    s.lighting_divisor = lighting_divisor
    return s


def measure_lights(sums: np.ndarray, anchors, brick_size: int, voxel_size: float, intensity: float = 1.0):
    """Each anchor's light from its scene-light sums (SceneLights.apply, SceneLights.ts:216-248):
    the anchor moved to the centroid of its emission, the colour normalised to its peak
    channel (no less than 1e-8), and an intensity of twice the emitted energy (each sample
    stands for a cube a quarter of a brick wide) times `intensity`, capped at 400. Returns
    (position, rgb, intensity) per anchor."""
    sample = (brick_size / 4) * voxel_size
    lights = []
    for row, anchor in zip(np.asarray(sums, np.float64), np.asarray(anchors, np.float64).reshape(-1, 3)):
        mass, offset, rgb = row[0], row[1:4], row[4:7]
        energy = max(0.0, mass) * sample ** 3
        position = anchor + (offset / mass if mass > 0 else 0.0)
        peak = max(float(rgb.max()), 1e-8)
        lights.append((position, rgb / peak, min(400.0, energy * 2 * intensity)))
    return lights
