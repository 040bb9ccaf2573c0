"""The bounds-checked build (lib/libfirepro_debug.so, FP_BOUNDS) on the GPU.

Its kernels check every index they read out of a table (neighbour-record and brick-entry
slots, tile neighbours and hash hits, work-list brick ids) and record the first bad one instead
of using it. Each case runs in a child process that opens the checked library (FIREPRO_LIBRARY),
steps a scene in lockstep with the FP64 oracle under the same parity rules as the release build,
renders it, and reports the simulation's record: no index may have been out of bounds. Nothing
here plants a bad index on the device; a planted mistake would fault the GPU it ran on.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from firepro import abi
from firepro.engine import FluidSimulation
from firepro import scenes

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
CHILD = r"""
import json, sys
sys.path[:0] = [{root!r}, {root!r} + "/threejs-fire-pro_b200", {root!r} + "/tests"]
from firepro import abi, render, scenes
from firepro.engine import FluidSimulation
import parity
from test_gpu_parity import check

sc = getattr(scenes, {scene!r})()
out = {{}}
def after(sim, orc):  # the last step's state, before the simulation is disposed
    cam = render.look_at((0.0, 1.0, 3.0), (0.0, 0.5, 0.0), 160, 90)
    sim.render(cam, render.default_settings(ray_steps=48, shadow_samples=8))
    b = sim.read_bounds()
    out.update(checked=b.checked, count=b.count, site=b.site, index=b.index, limit=b.limit)
reports = parity.lockstep(sc, {steps}, lambda g: FluidSimulation(g), budget={budget}, after=after)
check(reports, min_active={min_active})
print("BOUNDS " + json.dumps(out))
"""


def run_checked(scene: str, steps: int, budget: int, min_active: int) -> dict:
    env = dict(os.environ, FIREPRO_LIBRARY=str(abi.DEBUG_LIB_PATH))
    code = CHILD.format(root=str(ROOT), scene=scene, steps=steps, budget=budget, min_active=min_active)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("BOUNDS ")][-1]
    return json.loads(line[len("BOUNDS "):])


@pytest.mark.parametrize("scene,steps,budget,min_active", [("SinglePlume", 24, 2 ** 19, 216),
                                                           ("LargeScene", 34, 2 ** 20, 100)])
def test_checked_build_parity_and_no_bad_index(scene, steps, budget, min_active):
    if not abi.DEBUG_LIB_PATH.exists():
        pytest.fail("the bounds-checked build is missing: build.py --debug (or __graft_entry__.build())")
    b = run_checked(scene, steps, budget, min_active)
    assert b["checked"] == 1, "the child did not open the checked build"
    assert b["count"] == 0, f"out-of-bounds index: {b}"


def test_release_build_reports_unchecked():
    sim = FluidSimulation(scenes.SinglePlume().grid(budget=2 ** 19))
    b = sim.read_bounds()
    assert b.checked == 0 and b.count == 0
    sim.dispose()
