"""The C ABI without a GPU: the library loads, exports every function include/firepro.h
declares, and the ctypes mirror has the C layout of every struct."""
import ctypes as C
import re
import subprocess
import tempfile
from pathlib import Path

import pytest

from firepro import abi

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "firepro.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(fp_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_function(cuda_lib_path):
    lib = C.CDLL(str(cuda_lib_path))
    names = declared_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(abi.SIGNATURES), "the ctypes mirror declares exactly the header's functions"


def test_debug_library_exports_every_declared_function():
    """The bounds-checked build (build.py --debug) exports the same functions."""
    if not abi.DEBUG_LIB_PATH.exists():
        pytest.skip("the bounds-checked build is not built here")
    lib = C.CDLL(str(abi.DEBUG_LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_abi_version(cuda_lib_path):
    lib = abi.load_library(cuda_lib_path)
    assert lib.fp_abi_version() == 1


def test_struct_layouts_match_c():
    structs = ["fp_grid", "fp_settings", "fp_flame_ramp", "fp_combustion", "fp_fuel", "fp_source", "fp_force",
               "fp_collider", "fp_mesh_source", "fp_frame", "fp_stats", "fp_phase", "fp_server_config", "fp_completion",
               "fp_server_stats", "fp_solver_stats", "fp_camera", "fp_render_settings", "fp_bounds"]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"firepro.h\"\nint main(void){\n"
    for s in structs:
        src += f'  printf("{s} %zu\\n", sizeof({s}));\n'
    for s, cls in [(s, getattr(abi, s)) for s in structs]:
        for fname, _ in cls._fields_:
            src += f'  printf("{s}.{fname} %zu\\n", offsetof({s}, {fname}));\n'
    src += "  return 0;\n}\n"
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "layout.c"
        c.write_text(src)
        exe = Path(d) / "layout"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        name, value = line.split()
        if "." in name:
            s, f = name.split(".")
            assert getattr(getattr(abi, s), f).offset == int(value), name
        else:
            assert C.sizeof(getattr(abi, name)) == int(value), name


def test_create_rejects_invalid_grid_without_gpu(cuda_lib_path):
    """Validation runs before any device call, with the reference's messages."""
    lib = abi.load_library(cuda_lib_path)
    cases = [
        (dict(voxel_size=0.00001), "voxelSize must be from 0.0001 to 16 meters."),
        (dict(velocity_divisor=3), "velocityDivisor must be 1, 2 or 4."),
        (dict(brick_size=12), "brickSize must be 8, 16 or 32 fine cells."),
        (dict(smoke_divisor=3), "smokeDivisor must be 1, 2 or 4."),
        (dict(scalar_maccormack=2), "scalarMacCormack must be a boolean."),
    ]
    for change, message in cases:
        g = abi.fp_grid(voxel_size=0.025, velocity_divisor=1, brick_size=8, smoke_divisor=1, scalar_maccormack=1,
                        precision=0, voxel_budget=0)
        for k, v in change.items():
            setattr(g, k, v)
        h = C.c_void_p()
        rc = lib.fp_sim_create(C.byref(g), 0, C.byref(h))
        assert rc == abi.FP_EINVAL
        assert lib.fp_last_error(None).decode() == message
