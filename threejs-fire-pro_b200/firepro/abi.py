"""ctypes mirror of include/firepro.h and the loader of the CUDA library.

The structs follow the C header field for field. `load_library()` opens the in-tree
`libfirepro.so` built by `build.py`; it raises when the library is missing rather than
falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR.parent / "lib" / "libfirepro.so"
# The bounds-checked build (`build.py --debug`); FIREPRO_LIBRARY names the library to open instead
# of LIB_PATH (set it to this path to run a program on the checked build).
DEBUG_LIB_PATH = PACKAGE_DIR.parent / "lib" / "libfirepro_debug.so"

FP_OK = 0
FP_EINVAL = -1
FP_ENOMEM = -2
FP_ELIMIT = -3
FP_EDEVICE = -4
FP_ETIMEOUT = -5
FP_EUNSUPPORTED = -6

FP_PRECISION_FP32 = 0
FP_PRECISION_MIXED = 1

FP_SHAPE_SPHERE = 0
FP_SHAPE_BOX = 1
FP_SHAPE_MESH = 2

FP_FORCE_WIND = 0
FP_FORCE_TURBULENCE = 1
FP_FORCE_VORTEX = 2
FP_FORCE_RADIAL = 3

FP_FIELD_VELOCITY = 0
FP_FIELD_SCALARS = 1
FP_FIELD_EXPANSION = 2
FP_FIELD_PRESSURE = 3
FP_FIELD_DIVERGENCE = 4
FP_FIELD_CURL = 5
FP_FIELD_SMOKE = 6  # the coarse smoke grid, (B / smoke_divisor)^3 cells a slot
FIELD_CHANNELS = {0: 3, 1: 4, 2: 1, 3: 1, 4: 1, 5: 4, 6: 1}
# fields on the velocity lattice: (brick_size / velocity_divisor)^3 cells a slot
VELOCITY_FIELDS = (FP_FIELD_VELOCITY, FP_FIELD_PRESSURE, FP_FIELD_DIVERGENCE, FP_FIELD_CURL)

FP_TABLE_ENTRIES = 0
FP_TABLE_PAGES = 1
FP_TABLE_STATE = 2
FP_TABLE_ACTIVITY = 3
FP_TABLE_RECORDS = 4
FP_TABLE_FREE = 5
FP_TABLE_ACTIVE = 6
FP_TABLE_SOLIDS = 7
FP_TABLE_TILES = 8


class fp_grid(C.Structure):
    _fields_ = [
        ("voxel_size", C.c_float),
        ("velocity_divisor", C.c_int32),
        ("brick_size", C.c_int32),
        ("smoke_divisor", C.c_int32),
        ("scalar_maccormack", C.c_int32),
        ("precision", C.c_int32),
        ("voxel_budget", C.c_double),
    ]


class fp_settings(C.Structure):
    _fields_ = [
        ("buoyancy", C.c_float),
        ("smoke_weight", C.c_float),
        ("velocity_damping", C.c_float),
        ("cooling", C.c_float),
        ("dissipation", C.c_float),
        ("vorticity", C.c_float),
        ("seed", C.c_uint32),
    ]


class fp_flame_ramp(C.Structure):
    _fields_ = [("count", C.c_uint32), ("knots", (C.c_float * 2) * 8)]


class fp_combustion(C.Structure):
    _fields_ = [
        ("lifespan", C.c_float),
        ("smoke_rate", C.c_float),
        ("heat_rate", C.c_float),
        ("expansion_rate", C.c_float),
        ("ramps", fp_flame_ramp * 3),
    ]


class fp_fuel(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("ignition_heat", C.c_float), ("burn_rate", C.c_float)]


class fp_source(C.Structure):
    _fields_ = [
        ("id", C.c_uint64),
        ("shape", C.c_int32),
        ("position", C.c_float * 3),
        ("size", C.c_float * 3),
        ("flame", C.c_float),
        ("heat_rate", C.c_float),
        ("smoke_rate", C.c_float),
        ("fuel_rate", C.c_float),
        ("velocity", C.c_float * 3),
        ("velocity_response", C.c_float),
        ("outward_speed", C.c_float),
        ("has_variation", C.c_int32),
        ("variation_period", C.c_float),
        ("variation_strength", C.c_float),
    ]


class fp_force(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("vector", C.c_float * 3),
        ("center", C.c_float * 3),
        ("strength", C.c_float),
        ("scale", C.c_float),
        ("lift", C.c_float),
        ("inward", C.c_float),
        ("targeted", C.c_int32),
        ("first_target", C.c_uint32),
        ("target_count", C.c_uint32),
    ]


class fp_collider(C.Structure):
    _fields_ = [
        ("shape", C.c_int32),
        ("position", C.c_float * 3),
        ("size", C.c_float * 3),
        ("axes", (C.c_float * 3) * 3),
        ("lo", C.c_int32 * 3),
        ("dims", C.c_int32 * 3),
        ("mask_offset", C.c_uint32),
    ]


class fp_mesh_source(C.Structure):
    _fields_ = [("cell", C.c_int32 * 4), ("scalar", C.c_float * 4), ("motion", C.c_float * 4)]


class fp_frame(C.Structure):
    _fields_ = [
        ("simulation", fp_settings),
        ("combustion", fp_combustion),
        ("fuel", fp_fuel),
        ("sources", C.POINTER(fp_source)),
        ("source_count", C.c_uint32),
        ("forces", C.POINTER(fp_force)),
        ("force_count", C.c_uint32),
        ("force_targets", C.POINTER(fp_source)),
        ("force_target_count", C.c_uint32),
        ("colliders", C.POINTER(fp_collider)),
        ("collider_count", C.c_uint32),
        ("collider_masks", C.POINTER(C.c_uint32)),
        ("collider_mask_words", C.c_uint32),
        ("mesh_sources", C.POINTER(fp_mesh_source)),
        ("mesh_source_count", C.c_uint32),
        ("target_cells", C.POINTER(C.c_int32)),
        ("target_cell_count", C.c_uint32),
        ("target_cell_ranges", C.POINTER(C.c_uint32)),
    ]


class fp_stats(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("steps", C.c_uint64),
        ("active_bricks", C.c_uint32),
        ("brick_cells", C.c_uint32),
        ("pool_limited", C.c_int32),
        ("pool_slots", C.c_uint32),
        ("used_slots", C.c_uint32),
        ("tiles", C.c_uint32),
        ("tile_capacity", C.c_uint32),
        ("failures", C.c_uint32),
        ("memory_bytes", C.c_uint64),
        ("last_vcycles", C.c_uint32),
        ("last_residual", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("h2d_bytes", C.c_uint64),
        ("d2h_bytes", C.c_uint64),
        ("host_prepare_ms", C.c_double),
        ("host_wait_ms", C.c_double),
        ("last_divergence", C.c_double),
        ("bricks_stepped", C.c_uint64),
    ]


class fp_camera(C.Structure):
    _fields_ = [("inverse_view_projection", C.c_float * 16), ("width", C.c_uint32), ("height", C.c_uint32),
                ("time", C.c_float), ("scene_depth", C.POINTER(C.c_float)), ("half_resolution", C.c_uint32)]


class fp_render_settings(C.Structure):
    _fields_ = [
        ("optical", C.c_float * 4),
        ("light", C.c_float * 4),
        ("smoke", C.c_float * 4),
        ("fire", C.c_float * 4),
        ("scene_light", C.c_float * 3),
        ("ambient_light", C.c_float * 3),
        ("flame_opacity", C.c_float),
        ("shadow_samples", C.c_uint32),
        ("ray_steps", C.c_uint32),
        ("filter", C.c_int32),
        ("lighting_divisor", C.c_uint32),
    ]


FP_MAX_VCYCLES = 16


class fp_solver_stats(C.Structure):
    _fields_ = [
        ("vcycles", C.c_uint32),
        ("measured", C.c_int32),
        ("unknowns", C.c_double),
        ("rhs_rms", C.c_double),
        ("residual", C.c_double * FP_MAX_VCYCLES),
        ("divergence", C.c_double),
    ]


class fp_bounds(C.Structure):
    _fields_ = [("checked", C.c_int32), ("count", C.c_uint32), ("site", C.c_int32), ("pad", C.c_int32),
                ("index", C.c_int64), ("limit", C.c_int64)]


class fp_mesh(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("vertex_count", C.c_uint32),
                ("indices", C.POINTER(C.c_uint32)), ("index_count", C.c_uint32)]


class fp_mesh_emitter(C.Structure):
    _fields_ = [("samples", C.POINTER(C.c_double)), ("weights", C.POINTER(C.c_double)), ("sample_count", C.c_uint32),
                ("surface_area", C.c_double), ("flame", C.c_double), ("heat_rate", C.c_double),
                ("smoke_rate", C.c_double), ("fuel_rate", C.c_double), ("velocity", C.c_double * 3),
                ("velocity_response", C.c_double)]


FP_SMOOTHER_JACOBI = 0
FP_SMOOTHER_REDBLACK = 1
FP_KRYLOV_NONE = 0
FP_KRYLOV_FCG = 1


class fp_solver_schedule(C.Structure):
    _fields_ = [("smoother", C.c_int32), ("levels", C.c_int32), ("pre_sweeps", C.c_int32),
                ("post_sweeps", C.c_int32), ("bottom_sweeps", C.c_int32), ("krylov", C.c_int32),
                ("topology", C.c_int32)]


def schedule(smoother=FP_SMOOTHER_JACOBI, levels=0, pre=2, post=2, bottom=8, krylov=FP_KRYLOV_NONE, topology=0):
    """An fp_solver_schedule; the default is the reference's Jacobi V-cycle."""
    return fp_solver_schedule(smoother, levels, pre, post, bottom, krylov, topology)


class fp_phase(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_uint64), ("ms", C.c_double), ("voxels", C.c_double)]


FP_SESSION_WAITING = 0
FP_SESSION_LIVE = 1
FP_SESSION_CLOSING = 2
FP_SESSION_CLOSED = 3
FP_SESSION_FAILED = 4


class fp_server_config(C.Structure):
    _fields_ = [("device", C.c_int), ("brick_size", C.c_int), ("memory_budget", C.c_uint64),
                ("max_sessions", C.c_uint32)]


class fp_completion(C.Structure):
    _fields_ = [
        ("session", C.c_uint32),
        ("status", C.c_int),
        ("ticket", C.c_uint64),
        ("step", C.c_uint64),
        ("active_bricks", C.c_uint32),
        ("batch_size", C.c_uint32),
        ("submit_ms", C.c_double),
        ("done_ms", C.c_double),
    ]


class fp_server_stats(C.Structure):
    _fields_ = [
        ("live", C.c_uint32),
        ("waiting", C.c_uint32),
        ("queued_steps", C.c_uint32),
        ("memory_bytes", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("steps_done", C.c_uint64),
        ("launches", C.c_uint64),
        ("voxel_steps", C.c_double),
        ("elapsed_ms", C.c_double),
        ("latency_p50_ms", C.c_double),
        ("latency_p99_ms", C.c_double),
        ("mean_batch", C.c_double),
    ]


# Exported symbols of libfirepro.so (include/firepro.h), with their ctypes signatures.
SIGNATURES = {
    "fp_abi_version": (C.c_int, []),
    "fp_last_error": (C.c_char_p, [C.c_void_p]),
    "fp_sim_create": (C.c_int, [C.POINTER(fp_grid), C.c_int, C.POINTER(C.c_void_p)]),
    "fp_sim_destroy": (C.c_int, [C.c_void_p]),
    "fp_sim_reset": (C.c_int, [C.c_void_p]),
    "fp_sim_set_runtime": (C.c_int, [C.c_void_p, C.c_float, C.c_double, C.c_int]),
    "fp_sim_step": (C.c_int, [C.c_void_p, C.POINTER(fp_frame), C.c_float]),
    "fp_sim_synchronize": (C.c_int, [C.c_void_p]),
    "fp_sim_stats": (C.c_int, [C.c_void_p, C.POINTER(fp_stats)]),
    "fp_sim_read_field": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.c_size_t]),
    "fp_sim_read_table": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)]),
    "fp_sim_read_bricks": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    "fp_sim_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "fp_sim_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "fp_sim_read_profile": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    "fp_compact_ids_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fp_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "fp_batch_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "fp_batch_destroy": (C.c_int, [C.c_void_p]),
    "fp_batch_add": (C.c_int, [C.c_void_p, C.POINTER(fp_grid), C.POINTER(C.c_uint32)]),
    "fp_batch_remove": (C.c_int, [C.c_void_p, C.c_uint32]),
    "fp_batch_reset": (C.c_int, [C.c_void_p, C.c_uint32]),
    "fp_batch_set_runtime": (C.c_int, [C.c_void_p, C.c_uint32, C.c_float, C.c_double, C.c_int]),
    "fp_batch_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(fp_frame), C.POINTER(C.c_float),
                                C.c_uint32]),
    "fp_batch_synchronize": (C.c_int, [C.c_void_p]),
    "fp_batch_stats": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(fp_stats)]),
    "fp_batch_read_field": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_float), C.c_size_t]),
    "fp_batch_read_table": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)]),
    "fp_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "fp_batch_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "fp_batch_read_profile": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    "fp_grid_memory_bytes": (C.c_int, [C.POINTER(fp_grid), C.POINTER(C.c_uint64)]),
    "fp_grid_reserved_tiles": (C.c_int, [C.POINTER(fp_grid), C.POINTER(C.c_uint32)]),
    "fp_sim_reserve_tiles": (C.c_int, [C.c_void_p, C.c_uint32]),
    "fp_sim_set_solver": (C.c_int, [C.c_void_p, C.c_int, C.c_float]),
    "fp_sim_set_schedule": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fp_sim_render": (C.c_int, [C.c_void_p, C.POINTER(fp_camera), C.POINTER(fp_render_settings), C.c_void_p]),
    "fp_sim_render_device": (C.c_int, [C.c_void_p, C.POINTER(fp_camera), C.POINTER(fp_render_settings), C.c_void_p]),
    "fp_sim_collect_lights": (C.c_int, [C.c_void_p, C.POINTER(fp_render_settings), C.c_void_p, C.c_uint32, C.c_void_p]),
    "fp_sim_read_solver": (C.c_int, [C.c_void_p, C.POINTER(fp_solver_stats)]),
    "fp_sim_read_bounds": (C.c_int, [C.c_void_p, C.POINTER(fp_bounds)]),
    "fp_batch_set_solver": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.c_float]),
    "fp_batch_set_schedule": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "fp_server_set_solver": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_float]),
    "fp_sim_snapshot": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "fp_mesh_voxelize": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_uint32)]),
    "fp_mesh_splat": (C.c_int, [C.c_int, C.c_void_p, C.c_uint32, C.c_double, C.c_void_p, C.POINTER(C.c_uint32)]),
    "fp_sim_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "fp_batch_snapshot": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "fp_batch_restore": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t]),
    "fp_snapshot_free": (None, [C.c_void_p]),
    "fp_server_snapshot": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "fp_server_restore": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t]),
    "fp_batch_read_solver": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(fp_solver_stats)]),
    "fp_batch_reserve_tiles": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "fp_server_last_error": (C.c_char_p, [C.c_void_p]),
    "fp_server_create": (C.c_int, [C.POINTER(fp_server_config), C.POINTER(C.c_void_p)]),
    "fp_server_destroy": (C.c_int, [C.c_void_p]),
    "fp_server_open": (C.c_int, [C.c_void_p, C.POINTER(fp_grid), C.c_float, C.c_int, C.POINTER(C.c_uint32)]),
    "fp_server_close": (C.c_int, [C.c_void_p, C.c_uint32]),
    "fp_server_session_state": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_int)]),
    "fp_server_submit": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(fp_frame), C.c_float, C.POINTER(C.c_uint64)]),
    "fp_server_poll": (C.c_int, [C.c_void_p, C.POINTER(fp_completion), C.c_uint32, C.POINTER(C.c_uint32), C.c_int]),
    "fp_server_drain": (C.c_int, [C.c_void_p, C.c_int]),
    "fp_server_read_stats": (C.c_int, [C.c_void_p, C.POINTER(fp_server_stats)]),
    "fp_server_session_stats": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(fp_stats)]),
    "fp_server_read_field": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_float), C.c_size_t]),
}
FP_COMPACT_MAX_IDS = 1 << 22

_lib = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Open libfirepro.so and declare every exported signature. Raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else Path(os.environ.get("FIREPRO_LIBRARY") or LIB_PATH)
    if not p.exists():
        raise RuntimeError(
            f"The CUDA library {p} is missing: build it with "
            "`python threejs-fire-pro_b200/build.py` (or __graft_entry__.build())."
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
