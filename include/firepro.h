/*
 * firepro.h — C ABI of the B200 sparse-brick fire simulation step.
 *
 * This is the drop-in boundary for Fire Pro's engine layer: one call per method of the
 * reference's `FluidSimulation` class (src/engine/FluidSimulation.ts), with plain structs
 * and pointers in place of WebGPU resources and JS objects. A Node-API addon or Python
 * ctypes binds these symbols one to one.
 *
 * Conventions
 *  - Every function returns an `int` status (FP_OK or a negative FP_E* code) and never
 *    throws across the ABI. `fp_last_error` gives the message of the latest failure,
 *    worded as the reference's thrown Error messages where one exists.
 *  - Validation happens before any state changes, as in the reference.
 *  - A handle is not thread safe: calls on one handle are serialised by the caller.
 *  - Caller buffers are borrowed for the duration of a call only.
 *  - All world-space quantities are meters, seconds and the reference's units.
 */
#ifndef FIREPRO_H
#define FIREPRO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FP_ABI_VERSION 1

/* Status codes. */
#define FP_OK 0
#define FP_EINVAL (-1)   /* invalid argument: the reference throws an Error */
#define FP_ENOMEM (-2)   /* device memory or the session's HBM budget is exhausted */
#define FP_ELIMIT (-3)   /* a reference limit is exceeded (tiles, storage) */
#define FP_EDEVICE (-4)  /* CUDA error; the message names the call */
#define FP_ETIMEOUT (-5) /* a bounded device wait gave up; the context stays usable */
#define FP_EUNSUPPORTED (-6) /* a grid option this build does not implement */

/* Storage precision of the pools. Arithmetic is FP32 in every mode. */
#define FP_PRECISION_FP32 0  /* plain FP32 storage everywhere (the drop-in) */
#define FP_PRECISION_MIXED 1 /* FP16 scalar pools (smoke, heat, lifetime, fuel), BF16 multigrid
                                levels above the finest; velocity, the finest pressure level,
                                divergence and expansion FP32; measured every step */

/* Source shapes (types.ts:248 SimulationSource.shape). */
#define FP_SHAPE_SPHERE 0
#define FP_SHAPE_BOX 1
#define FP_SHAPE_MESH 2

/* Force kinds (ForceFields.ts:64 — the index of the type name). */
#define FP_FORCE_WIND 0
#define FP_FORCE_TURBULENCE 1
#define FP_FORCE_VORTEX 2
#define FP_FORCE_RADIAL 3

/* The simulation lattice: replaces `SimulationGrid` (src/engine/types.ts:26-36), validated
 * as `FluidSimulation`'s constructor does (FluidSimulation.ts:359-379). */
typedef struct fp_grid {
  float voxel_size;        /* meters, [0.0001, 16] */
  int32_t velocity_divisor;/* 1, 2 or 4: velocity cells are that many fine cells a side */
  int32_t brick_size;      /* fine cells per brick side: 8, 16 or 32 */
  int32_t smoke_divisor;   /* 1, 2 or 4: smoke density on a grid that many times coarser */
  int32_t scalar_maccormack; /* bounded MacCormack scalar transport: 0 or 1 */
  int32_t precision;       /* FP_PRECISION_* */
  double voxel_budget;     /* grid.maxVoxels; 0 means the reference default 8,000,000 */
} fp_grid;

/* `SimulationSettings` (types.ts:235-243). */
typedef struct fp_settings {
  float buoyancy, smoke_weight, velocity_damping, cooling, dissipation, vorticity;
  uint32_t seed;
} fp_settings;

/* One flame response ramp: 2..8 knots [lifetime, response] (flame.ts:3, :66-85). */
typedef struct fp_flame_ramp {
  uint32_t count;
  float knots[8][2];
} fp_flame_ramp;

/* `FlameSettings` (flame.ts:7-13); ramps are smoke, heat, expansion. */
typedef struct fp_combustion {
  float lifespan, smoke_rate, heat_rate, expansion_rate;
  fp_flame_ramp ramps[3];
} fp_combustion;

/* `FuelSettings` (fuel.ts:7-14). */
typedef struct fp_fuel {
  int32_t enabled;
  float ignition_heat, burn_rate;
} fp_fuel;

/* `SimulationSource` (types.ts:246-268). `id` replaces the string id: a source whose id
 * was absent last step is new. A mesh source's surface samples arrive already splatted to
 * lattice cells, as the frame's `mesh_sources` records. */
typedef struct fp_source {
  uint64_t id;
  int32_t shape;            /* FP_SHAPE_* */
  float position[3];
  float size[3];            /* sphere radii or box half extents */
  float flame, heat_rate, smoke_rate, fuel_rate;
  float velocity[3];
  float velocity_response;
  float outward_speed;
  int32_t has_variation;    /* burst-only initial variation */
  float variation_period, variation_strength;
} fp_source;

/* `SimulationForce` (types.ts:284-293). When `targeted` is set the force reaches only the
 * union of the regions of `force_targets[first_target .. first_target+target_count)`. */
typedef struct fp_force {
  int32_t type;             /* FP_FORCE_* */
  float vector[3];          /* wind direction or vortex axis, unit length */
  float center[3];
  float strength, scale, lift, inward;
  int32_t targeted;
  uint32_t first_target, target_count;
} fp_force;

/* `SimulationCollider` (types.ts:271-281). Spheres and boxes use position/size/axes
 * (axes are the columns of the world rotation; spheres ignore them); mesh colliders use
 * a cell-center occupancy mask of dims[0]*dims[1]*dims[2] bits from lattice cell `lo`,
 * stored at collider_masks[mask_offset ...], one bit per cell, x fastest. */
typedef struct fp_collider {
  int32_t shape;            /* FP_SHAPE_SPHERE, FP_SHAPE_BOX or FP_SHAPE_MESH */
  float position[3];
  float size[3];
  float axes[3][3];
  int32_t lo[3];
  int32_t dims[3];
  uint32_t mask_offset;
} fp_collider;

/* `SimulationFrame` (types.ts:295-302). */
/* Mesh emission (a `SimulationSource` with `samples`, types.ts): the reference's
 * MeshSourceRasterizer (MeshSourceRasterizer.ts:64-167) splats the surface samples to lattice
 * cells on the host side of this boundary; each record is one field cell, 48 bytes as the
 * reference packs them (MeshSource, fluid-common.wgsl:53-57). A mesh source itself is an
 * fp_source of shape FP_SHAPE_MESH whose `position` is its samples' lower bound and `size`
 * their upper bound (the tiles around it, FluidSimulation.ts:879-893). */
typedef struct fp_mesh_source {
  int32_t cell[4];  /* lattice cell x, y, z; w unused */
  float scalar[4];  /* flame lifetime, heat rate, smoke rate, fuel rate */
  float motion[4];  /* velocity x response per axis, then the response (0: no coupling) */
} fp_mesh_source;

typedef struct fp_frame {
  fp_settings simulation;
  fp_combustion combustion;
  fp_fuel fuel;
  const fp_source* sources;
  uint32_t source_count;
  const fp_force* forces;
  uint32_t force_count;
  const fp_source* force_targets;
  uint32_t force_target_count;
  const fp_collider* colliders;
  uint32_t collider_count;
  const uint32_t* collider_masks;
  uint32_t collider_mask_words;
  const fp_mesh_source* mesh_sources; /* the step's mesh emission records (records 1..count) */
  uint32_t mesh_source_count;
  /* Mesh force targets (ForceFields.ts:115-179): a force target of FP_SHAPE_MESH (its
   * `position` the samples' lower bound, `size` the upper) covers the lattice cells
   * target_cells[3k .. 3k+2] for k in [first, first + count), with (first, count) =
   * target_cell_ranges[2t], [2t + 1] for target t of force_targets. */
  const int32_t* target_cells;
  uint32_t target_cell_count;         /* cells, three words each */
  const uint32_t* target_cell_ranges; /* two words per force target (force_target_count) */
} fp_frame;

/* What `FireSimulation.stats` and `FluidSimulation`'s getters report
 * (FireSimulation.ts:295-334; FluidSimulation.ts:230-245). */
typedef struct fp_stats {
  double time;              /* simulated seconds */
  uint64_t steps;
  uint32_t active_bricks;   /* at the latest measurement */
  uint32_t brick_cells;     /* fine cells per brick */
  int32_t pool_limited;     /* gridLimited */
  uint32_t pool_slots;      /* slots the pools hold */
  uint32_t used_slots;
  uint32_t tiles;           /* live tiles */
  uint32_t tile_capacity;   /* tile slots the per-brick tables hold */
  uint32_t failures;        /* failed allocations at the latest measurement */
  uint64_t memory_bytes;    /* device bytes this simulation owns */
  uint32_t last_vcycles;    /* V-cycles the latest pressure solve ran */
  double last_residual;     /* FP64 RMS residual after the latest solve (mixed mode), else -1 */
  uint64_t kernel_launches; /* kernels this simulation has launched since creation */
  uint64_t h2d_bytes;       /* host-to-device bytes the latest step copied (scene, parameters) */
  uint64_t d2h_bytes;       /* device-to-host bytes the latest step read back (its measurement) */
  double host_prepare_ms;   /* host time in fp_sim_step since creation, waits excluded */
  double host_wait_ms;      /* host time spent waiting for the previous step's measurement */
  double last_divergence;   /* post-projection RMS(h (div u - e)) / RMS(u) of that solve when measured, else -1 */
  uint64_t bricks_stepped;  /* computing bricks summed over the measured steps since creation or reset */
} fp_stats;

/* The latest step's pressure solve (`fp_sim_read_solver`). No reference counterpart: the
 * reference runs one V-cycle and measures nothing. Norms are FP64 sums on the GPU over the
 * finest level's pressure unknowns. */
#define FP_MAX_VCYCLES 16
typedef struct fp_solver_stats {
  uint32_t vcycles;                  /* V-cycles the solve ran */
  int32_t measured;                  /* the post-projection divergence was measured */
  double unknowns;                   /* unknown cells */
  double rhs_rms;                    /* RMS of the right-hand side h^2 (div u* - expansion) */
  double residual[FP_MAX_VCYCLES];   /* RMS residual / RMS right-hand side after each V-cycle */
  double divergence;                 /* RMS(h (div u - e)) / RMS(u) of the projected velocity over
                                        the interior unknowns, e the expansion rate the projection
                                        keeps (computeDivergence's source), or -1 */
} fp_solver_stats;

/* The bounds-checked build (`fp_sim_read_bounds`): the library built with `build.py --debug`
 * (lib/libfirepro_debug.so) checks every index its kernels read out of a table (a slot from a
 * brick entry or a neighbour record, a tile from the directory or its hash, a brick id from a
 * work list) against the table's size before using it. A bad index is counted, the first is
 * kept, and its access is skipped (it reads as "no slot"): no kernel traps or faults. No
 * reference counterpart (the reference relies on WebGPU's validation of its bindings). */
typedef struct fp_bounds {
  int32_t checked; /* 1: this library checks (the debug build); 0: the release build, nothing below */
  uint32_t count;  /* bad indices seen since the simulation was created or reset */
  int32_t site;    /* where the first was read: 1 neighbour record, 2 brick entry, 3 tile neighbour,
                      4 tile hash, 5 brick id of a work list */
  int32_t pad;
  int64_t index;   /* the first bad index */
  int64_t limit;   /* the size of its table */
} fp_bounds;

/* Device time of one phase of the step, accumulated while profiling is on: the restatement
 * of the reference's per-pass GPU timestamps (src/engine/GpuProfiler.ts:21-109). */
typedef struct fp_phase {
  char name[32];
  uint64_t launches;  /* kernels the phase launched */
  double ms;          /* device milliseconds, CUDA events on the simulation's stream */
  double voxels;      /* active voxels the phase covered, summed over steps */
} fp_phase;

/* Per-slot field arrays a test or debug view may copy out (`fp_sim_read_field`). Each
 * is [slot][channel][cell] in FP32, cells x fastest within a brick. */
#define FP_FIELD_VELOCITY 0   /* 3 channels: MAC face velocities u, v, w */
#define FP_FIELD_SCALARS 1    /* 4 channels: smoke, heat, flame lifetime, fuel */
#define FP_FIELD_EXPANSION 2  /* 1 channel */
#define FP_FIELD_PRESSURE 3   /* 1 channel: the latest solution */
#define FP_FIELD_DIVERGENCE 4 /* 1 channel: the Poisson right-hand side */
#define FP_FIELD_CURL 5       /* 4 channels: curl xyz and magnitude */
#define FP_FIELD_SMOKE 6      /* 1 channel on the coarse smoke grid (smoke_divisor d > 1): (B/d)^3
                                 cells a slot; with coarse smoke the smoke channel of
                                 FP_FIELD_SCALARS holds only the step's source production */

/* Integer tables a test may copy out (`fp_sim_read_table`), bit-exact against the oracle. */
#define FP_TABLE_ENTRIES 0     /* int32 per brick id: slot | FRESH (0x2000000), or -1 */
#define FP_TABLE_PAGES 1       /* int32 per brick id: the allocator's slot, or -1 */
#define FP_TABLE_STATE 2       /* uint32 per brick id */
#define FP_TABLE_ACTIVITY 3    /* uint32 per brick id, then per tile slot */
#define FP_TABLE_RECORDS 4     /* int32[28] per brick id: 27 neighbour entries + pressure flag */
#define FP_TABLE_FREE 5        /* uint32: free count, failures, then the free stack */
#define FP_TABLE_ACTIVE 6      /* uint32: count, then brick ids in ascending order */
#define FP_TABLE_SOLIDS 7      /* uint32 words per slot: one bit per fine cell */
#define FP_TABLE_TILES 8       /* int32[4] per tile slot: x, y, z, state (0 free 1 live 2 closing) */

typedef struct fp_sim fp_sim;

/* Library */
int fp_abi_version(void);
const char* fp_last_error(const fp_sim* sim); /* sim may be NULL: the thread's last error */

/* `FluidSimulation.create(device, grid)` (FluidSimulation.ts:419-475). `device` is the CUDA
 * ordinal. */
int fp_sim_create(const fp_grid* grid, int device, fp_sim** out);
/* `FluidSimulation.dispose()` (FluidSimulation.ts:1780-1802). */
int fp_sim_destroy(fp_sim* sim);
/* `FluidSimulation.reset()` (FluidSimulation.ts:768-779). */
int fp_sim_reset(fp_sim* sim);
/* The fields `FireSimulation.step` sets before each step (FireSimulation.ts:457-459):
 * cutoff, voxelBudget (maxVoxels), ground. */
int fp_sim_set_runtime(fp_sim* sim, float cutoff, double voxel_budget, int ground);
/* `FluidSimulation.step(frame, dt)` (FluidSimulation.ts:1367-1373): dt in (0, 1/30].
 * Enqueues the step on the simulation's CUDA stream; returns before it completes. */
int fp_sim_step(fp_sim* sim, const fp_frame* frame, float dt);
/* Hold at least `tiles` tile slots from now on, so that steps never stop to grow the
 * per-brick tables (the reference doubles them when the tiles outgrow them,
 * FluidSimulation.ts:629-678). Storage only: results do not change. No reference counterpart. */
int fp_sim_reserve_tiles(fp_sim* sim, uint32_t tiles);
/* The pressure solve: up to `vcycles` (1..FP_MAX_VCYCLES) V-cycles a step; after each, the
 * FP64 residual decides, and the solve stops once RMS residual <= tolerance x RMS right-hand
 * side (tolerance 0: run all of them). Every V-cycle after the first is a defect correction:
 * the finest level stays FP32 and the coarse correction comes from the residual of the current
 * iterate. The default (1, 0) is the reference's schedule (PressureSolver.ts:276-365). */
int fp_sim_set_solver(fp_sim* sim, int vcycles, float tolerance);
/* The latest step's solve (waits for the step's work). */
int fp_sim_read_solver(fp_sim* sim, fp_solver_stats* out);
/* The bounds-checked build's record of this simulation (waits for its work); `checked` 0 in
 * the release build. */
int fp_sim_read_bounds(fp_sim* sim, fp_bounds* out);

/* The pressure solve's schedule. The default (all fields zero) is the reference's V-cycle
 * (PressureSolver.ts:276-365): weighted Jacobi (omega 0.8), every level down to one cell a
 * tile, the first iterate from zero and 2 more sweeps before each restriction below the finest
 * level, 3 after each prolongation, 19 bottom iterations; the red-black fields are then
 * ignored. No reference counterpart for the rest:
 *  - FP_SMOOTHER_REDBLACK: red-black Gauss-Seidel, in place (the cells of a level with x + y + z
 *    even, then the odd ones; after a prolongation the odd ones first), on the `levels` finest
 *    levels: `pre_sweeps` before each restriction, `post_sweeps` after each prolongation and
 *    `bottom_sweeps` on the coarsest of them; every level starts from zero.
 *  - FP_KRYLOV_FCG: flexible conjugate gradients on the finest level with one V-cycle of the
 *    smoother as the preconditioner (either smoother): the first V-cycle gives the start, each
 *    later one a search direction made A-orthogonal to the previous one; the dot products and
 *    the residual norm are FP64 sums on the GPU. fp_sim_set_solver's `vcycles` then counts the
 *    V-cycles of the whole solve and its tolerance applies to the CG residual.
 * One launch steps simulations of one schedule: a batch step of simulations that differ fails. */
#define FP_SMOOTHER_JACOBI 0
#define FP_SMOOTHER_REDBLACK 1
#define FP_KRYLOV_NONE 0
#define FP_KRYLOV_FCG 1
typedef struct fp_solver_schedule {
  int32_t smoother;       /* FP_SMOOTHER_* */
  int32_t levels;         /* red-black: levels from the finest, 2 up to all of them; 0 = all */
  int32_t pre_sweeps;     /* red-black: 1..8 */
  int32_t post_sweeps;    /* red-black: 0..8 */
  int32_t bottom_sweeps;  /* red-black: 1..64 */
  int32_t krylov;         /* FP_KRYLOV_* */
  /* 0: the reference's multigrid topology, rebuilt for fresh bricks each step (a brick's cells
   * keep the open sides they had when a neighbour brick without a slot was granted one, so near
   * a collider the solve and the projection may disagree on which faces are solid);
   * 1: every brick's topology rebuilt each step, so the solve's operator always sees the solids
   * the projection sees (what the accuracy gate needs near colliders). */
  int32_t topology;
} fp_solver_schedule;
int fp_sim_set_schedule(fp_sim* sim, const fp_solver_schedule* schedule);
/* ---- Volume rendering: a headless restatement of the renderer's compute passes and camera
 * march (lighting.wgsl smoothSmoke/buildOccupancy/buildLighting, volume-slices.wgsl
 * buildSlices, volume-march.wgsl fireProMarch, scene-volume.wgsl fireProSceneVolume with an
 * optional scene depth buffer and half-resolution slices, fire-emission.wgsl,
 * volume-reconstruction.wgsl, blackbody.ts). The image is linear radiance and opacity,
 * row-major from the top-left pixel, four floats a pixel. */
typedef struct fp_camera {
  float inverse_view_projection[16]; /* clip to world, column-major (the WGSL mat4x4f's columns) */
  uint32_t width, height;            /* pixels */
  float time;                        /* seconds: the jitter's frame is floor(time x 60) */
  /* The scene's depth buffer, host memory (width x height floats, clip-space z from 0 near to 1
   * far, rows from the top): a ray ends where the scene's geometry is (fireProSceneDistance,
   * volume-march.wgsl:76-89). Null: nothing in front of the volume. */
  const float* scene_depth;
  /* 1: a half-resolution pass first records the march at 8 depths, and each pixel resumes from
   * the last one in front of the scene (scene-volume.wgsl:146-160, volume-slices.wgsl). */
  uint32_t half_resolution;
} fp_camera;
typedef struct fp_render_settings {
  float optical[4];       /* smoke extinction, fire brightness, shadow extinction, anisotropy g */
  float light[4];         /* directional light direction (towards the light), intensity */
  float smoke[4];         /* smoke albedo RGB, hot-soot glow */
  float fire[4];          /* fire tint RGB, temperature in kelvin */
  float scene_light[3];   /* the scene's light colour on the sun term */
  float ambient_light[3]; /* ambient light on the smoke */
  float flame_opacity;
  uint32_t shadow_samples;   /* samples towards the sun per lighting texel (the reference: 32) */
  uint32_t ray_steps;        /* the march's step count over the ray's length in the box (256) */
  int32_t filter;            /* 0 trilinear, 1 quadratic B-spline, 2 cubic B-spline (flame only) */
  uint32_t lighting_divisor; /* fine cells per lighting texel side: 1, 2 or 4 (4) */
} fp_render_settings;
/* Render the simulation's latest state into `rgba` (host, width x height x 4 floats). */
int fp_sim_render(fp_sim* sim, const fp_camera* camera, const fp_render_settings* settings, float* rgba);
/* The same into device memory of this simulation's GPU (width x height x 4 floats); enqueued
 * on the simulation's stream. */
int fp_sim_render_device(fp_sim* sim, const fp_camera* camera, const fp_render_settings* settings, float* rgba);
/* Scene lights (collectLights, scene-lights.wgsl:37-106; replaces SceneLights.sample's GPU
 * pass, SceneLights.ts:150-214): every brick that computed in the latest step samples its
 * cells on a 4^3 lattice and adds, to the anchor nearest the brick's centre (height above an
 * anchor counts a quarter; ties go to the first), the luminance of their emission, its
 * luminance-weighted offset from the anchor and its RGB. `anchors` holds `anchor_count`
 * world positions (3 floats each); `sums` receives 8 floats per anchor (luminance, offset
 * xyz, RGB, 0), the totals SceneLights.apply turns into lights. Synchronous. With coarse smoke a
 * sample's density is the coarse grid's, trilinear at the cell's centre. */
int fp_sim_collect_lights(fp_sim* sim, const fp_render_settings* settings, const float* anchors,
                          uint32_t anchor_count, float* sums);
/* Wait for the simulation's queued work. */
int fp_sim_synchronize(fp_sim* sim);
/* Stats (waits for the latest step's measurement). */
int fp_sim_stats(fp_sim* sim, fp_stats* out);
/* Copy a per-slot field (FP_FIELD_*) into `host`, `bytes` long: slots*channels*cells*4. */
int fp_sim_read_field(fp_sim* sim, int field, float* host, size_t bytes);
/* Copy an integer table (FP_TABLE_*) into `host`; `*bytes` in: capacity, out: bytes written. */
int fp_sim_read_table(fp_sim* sim, int table, void* host, size_t* bytes);
/* `FluidSimulation.readBricks()` (FluidSimulation.ts:1749-1779): the world boxes of the
 * bricks that hold a slot, six floats each (min xyz, max xyz). `*count` in: capacity in
 * boxes, out: boxes written (or needed, with FP_ELIMIT). */
int fp_sim_read_bricks(fp_sim* sim, float* boxes, uint32_t* count);
/* Session snapshot and restore (no reference counterpart: the reference's document,
 * editor/document.ts:60-61, saves settings, not state). `fp_sim_snapshot` waits for the
 * simulation's work and copies its whole state between steps (host tables, device pools,
 * tables and multigrid levels) into one blob the library allocates in host memory:
 * `*blob` and `*bytes` receive it; release it with fp_snapshot_free. `fp_sim_restore` puts
 * a blob back into a simulation of the same grid (another simulation, another device, or the
 * same one rewound); the restored simulation then steps bit for bit as the original would
 * have. A blob of another grid, truncated or inconsistent is FP_EINVAL and changes nothing.
 * The blob is for this library build on this host architecture only. */
int fp_sim_snapshot(fp_sim* sim, void** blob, size_t* bytes);
int fp_sim_restore(fp_sim* sim, const void* blob, size_t bytes);
void fp_snapshot_free(void* blob);
/* The cudaStream_t the simulation enqueues on, for callers that order their own work after
 * it or record events against it. No reference counterpart: WebGPU has one queue. */
int fp_sim_stream(fp_sim* sim, void** stream);
/* Start (clearing the totals) or stop per-phase device timing: `GpuProfiler` of the
 * reference (src/engine/GpuProfiler.ts:21-68) with CUDA events. */
int fp_sim_set_profiling(fp_sim* sim, int enabled);
/* The per-phase totals since profiling started. `*count` in: capacity, out: phases. */
int fp_sim_read_profile(fp_sim* sim, fp_phase* phases, uint32_t* count);

/* ---- Batches: many independent simulations stepped by one launch.
 * No reference counterpart: the reference steps one `FluidSimulation` per call. A batch owns
 * one CUDA stream; its simulations share a brick size and may differ in everything else
 * (voxel size, budget, scene, dt). `fp_batch_step` steps any subset of them with one upload
 * and one CUDA graph whose kernels cover every listed simulation's bricks; each simulation's
 * results are bit-identical to stepping it alone. A simulation is named by the id
 * `fp_batch_add` returned. Errors of a step name the simulation's position in `ids`. */
typedef struct fp_batch fp_batch;
const char* fp_batch_last_error(const fp_batch* batch);
int fp_batch_create(int device, int brick_size, fp_batch** out);
int fp_batch_destroy(fp_batch* batch);
/* Add a simulation of `grid` (validated as by fp_sim_create); `*id` receives its id. */
int fp_batch_add(fp_batch* batch, const fp_grid* grid, uint32_t* id);
/* Remove a simulation and free its device memory; its id may be reused. */
int fp_batch_remove(fp_batch* batch, uint32_t id);
int fp_batch_reset(fp_batch* batch, uint32_t id);
int fp_batch_set_runtime(fp_batch* batch, uint32_t id, float cutoff, double voxel_budget, int ground);
/* As fp_sim_reserve_tiles. */
int fp_batch_reserve_tiles(fp_batch* batch, uint32_t id, uint32_t tiles);
/* As fp_sim_set_solver and fp_sim_read_solver. A launch runs as many V-cycles as its most
 * demanding simulation asks for; each simulation stops at its own limit or tolerance. */
int fp_batch_set_solver(fp_batch* batch, uint32_t id, int vcycles, float tolerance);
int fp_batch_read_solver(fp_batch* batch, uint32_t id, fp_solver_stats* out);
/* As fp_sim_snapshot and fp_sim_restore, for a simulation of the batch. */
int fp_batch_snapshot(fp_batch* batch, uint32_t id, void** blob, size_t* bytes);
int fp_batch_restore(fp_batch* batch, uint32_t id, const void* blob, size_t bytes);
/* As fp_sim_set_schedule; the simulations of one fp_batch_step must share a schedule. */
int fp_batch_set_schedule(fp_batch* batch, uint32_t id, const fp_solver_schedule* schedule);
/* Step the `count` simulations `ids` (distinct) with frames[i] and dts[i], in one launch. */
int fp_batch_step(fp_batch* batch, const uint32_t* ids, const fp_frame* frames, const float* dts, uint32_t count);
int fp_batch_synchronize(fp_batch* batch);
int fp_batch_stats(fp_batch* batch, uint32_t id, fp_stats* out);
int fp_batch_read_field(fp_batch* batch, uint32_t id, int field, float* host, size_t bytes);
int fp_batch_read_table(fp_batch* batch, uint32_t id, int table, void* host, size_t* bytes);
int fp_batch_stream(fp_batch* batch, void** stream);
int fp_batch_set_profiling(fp_batch* batch, int enabled);
int fp_batch_read_profile(fp_batch* batch, fp_phase* phases, uint32_t* count);
/* Device bytes a simulation of `grid` holds once created: the admission estimate. */
int fp_grid_memory_bytes(const fp_grid* grid, uint64_t* bytes);
/* The tile reservation a server gives a session of `grid`: one tile slot per four bricks of
 * its budget, a power of two (at least 16). */
int fp_grid_reserved_tiles(const fp_grid* grid, uint32_t* tiles);

/* ---- Serving: sessions admitted by device-memory budget, their step requests batched as
 * they arrive. No reference counterpart. A server owns a batch and a scheduler thread: every
 * launch steps each live session that has a request queued (the oldest one), so requests
 * that arrive while a launch runs go into the next; sessions waiting for admission join as
 * memory and session slots free up. A session's steps run in submission order; a result is
 * the same alone and among any other sessions (bit for bit). Times are milliseconds on the
 * server's steady clock since creation. */
typedef struct fp_server fp_server;
typedef struct {
  int device;
  int brick_size;          /* 8, 16 or 32, the same for every session */
  uint64_t memory_budget;  /* admission: the sessions' device bytes (fp_grid_memory_bytes) */
  uint32_t max_sessions;   /* live sessions at most */
} fp_server_config;
#define FP_SESSION_WAITING 0 /* queued for admission */
#define FP_SESSION_LIVE 1
#define FP_SESSION_CLOSING 2 /* closed by the caller, its queued steps still run */
#define FP_SESSION_CLOSED 3
#define FP_SESSION_FAILED 4  /* admission failed (device memory): see fp_server_last_error */
typedef struct {
  uint32_t session;
  int status;             /* FP_OK, or the step's error */
  uint64_t ticket;        /* fp_server_submit's ticket */
  uint64_t step;          /* the session's steps after this one */
  uint32_t active_bricks; /* computing bricks of this step */
  uint32_t batch_size;    /* sessions in the launch that ran it */
  double submit_ms, done_ms;
} fp_completion;
typedef struct {
  uint32_t live, waiting, queued_steps;
  uint64_t memory_bytes;     /* admitted sessions' admission estimate */
  uint64_t device_bytes;     /* their device memory now */
  uint64_t steps_done, launches;
  double voxel_steps;        /* sum over completed steps of computing bricks x cells */
  double elapsed_ms;         /* since creation */
  double latency_p50_ms, latency_p99_ms; /* submit to done, over completed steps */
  double mean_batch;         /* sessions per launch */
} fp_server_stats;
const char* fp_server_last_error(const fp_server* server);
int fp_server_create(const fp_server_config* config, fp_server** out);
/* Stops the scheduler after the launched steps complete; queued steps are dropped. */
int fp_server_destroy(fp_server* server);
/* Open a session of `grid` with the runtime fields of fp_sim_set_runtime; it waits for
 * admission (FP_SESSION_WAITING) unless memory and a slot are free now. FP_ELIMIT when the
 * grid alone exceeds the memory budget. Every session of a server shares the velocity
 * divisor of the first one opened: another divisor is FP_EINVAL. */
int fp_server_open(fp_server* server, const fp_grid* grid, float cutoff, int ground, uint32_t* session);
/* The session leaves once its queued steps have run; its memory then returns to the budget. */
int fp_server_close(fp_server* server, uint32_t session);
int fp_server_session_state(fp_server* server, uint32_t session, int* state);
/* Queue one step of `session` (the frame and every array it points into are copied; dt as
 * fp_sim_step). The frame's full check (flame ramps, mesh arrays) runs when its launch is
 * built: a frame that fails it completes with that status alone, the other sessions' steps of
 * the launch run. */
int fp_server_submit(fp_server* server, uint32_t session, const fp_frame* frame, float dt, uint64_t* ticket);
/* Completed steps, oldest first: up to `capacity` into `out`, `*count` written. Waits up to
 * `wait_ms` for the first one when none is ready. */
int fp_server_poll(fp_server* server, fp_completion* out, uint32_t capacity, uint32_t* count, int wait_ms);
/* Wait until every queued step has completed (or `wait_ms` passed: FP_ETIMEOUT). */
int fp_server_drain(fp_server* server, int wait_ms);
int fp_server_read_stats(fp_server* server, fp_server_stats* out);
/* A live session's stats (as fp_sim_stats), as of its latest measured step. */
int fp_server_session_stats(fp_server* server, uint32_t session, fp_stats* out);
/* A live session's snapshot (as fp_sim_snapshot) once its queued steps have run (FP_EINVAL
 * while any is queued or running), and a snapshot restored into a live session of the same
 * grid with no steps queued: a server evicts a session to host memory by snapshot and close,
 * and brings it back by open and restore. */
int fp_server_snapshot(fp_server* server, uint32_t session, void** blob, size_t* bytes);
int fp_server_restore(fp_server* server, uint32_t session, const void* blob, size_t bytes);
/* The pressure solve of every session admitted from now on (as fp_sim_set_schedule and
 * fp_sim_set_solver; by default the reference's single V-cycle). One launch runs one schedule,
 * so set it before opening the sessions it should apply to. */
int fp_server_set_solver(fp_server* server, const fp_solver_schedule* schedule, int vcycles, float tolerance);
/* A live session's field (as fp_sim_read_field), between its steps. */
int fp_server_read_field(fp_server* server, uint32_t session, int field, float* host, size_t bytes);

/* ---- Mesh colliders and mesh emitters on the GPU: the reference's host-side passes that turn
 * a triangle mesh into what fp_frame takes (a collider's occupancy bits, an emitter's records).
 * Arithmetic is FP64 as the reference's JavaScript numbers are. */
typedef struct fp_mesh {
  const float* positions;   /* vertex_count x 3: the geometry's local vertex positions */
  uint32_t vertex_count;
  const uint32_t* indices;  /* index_count indices, three a triangle; NULL: the vertices in threes */
  uint32_t index_count;
} fp_mesh;
/* Collider.meshMask (handles.ts:299-325) with MeshCollider.voxelize (MeshCollider.ts:85-167):
 * the occupancy of the lattice cells of `spacing` meters from the world origin whose centres the
 * closed mesh, placed by `world` (4x4 column-major, Matrix4.elements), encloses: a box one cell
 * beyond the mesh's transformed bounds, each column a ray along +z whose crossings' winding
 * decides. Writes the box's first cell `lo` and `dims`; `*word_count` receives the words its
 * bits take (one bit a cell, x fastest, fp_collider's mask layout) and, when `words` is not NULL
 * and `*word_count` held at least that many on entry, the bits. The caller has checked the mesh
 * as MeshCollider's constructor does (closed, consistently wound). */
int fp_mesh_voxelize(int device, const fp_mesh* mesh, const double world[16], double spacing, int32_t lo[3],
                     int32_t dims[3], uint32_t* words, uint32_t* word_count);
/* A mesh emitter's surface samples as `Emitter.source` gives them (handles.ts:143-184): world
 * positions and weights (MeshSurface, MeshSurface.ts:15-103), the mesh's surface area, the
 * source's rates and velocity. */
typedef struct fp_mesh_emitter {
  const double* samples;   /* sample_count x 3 world positions */
  const double* weights;   /* sample_count */
  uint32_t sample_count;
  double surface_area;
  double flame, heat_rate, smoke_rate, fuel_rate;
  double velocity[3];
  double velocity_response;
} fp_mesh_emitter;
/* MeshSourceRasterizer.prepare (MeshSourceRasterizer.ts:64-167): every sample splats its weight
 * x the surface area over the 8 lattice cells around it (trilinear, cells of `spacing`, divided
 * by the mean face area); per emitter a cell's coverage is capped at 1 and scales its rates;
 * emitters sum (the flame takes the maximum). `records` receives one fp_mesh_source per covered
 * cell, ascending by (x, y, z) (fp_frame.mesh_sources takes them as they are); `*count` in:
 * capacity, out: records (FP_ELIMIT and the number needed when they do not fit). The reference's
 * limit of two million cell visits and its errors apply. */
int fp_mesh_splat(int device, const fp_mesh_emitter* emitters, uint32_t emitter_count, double spacing,
                  fp_mesh_source* records, uint32_t* count);

/* Most ids fp_compact_ids_noalloc accepts in one call. */
#define FP_COMPACT_MAX_IDS (1u << 22)

/* Ordered compaction that allocates nothing. No counterpart in the reference: it is the
 * step's own ranking of computing bricks (ascending ids of the nonzero flags, as the
 * allocation lists them) offered to callers that cannot allocate device memory where they
 * call it, such as a renderer's frame loop that must not stall on cudaMalloc/cudaFree, a host
 * that owns all device memory through its own allocator or budget, or code inside a stream
 * capture.
 *   flags  device array of n words; a nonzero word keeps its index
 *   ids    device array of at least n words: the kept indices, ascending
 *   count  device word: how many were kept
 *   stream a cudaStream_t, or NULL for the default stream; the call only enqueues
 * n may be at most FP_COMPACT_MAX_IDS; larger n returns FP_ELIMIT and launches nothing.
 * Scratch is a 64 KB array inside the library that every GPU loading it holds until exit.
 * The first call on a device looks up that array's address with the device current; make
 * that first call before any stream capture. The address is kept for the process: after a
 * cudaDeviceReset (or any teardown of the device's primary context) it is stale, so do not
 * call this entry point again in that process. All calls share the array, so calls whose
 * work overlaps on the GPU race; order them on one stream. */
int fp_compact_ids_noalloc(const uint32_t* flags, uint32_t n, uint32_t* ids, uint32_t* count, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FIREPRO_H */
