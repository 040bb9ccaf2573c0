// extern "C" entry points of include/firepro.h. Each validates its arguments, forwards to
// the host engine and turns any failure into a status code with a message; nothing throws
// across the ABI. A single simulation is an Engine stepped by a Stepper of its own; a batch
// shares one Stepper among many Engines.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/firepro.h"
#include "fp_engine.hpp"
#include "fp_error.h"

struct fp_sim {
  fp::Stepper* stepper;
  fp::Engine* engine;
};

struct fp_batch {
  fp::Stepper* stepper;
  std::vector<fp::Engine*> sims;  // by id; null where removed
  std::string error;
  // per-step scratch
  std::vector<fp::Engine*> stepSims;
  std::vector<const fp_frame*> stepFrames;
};

static thread_local std::string g_error;

static int failed(const std::string& message, int code) {
  g_error = message;
  return code;
}

int fp_set_error(int code, const std::string& message) { return failed(message, code); }

// The grid validation of FluidSimulation's constructor (FluidSimulation.ts:359-379).
static int validateGrid(const fp_grid* grid) {
  if (!std::isfinite(grid->voxel_size) || grid->voxel_size < 0.0001f || grid->voxel_size > 16.f)
    return failed("voxelSize must be from 0.0001 to 16 meters.", FP_EINVAL);
  int vd = grid->velocity_divisor;
  if (vd != 1 && vd != 2 && vd != 4) return failed("velocityDivisor must be 1, 2 or 4.", FP_EINVAL);
  int bs = grid->brick_size;
  if (bs != 8 && bs != 16 && bs != 32) return failed("brickSize must be 8, 16 or 32 fine cells.", FP_EINVAL);
  if (grid->scalar_maccormack != 0 && grid->scalar_maccormack != 1)
    return failed("scalarMacCormack must be a boolean.", FP_EINVAL);
  int sd = grid->smoke_divisor;
  if (sd != 1 && sd != 2 && sd != 4) return failed("smokeDivisor must be 1, 2 or 4.", FP_EINVAL);
  if (grid->precision != FP_PRECISION_FP32 && grid->precision != FP_PRECISION_MIXED)
    return failed("precision must be FP_PRECISION_FP32 or FP_PRECISION_MIXED.", FP_EINVAL);
  if (!(grid->voxel_budget >= 0) || !std::isfinite(grid->voxel_budget))
    return failed("voxel_budget must be a finite, nonnegative voxel count.", FP_EINVAL);
  return FP_OK;
}

static bool frameArraysValid(const fp_frame* f) {
  return !((f->source_count && !f->sources) || (f->force_count && !f->forces) ||
           (f->collider_count && !f->colliders) || (f->force_target_count && !f->force_targets) ||
           (f->collider_mask_words && !f->collider_masks) || (f->mesh_source_count && !f->mesh_sources) ||
           (f->target_cell_count && (!f->target_cells || !f->target_cell_ranges)));
}

static fp::Stepper* newStepper(int device, int brickSize, int& rc) {
  fp::Stepper* st = new (std::nothrow) fp::Stepper(device, brickSize);
  if (!st) {
    rc = failed("out of host memory", FP_ENOMEM);
    return nullptr;
  }
  rc = st->initialize();
  if (rc) {
    g_error = st->error();
    delete st;
    return nullptr;
  }
  return st;
}

extern "C" {

int fp_abi_version(void) { return FP_ABI_VERSION; }

const char* fp_last_error(const fp_sim* sim) {
  if (sim && sim->engine) return sim->engine->error().c_str();
  return g_error.c_str();
}

int fp_sim_create(const fp_grid* grid, int device, fp_sim** out) {
  if (!grid || !out) return failed("fp_sim_create needs a grid and an output handle.", FP_EINVAL);
  *out = nullptr;
  int rc = validateGrid(grid);
  if (rc) return rc;
  fp::Stepper* st = newStepper(device, grid->brick_size, rc);
  if (!st) return rc;
  fp::Engine* e = new (std::nothrow) fp::Engine(*grid, st);
  if (!e) {
    delete st;
    return failed("out of host memory", FP_ENOMEM);
  }
  rc = e->initialize();
  if (rc) {
    g_error = e->error();
    delete e;
    delete st;
    return rc;
  }
  fp_sim* s = new (std::nothrow) fp_sim{st, e};
  if (!s) {
    delete e;
    delete st;
    return failed("out of host memory", FP_ENOMEM);
  }
  *out = s;
  return FP_OK;
}

int fp_sim_destroy(fp_sim* sim) {
  if (!sim) return FP_OK;
  delete sim->engine;
  delete sim->stepper;
  delete sim;
  return FP_OK;
}

int fp_sim_reset(fp_sim* sim) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  return sim->engine->reset();
}

int fp_sim_set_runtime(fp_sim* sim, float cutoff, double voxel_budget, int ground) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  return sim->engine->setRuntime(cutoff, voxel_budget, ground);
}

int fp_sim_step(fp_sim* sim, const fp_frame* frame, float dt) {
  if (!sim || !frame) return failed("fp_sim_step needs a simulation and a frame.", FP_EINVAL);
  if (!frameArraysValid(frame)) return sim->engine->fail(FP_EINVAL, "frame arrays are null but their counts are not");
  fp::Engine* e = sim->engine;
  int rc = sim->stepper->step(&e, &frame, &dt, 1);
  if (rc) e->fail(rc, sim->stepper->error());
  return rc;
}

int fp_sim_reserve_tiles(fp_sim* sim, uint32_t tiles) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  return sim->engine->reserveTiles(tiles);
}

int fp_sim_render(fp_sim* sim, const fp_camera* camera, const fp_render_settings* settings, float* rgba) {
  if (!sim || !camera || !settings || !rgba)
    return failed("fp_sim_render needs a simulation, a camera, settings and an image.", FP_EINVAL);
  return sim->engine->render(*camera, *settings, nullptr, rgba);
}

int fp_sim_render_device(fp_sim* sim, const fp_camera* camera, const fp_render_settings* settings, float* rgba) {
  if (!sim || !camera || !settings || !rgba)
    return failed("fp_sim_render_device needs a simulation, a camera, settings and an image.", FP_EINVAL);
  return sim->engine->render(*camera, *settings, rgba, nullptr);
}

int fp_sim_collect_lights(fp_sim* sim, const fp_render_settings* settings, const float* anchors,
                          uint32_t anchor_count, float* sums) {
  if (!sim || !settings || (anchor_count && (!anchors || !sums)))
    return failed("fp_sim_collect_lights needs a simulation, settings, anchors and sums.", FP_EINVAL);
  return sim->engine->collectLights(*settings, anchors, anchor_count, sums);
}

int fp_sim_set_solver(fp_sim* sim, int vcycles, float tolerance) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  return sim->engine->setSolver(vcycles, tolerance);
}

int fp_sim_set_schedule(fp_sim* sim, const fp_solver_schedule* schedule) {
  if (!sim || !schedule) return failed("fp_sim_set_schedule needs a simulation and a schedule.", FP_EINVAL);
  return sim->engine->setSchedule(*schedule);
}

int fp_sim_read_solver(fp_sim* sim, fp_solver_stats* out) {
  if (!sim || !out) return failed("fp_sim_read_solver needs a simulation and an output.", FP_EINVAL);
  return sim->engine->readSolver(out);
}

int fp_sim_read_bounds(fp_sim* sim, fp_bounds* out) {
  if (!sim || !out) return failed("fp_sim_read_bounds needs a simulation and an output.", FP_EINVAL);
  return sim->engine->readBounds(out);
}

int fp_sim_synchronize(fp_sim* sim) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  int rc = sim->stepper->synchronize();
  if (rc) sim->engine->fail(rc, sim->stepper->error());
  return rc;
}

int fp_sim_stats(fp_sim* sim, fp_stats* out) {
  if (!sim || !out) return failed("fp_sim_stats needs a simulation and an output.", FP_EINVAL);
  return sim->engine->stats(out);
}

int fp_sim_read_field(fp_sim* sim, int field, float* host, size_t bytes) {
  if (!sim || !host) return failed("fp_sim_read_field needs a simulation and a buffer.", FP_EINVAL);
  return sim->engine->readField(field, host, bytes);
}

int fp_sim_read_table(fp_sim* sim, int table, void* host, size_t* bytes) {
  if (!sim || !bytes) return failed("fp_sim_read_table needs a simulation and a size.", FP_EINVAL);
  return sim->engine->readTable(table, host, bytes);
}

// A snapshot blob in malloc'd host memory for the caller (fp_snapshot_free releases it).
static int handOut(std::vector<uint8_t>& v, void** blob, size_t* bytes) {
  void* p = std::malloc(v.size() ? v.size() : 1);
  if (!p) return failed("out of host memory for the snapshot", FP_ENOMEM);
  std::memcpy(p, v.data(), v.size());
  *blob = p;
  *bytes = v.size();
  return FP_OK;
}

int fp_sim_snapshot(fp_sim* sim, void** blob, size_t* bytes) {
  if (!sim || !blob || !bytes) return failed("fp_sim_snapshot needs a simulation and outputs.", FP_EINVAL);
  std::vector<uint8_t> v;
  int rc = sim->engine->snapshot(v);
  return rc ? rc : handOut(v, blob, bytes);
}

int fp_sim_restore(fp_sim* sim, const void* blob, size_t bytes) {
  if (!sim || !blob) return failed("fp_sim_restore needs a simulation and a snapshot.", FP_EINVAL);
  return sim->engine->restore(static_cast<const uint8_t*>(blob), bytes);
}

void fp_snapshot_free(void* blob) { std::free(blob); }

int fp_sim_read_bricks(fp_sim* sim, float* boxes, uint32_t* count) {
  if (!sim || !count) return failed("fp_sim_read_bricks needs a simulation and a count.", FP_EINVAL);
  return sim->engine->readBricks(boxes, count);
}

int fp_sim_stream(fp_sim* sim, void** stream) {
  if (!sim || !stream) return failed("fp_sim_stream needs a simulation and an output.", FP_EINVAL);
  *stream = (void*)sim->stepper->stream();
  return FP_OK;
}

int fp_sim_set_profiling(fp_sim* sim, int enabled) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  int rc = sim->stepper->setProfiling(enabled != 0);
  if (rc) sim->engine->fail(rc, sim->stepper->error());
  return rc;
}

int fp_sim_read_profile(fp_sim* sim, fp_phase* phases, uint32_t* count) {
  if (!sim || !count) return failed("fp_sim_read_profile needs a simulation and a count.", FP_EINVAL);
  int rc = sim->stepper->readProfile(phases, count);
  if (rc) sim->engine->fail(rc, sim->stepper->error());
  return rc;
}

// ---------------------------------------------------------------------------- batches

const char* fp_batch_last_error(const fp_batch* batch) { return batch ? batch->error.c_str() : g_error.c_str(); }

static int batchFail(fp_batch* b, int code, const std::string& message) {
  b->error = message;
  g_error = message;
  return code;
}

static fp::Engine* batchSim(fp_batch* b, uint32_t id) { return id < b->sims.size() ? b->sims[id] : nullptr; }

int fp_batch_create(int device, int brick_size, fp_batch** out) {
  if (!out) return failed("fp_batch_create needs an output handle.", FP_EINVAL);
  *out = nullptr;
  if (brick_size != 8 && brick_size != 16 && brick_size != 32)
    return failed("a batch's brickSize must be 8, 16 or 32.", FP_EINVAL);
  int rc;
  fp::Stepper* st = newStepper(device, brick_size, rc);
  if (!st) return rc;
  fp_batch* b = new (std::nothrow) fp_batch{};
  if (!b) {
    delete st;
    return failed("out of host memory", FP_ENOMEM);
  }
  b->stepper = st;
  *out = b;
  return FP_OK;
}

int fp_batch_destroy(fp_batch* batch) {
  if (!batch) return FP_OK;
  for (fp::Engine* e : batch->sims) delete e;
  delete batch->stepper;
  delete batch;
  return FP_OK;
}

int fp_batch_add(fp_batch* batch, const fp_grid* grid, uint32_t* id) {
  if (!batch || !grid || !id) return failed("fp_batch_add needs a batch, a grid and an output id.", FP_EINVAL);
  int rc = validateGrid(grid);
  if (rc) return batchFail(batch, rc, g_error);
  if (grid->brick_size != batch->stepper->brickSize())
    return batchFail(batch, FP_EINVAL, "brickSize differs from the batch's.");
  fp::Engine* e = new (std::nothrow) fp::Engine(*grid, batch->stepper);
  if (!e) return batchFail(batch, FP_ENOMEM, "out of host memory");
  if ((rc = e->initialize())) {
    std::string m = e->error();
    delete e;
    return batchFail(batch, rc, m);
  }
  uint32_t slot = 0;
  while (slot < batch->sims.size() && batch->sims[slot]) slot++;
  if (slot == batch->sims.size()) batch->sims.push_back(nullptr);
  batch->sims[slot] = e;
  *id = slot;
  return FP_OK;
}

int fp_batch_remove(fp_batch* batch, uint32_t id) {
  if (!batch) return failed("null batch", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = batch->stepper->consume();
  if (rc) return batchFail(batch, rc, batch->stepper->error());
  delete e;
  batch->sims[id] = nullptr;
  return FP_OK;
}

int fp_batch_reset(fp_batch* batch, uint32_t id) {
  if (!batch) return failed("null batch", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->reset();
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_set_runtime(fp_batch* batch, uint32_t id, float cutoff, double voxel_budget, int ground) {
  if (!batch) return failed("null batch", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->setRuntime(cutoff, voxel_budget, ground);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_reserve_tiles(fp_batch* batch, uint32_t id, uint32_t tiles) {
  if (!batch) return failed("null batch", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->reserveTiles(tiles);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_set_solver(fp_batch* batch, uint32_t id, int vcycles, float tolerance) {
  if (!batch) return failed("null batch", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->setSolver(vcycles, tolerance);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_snapshot(fp_batch* batch, uint32_t id, void** blob, size_t* bytes) {
  if (!batch || !blob || !bytes) return failed("fp_batch_snapshot needs a batch and outputs.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  std::vector<uint8_t> v;
  int rc = e->snapshot(v);
  if (rc) return batchFail(batch, rc, e->error());
  return handOut(v, blob, bytes);
}

int fp_batch_restore(fp_batch* batch, uint32_t id, const void* blob, size_t bytes) {
  if (!batch || !blob) return failed("fp_batch_restore needs a batch and a snapshot.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->restore(static_cast<const uint8_t*>(blob), bytes);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_set_schedule(fp_batch* batch, uint32_t id, const fp_solver_schedule* schedule) {
  if (!batch || !schedule) return failed("fp_batch_set_schedule needs a batch and a schedule.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->setSchedule(*schedule);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_read_solver(fp_batch* batch, uint32_t id, fp_solver_stats* out) {
  if (!batch || !out) return failed("fp_batch_read_solver needs a batch and an output.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->readSolver(out);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_step(fp_batch* batch, const uint32_t* ids, const fp_frame* frames, const float* dts, uint32_t count) {
  if (!batch) return failed("null batch", FP_EINVAL);
  if (count && (!ids || !frames || !dts)) return batchFail(batch, FP_EINVAL, "fp_batch_step needs ids, frames and dts.");
  batch->stepSims.assign(count, nullptr);
  batch->stepFrames.assign(count, nullptr);
  for (uint32_t i = 0; i < count; i++) {
    fp::Engine* e = batchSim(batch, ids[i]);
    if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(ids[i]));
    for (uint32_t j = 0; j < i; j++)
      if (ids[j] == ids[i]) return batchFail(batch, FP_EINVAL, "simulation " + std::to_string(ids[i]) + " listed twice");
    if (!frameArraysValid(&frames[i]))
      return batchFail(batch, FP_EINVAL,
                       "simulation " + std::to_string(i) + ": frame arrays are null but their counts are not");
    batch->stepSims[i] = e;
    batch->stepFrames[i] = &frames[i];
  }
  int rc = batch->stepper->step(batch->stepSims.data(), batch->stepFrames.data(), dts, (int)count);
  return rc ? batchFail(batch, rc, batch->stepper->error()) : FP_OK;
}

int fp_batch_synchronize(fp_batch* batch) {
  if (!batch) return failed("null batch", FP_EINVAL);
  int rc = batch->stepper->synchronize();
  return rc ? batchFail(batch, rc, batch->stepper->error()) : FP_OK;
}

int fp_batch_stats(fp_batch* batch, uint32_t id, fp_stats* out) {
  if (!batch || !out) return failed("fp_batch_stats needs a batch and an output.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->stats(out);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_read_field(fp_batch* batch, uint32_t id, int field, float* host, size_t bytes) {
  if (!batch || !host) return failed("fp_batch_read_field needs a batch and a buffer.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->readField(field, host, bytes);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_read_table(fp_batch* batch, uint32_t id, int table, void* host, size_t* bytes) {
  if (!batch || !bytes) return failed("fp_batch_read_table needs a batch and a size.", FP_EINVAL);
  fp::Engine* e = batchSim(batch, id);
  if (!e) return batchFail(batch, FP_EINVAL, "no simulation with id " + std::to_string(id));
  int rc = e->readTable(table, host, bytes);
  return rc ? batchFail(batch, rc, e->error()) : FP_OK;
}

int fp_batch_stream(fp_batch* batch, void** stream) {
  if (!batch || !stream) return failed("fp_batch_stream needs a batch and an output.", FP_EINVAL);
  *stream = (void*)batch->stepper->stream();
  return FP_OK;
}

int fp_batch_set_profiling(fp_batch* batch, int enabled) {
  if (!batch) return failed("null batch", FP_EINVAL);
  int rc = batch->stepper->setProfiling(enabled != 0);
  return rc ? batchFail(batch, rc, batch->stepper->error()) : FP_OK;
}

int fp_batch_read_profile(fp_batch* batch, fp_phase* phases, uint32_t* count) {
  if (!batch || !count) return failed("fp_batch_read_profile needs a batch and a count.", FP_EINVAL);
  int rc = batch->stepper->readProfile(phases, count);
  return rc ? batchFail(batch, rc, batch->stepper->error()) : FP_OK;
}

int fp_grid_memory_bytes(const fp_grid* grid, uint64_t* bytes) {
  if (!grid || !bytes) return failed("fp_grid_memory_bytes needs a grid and an output.", FP_EINVAL);
  int rc = validateGrid(grid);
  if (rc) return rc;
  *bytes = fp::Engine::estimateBytes(*grid, fp::Engine::tilesForBudget(grid->voxel_budget, grid->brick_size *
                                                                                             grid->brick_size *
                                                                                             grid->brick_size));
  return FP_OK;
}

int fp_grid_reserved_tiles(const fp_grid* grid, uint32_t* tiles) {
  if (!grid || !tiles) return failed("fp_grid_reserved_tiles needs a grid and an output.", FP_EINVAL);
  int rc = validateGrid(grid);
  if (rc) return rc;
  *tiles = fp::Engine::tilesForBudget(grid->voxel_budget, grid->brick_size * grid->brick_size * grid->brick_size);
  return FP_OK;
}

}  // extern "C"
