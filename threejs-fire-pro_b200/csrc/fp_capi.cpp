// extern "C" entry points of include/firepro.h. Each validates its arguments, forwards to
// the host engine and turns any failure into a status code with a message; nothing throws
// across the ABI.
#include <cmath>
#include <new>
#include <string>

#include "../../include/firepro.h"
#include "fp_engine.hpp"
#include "fp_error.h"

struct fp_sim {
  fp::Engine* engine;
};

static thread_local std::string g_error;

static int failed(const std::string& message, int code) {
  g_error = message;
  return code;
}

int fp_set_error(int code, const std::string& message) { return failed(message, code); }

extern "C" {

int fp_abi_version(void) { return FP_ABI_VERSION; }

const char* fp_last_error(const fp_sim* sim) {
  if (sim && sim->engine) return sim->engine->error().c_str();
  return g_error.c_str();
}

// The grid validation of FluidSimulation's constructor (FluidSimulation.ts:359-379).
int fp_sim_create(const fp_grid* grid, int device, fp_sim** out) {
  if (!grid || !out) return failed("fp_sim_create needs a grid and an output handle.", FP_EINVAL);
  *out = nullptr;
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
  if (vd != 1) return failed("velocityDivisor 2 and 4 are not implemented by this build.", FP_EUNSUPPORTED);
  if (sd != 1) return failed("smokeDivisor 2 and 4 are not implemented by this build.", FP_EUNSUPPORTED);
  if (bs == 32) return failed("brickSize 32 is not implemented by this build.", FP_EUNSUPPORTED);
  if (grid->precision != FP_PRECISION_FP32)
    return failed("FP_PRECISION_MIXED is not implemented by this build.", FP_EUNSUPPORTED);
  fp::Engine* e = new (std::nothrow) fp::Engine(*grid, device);
  if (!e) return failed("out of host memory", FP_ENOMEM);
  int rc = e->initialize();
  if (rc) {
    g_error = e->error();
    delete e;
    return rc;
  }
  fp_sim* s = new (std::nothrow) fp_sim{e};
  if (!s) {
    delete e;
    return failed("out of host memory", FP_ENOMEM);
  }
  *out = s;
  return FP_OK;
}

int fp_sim_destroy(fp_sim* sim) {
  if (!sim) return FP_OK;
  delete sim->engine;
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
  if ((frame->source_count && !frame->sources) || (frame->force_count && !frame->forces) ||
      (frame->collider_count && !frame->colliders) || (frame->force_target_count && !frame->force_targets) ||
      (frame->collider_mask_words && !frame->collider_masks))
    return sim->engine->fail(FP_EINVAL, "frame arrays are null but their counts are not");
  return sim->engine->step(*frame, dt);
}

int fp_sim_synchronize(fp_sim* sim) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  return sim->engine->synchronize();
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

int fp_sim_read_bricks(fp_sim* sim, float* boxes, uint32_t* count) {
  if (!sim || !count) return failed("fp_sim_read_bricks needs a simulation and a count.", FP_EINVAL);
  return sim->engine->readBricks(boxes, count);
}

int fp_sim_stream(fp_sim* sim, void** stream) {
  if (!sim || !stream) return failed("fp_sim_stream needs a simulation and an output.", FP_EINVAL);
  *stream = (void*)sim->engine->stream();
  return FP_OK;
}

int fp_sim_set_profiling(fp_sim* sim, int enabled) {
  if (!sim) return failed("null simulation", FP_EINVAL);
  return sim->engine->setProfiling(enabled != 0);
}

int fp_sim_read_profile(fp_sim* sim, fp_phase* phases, uint32_t* count) {
  if (!sim || !count) return failed("fp_sim_read_profile needs a simulation and a count.", FP_EINVAL);
  return sim->engine->readProfile(phases, count);
}

}  // extern "C"
