// Serving front end (fp_server_* of include/firepro.h): sessions admitted by device-memory
// budget, step requests batched as they arrive.
//
// A scheduler thread owns the Stepper and every session's Engine. Each turn it closes the
// sessions that asked to leave and whose steps ran, admits waiting sessions in arrival order
// while the budget and the session limit allow, takes the oldest queued request of every live
// session and steps them in one launch. Right after the launch it enqueues a host function on
// the batch's stream: when the GPU finishes the step, the function stamps the completion time
// of each request and reads its measurement from the launch's host-mapped words. The
// Stepper's own pipelining (the next launch waits only for the previous measurement) lets
// requests that arrive while a step runs be prepared and launched right behind it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/firepro.h"
#include "fp_engine.hpp"
#include "fp_error.h"

namespace {

// A frame and every array it points into, owned by the request: the scheduler reads them
// after fp_server_submit has returned, when the caller's arrays may be gone.
struct FrameCopy {
  fp_frame frame;
  std::vector<fp_source> sources, targets;
  std::vector<fp_force> forces;
  std::vector<fp_collider> colliders;
  std::vector<uint32_t> masks;
  std::vector<fp_mesh_source> meshSources;
  std::vector<int32_t> targetCells;
  std::vector<uint32_t> targetRanges;
  template <class T>
  static const T* own(std::vector<T>& v, const T* src, size_t n) {
    if (!src || !n) {
      v.clear();
      return src && !n ? nullptr : src;
    }
    v.assign(src, src + n);
    return v.data();
  }
  void assign(const fp_frame& f) {
    frame = f;
    frame.sources = own(sources, f.sources, f.source_count);
    frame.force_targets = own(targets, f.force_targets, f.force_target_count);
    frame.forces = own(forces, f.forces, f.force_count);
    frame.colliders = own(colliders, f.colliders, f.collider_count);
    frame.collider_masks = own(masks, f.collider_masks, f.collider_mask_words);
    frame.mesh_sources = own(meshSources, f.mesh_sources, f.mesh_source_count);
    frame.target_cells = own(targetCells, f.target_cells, (size_t)f.target_cell_count * 3);
    // Two words per force target; present only with target cells.
    frame.target_cell_ranges =
        f.target_cell_ranges ? own(targetRanges, f.target_cell_ranges, (size_t)f.force_target_count * 2) : nullptr;
  }
};

struct Request {
  uint32_t session;
  uint64_t ticket;
  FrameCopy frame;
  float dt;
  double submitMs;
};

struct Session {
  fp_grid grid;
  float cutoff;
  int ground;
  fp_solver_schedule schedule;  // the server's solve when the session opened
  int vcycles;
  float tolerance;
  int state = FP_SESSION_WAITING;
  fp::Engine* engine = nullptr;
  uint64_t bytes = 0;
  uint64_t steps = 0;
  int inflight = 0;  // steps launched and not yet completed
  std::deque<Request*> queue;
};

}  // namespace

struct fp_server {
  fp_server_config cfg;
  fp::Stepper* stepper = nullptr;
  std::mutex mu;   // sessions, queues, completions, statistics
  std::mutex gpu;  // the Stepper and the Engines
  std::condition_variable work, done;
  std::thread worker;
  bool stop = false;
  std::string error;
  std::vector<Session*> sessions;
  std::deque<uint32_t> waiting;
  uint64_t memory = 0;
  uint32_t live = 0;
  int velocityDivisor = 0;  // the sessions' velocity divisor, from the first one opened
  fp_solver_schedule schedule{};  // the pressure solve of sessions admitted from now on
  int vcycles = 1;
  float tolerance = 0.f;
  uint64_t nextTicket = 1;
  uint64_t queued = 0, inFlight = 0;
  std::deque<fp_completion> completed;
  std::chrono::steady_clock::time_point t0;
  // statistics
  uint64_t stepsDone = 0, launches = 0, batchSessions = 0;
  double voxelSteps = 0;
  std::vector<double> latencies;

  double now() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// The requests of one launch, completed by a host function on the stream.
struct Launch {
  fp_server* S;
  std::vector<Request*> requests;
  std::vector<const uint32_t*> words;
  std::vector<uint64_t> steps;
  int cells;
};

void CUDART_CB onLaunchDone(void* p) {
  Launch* L = static_cast<Launch*>(p);
  fp_server* S = L->S;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    double t = S->now();
    for (size_t i = 0; i < L->requests.size(); i++) {
      Request* r = L->requests[i];
      const FpCounters* c = reinterpret_cast<const FpCounters*>(L->words[i]);
      fp_completion out{};
      out.session = r->session;
      out.status = FP_OK;
      out.ticket = r->ticket;
      out.step = L->steps[i];
      out.active_bricks = c->active;
      out.batch_size = (uint32_t)L->requests.size();
      out.submit_ms = r->submitMs;
      out.done_ms = t;
      S->completed.push_back(out);
      S->latencies.push_back(t - r->submitMs);
      S->voxelSteps += (double)c->active * L->cells;
      S->stepsDone++;
      S->inFlight--;
      S->sessions[r->session]->inflight--;
      delete r;
    }
  }
  S->done.notify_all();
  delete L;
}

void failRequests(fp_server* S, std::vector<Request*>& reqs, int status) {
  std::lock_guard<std::mutex> lk(S->mu);
  double t = S->now();
  for (Request* r : reqs) {
    fp_completion out{};
    out.session = r->session;
    out.status = status;
    out.ticket = r->ticket;
    out.submit_ms = r->submitMs;
    out.done_ms = t;
    S->completed.push_back(out);
    S->inFlight--;
    S->sessions[r->session]->inflight--;
    delete r;
  }
  reqs.clear();
}

void schedule(fp_server* S) {
  cudaSetDevice(S->cfg.device);
  std::vector<Session*> admit, close;
  std::vector<fp::Engine*> engines;
  std::vector<const fp_frame*> frames;
  std::vector<float> dts;
  std::vector<Request*> reqs;
  std::vector<uint64_t> stepsAfter;
  while (true) {
    admit.clear();
    close.clear();
    reqs.clear();
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->work.wait_for(lk, std::chrono::milliseconds(20), [&] {
        if (S->stop) return true;
        if (!S->waiting.empty()) return true;
        for (Session* s : S->sessions)
          if (s && ((s->state == FP_SESSION_LIVE && !s->queue.empty()) ||
                    (s->state == FP_SESSION_CLOSING && s->queue.empty())))
            return true;
        return false;
      });
      if (S->stop) break;
      for (Session* s : S->sessions)
        if (s && s->state == FP_SESSION_CLOSING && s->queue.empty()) close.push_back(s);
      // Admission in arrival order while the budget and the session limit allow.
      while (!S->waiting.empty()) {
        Session* s = S->sessions[S->waiting.front()];
        if (s->state != FP_SESSION_WAITING) {
          S->waiting.pop_front();
          continue;
        }
        if (S->live >= S->cfg.max_sessions || S->memory + s->bytes > S->cfg.memory_budget) break;
        S->waiting.pop_front();
        S->memory += s->bytes;
        S->live++;
        admit.push_back(s);
      }
      for (Session* s : S->sessions)
        if (s && s->state == FP_SESSION_LIVE && !s->queue.empty()) {
          reqs.push_back(s->queue.front());
          s->inflight++;
          s->queue.pop_front();
          S->queued--;
          S->inFlight++;
        }
    }
    std::lock_guard<std::mutex> g(S->gpu);
    for (Session* s : close) {
      S->stepper->consume();
      delete s->engine;
      s->engine = nullptr;
      std::lock_guard<std::mutex> lk(S->mu);
      S->memory -= s->bytes;
      S->live--;
      s->state = FP_SESSION_CLOSED;
    }
    for (Session* s : admit) {
      fp::Engine* e = new (std::nothrow) fp::Engine(s->grid, S->stepper);
      int rc = e ? e->initialize() : FP_ENOMEM;
      if (!rc) rc = e->setRuntime(s->cutoff, s->grid.voxel_budget, s->ground);
      // Tables sized for the budget up front: no step of the batch stops to grow them.
      int cells = s->grid.brick_size * s->grid.brick_size * s->grid.brick_size;
      if (!rc) rc = e->reserveTiles(fp::Engine::tilesForBudget(s->grid.voxel_budget, cells));
      if (!rc) rc = e->setSchedule(s->schedule);
      if (!rc) rc = e->setSolver(s->vcycles, s->tolerance);
      std::lock_guard<std::mutex> lk(S->mu);
      if (rc) {
        S->error = e ? e->error() : "out of host memory";
        delete e;
        S->memory -= s->bytes;
        S->live--;
        s->state = FP_SESSION_FAILED;
        continue;
      }
      s->engine = e;
      // A session opened live by fp_server_open may already be marked closing.
      if (s->state == FP_SESSION_WAITING) s->state = FP_SESSION_LIVE;
    }
    if (reqs.empty()) {
      S->done.notify_all();
      continue;
    }
    engines.clear();
    frames.clear();
    dts.clear();
    stepsAfter.clear();
    {
      // Each request is checked on its own (flame ramps, dt, mesh arrays) before the launch is
      // built: one session's invalid frame fails only its own step, with its message, and the
      // others run (the reference validates before any state changes, flame.ts:47-85,
      // FluidSimulation.ts:1368-1369).
      std::vector<Request*> bad;
      std::vector<std::string> why;
      std::vector<int> codes;
      std::vector<Request*> good;
      for (Request* r : reqs) {
        fp::Engine* e;
        {
          std::lock_guard<std::mutex> lk(S->mu);
          e = S->sessions[r->session]->engine;
        }
        int vrc = e->validate(r->frame.frame, r->dt);
        if (vrc) {
          bad.push_back(r);
          codes.push_back(vrc);
          why.push_back("session " + std::to_string(r->session) + ": " + e->error());
        } else {
          good.push_back(r);
        }
      }
      for (size_t k = 0; k < bad.size(); k++) {
        std::vector<Request*> one{bad[k]};
        {
          std::lock_guard<std::mutex> lk(S->mu);
          S->error = why[k];
        }
        failRequests(S, one, codes[k]);
      }
      reqs.swap(good);
      if (reqs.empty()) {
        S->done.notify_all();
        continue;
      }
      std::lock_guard<std::mutex> lk(S->mu);
      for (Request* r : reqs) {
        Session* s = S->sessions[r->session];
        engines.push_back(s->engine);
        frames.push_back(&r->frame.frame);
        dts.push_back(r->dt);
      }
    }
    int rc = S->stepper->step(engines.data(), frames.data(), dts.data(), (int)engines.size());
    if (rc) {
      {
        std::lock_guard<std::mutex> lk(S->mu);
        S->error = S->stepper->error();
      }
      failRequests(S, reqs, rc);
      S->done.notify_all();
      continue;
    }
    Launch* L = new Launch{S, reqs, {}, {}, S->stepper->brickSize() * S->stepper->brickSize() * S->stepper->brickSize()};
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (size_t i = 0; i < reqs.size(); i++) {
        Session* s = S->sessions[reqs[i]->session];
        s->steps++;
        L->steps.push_back(s->steps);
        L->words.push_back(S->stepper->lastReadback((int)i));
      }
      S->launches++;
      S->batchSessions += reqs.size();
    }
    reqs.clear();
    cudaLaunchHostFunc(S->stepper->stream(), onLaunchDone, L);
  }
  // Leave: the launched steps complete, queued ones are dropped.
  std::lock_guard<std::mutex> g(S->gpu);
  cudaStreamSynchronize(S->stepper->stream());
}

int serverFail(fp_server* S, int code, const std::string& m) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->error = m;
  fp_set_error(code, m);
  return code;
}

Session* sessionOf(fp_server* S, uint32_t id) { return id < S->sessions.size() ? S->sessions[id] : nullptr; }

}  // namespace

extern "C" {

const char* fp_server_last_error(const fp_server* server) {
  return server ? server->error.c_str() : fp_last_error(nullptr);
}

int fp_server_create(const fp_server_config* config, fp_server** out) {
  if (!config || !out) return fp_set_error(FP_EINVAL, "fp_server_create needs a configuration and an output.");
  *out = nullptr;
  if (config->brick_size != 8 && config->brick_size != 16 && config->brick_size != 32)
    return fp_set_error(FP_EINVAL, "a server's brickSize must be 8, 16 or 32.");
  if (config->max_sessions == 0) return fp_set_error(FP_EINVAL, "max_sessions must be positive.");
  fp_server* S = new (std::nothrow) fp_server{};
  if (!S) return fp_set_error(FP_ENOMEM, "out of host memory");
  S->cfg = *config;
  S->t0 = std::chrono::steady_clock::now();
  S->stepper = new (std::nothrow) fp::Stepper(config->device, config->brick_size);
  int rc = S->stepper ? S->stepper->initialize() : FP_ENOMEM;
  if (rc) {
    fp_set_error(rc, S->stepper ? S->stepper->error() : "out of host memory");
    delete S->stepper;
    delete S;
    return rc;
  }
  S->worker = std::thread(schedule, S);
  *out = S;
  return FP_OK;
}

int fp_server_destroy(fp_server* S) {
  if (!S) return FP_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  for (Session* s : S->sessions) {
    if (!s) continue;
    delete s->engine;
    for (Request* r : s->queue) delete r;
    delete s;
  }
  delete S->stepper;
  delete S;
  return FP_OK;
}

int fp_server_open(fp_server* S, const fp_grid* grid, float cutoff, int ground, uint32_t* session) {
  if (!S || !grid || !session) return fp_set_error(FP_EINVAL, "fp_server_open needs a server, a grid and an output.");
  uint64_t bytes = 0;
  int rc = fp_grid_memory_bytes(grid, &bytes);
  if (rc) return serverFail(S, rc, fp_last_error(nullptr));
  if (grid->brick_size != S->cfg.brick_size) return serverFail(S, FP_EINVAL, "brickSize differs from the server's.");
  {
    // One launch steps every live session on one velocity lattice: the server takes the
    // velocity divisor of its first session, and a grid with another one is refused here
    // rather than failing every launch it would join.
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->velocityDivisor == 0) S->velocityDivisor = grid->velocity_divisor;
    if (grid->velocity_divisor != S->velocityDivisor) {
      S->error = "velocityDivisor " + std::to_string(grid->velocity_divisor) + " differs from the server's (" +
                 std::to_string(S->velocityDivisor) + ").";
      fp_set_error(FP_EINVAL, S->error);
      return FP_EINVAL;
    }
  }
  if (!std::isfinite(cutoff)) return serverFail(S, FP_EINVAL, "grid.cutoff must be a finite number from 0 to 1.");
  if (bytes > S->cfg.memory_budget)
    return serverFail(S, FP_ELIMIT, "the session needs " + std::to_string(bytes) + " device bytes, more than the budget");
  Session* s = new (std::nothrow) Session{};
  if (!s) return serverFail(S, FP_ENOMEM, "out of host memory");
  s->grid = *grid;
  s->cutoff = cutoff;
  s->ground = ground;
  s->bytes = bytes;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    s->schedule = S->schedule;
    s->vcycles = S->vcycles;
    s->tolerance = S->tolerance;
    uint32_t id = 0;
    while (id < S->sessions.size() && S->sessions[id]) id++;
    if (id == S->sessions.size()) S->sessions.push_back(nullptr);
    S->sessions[id] = s;
    S->waiting.push_back(id);
    *session = id;
  }
  S->work.notify_all();
  return FP_OK;
}

int fp_server_set_solver(fp_server* S, const fp_solver_schedule* schedule, int vcycles, float tolerance) {
  if (!S || !schedule) return fp_set_error(FP_EINVAL, "fp_server_set_solver needs a server and a schedule.");
  if (schedule->smoother != FP_SMOOTHER_JACOBI && schedule->smoother != FP_SMOOTHER_REDBLACK)
    return serverFail(S, FP_EINVAL, "smoother must be FP_SMOOTHER_JACOBI or FP_SMOOTHER_REDBLACK.");
  if (schedule->krylov != FP_KRYLOV_NONE && schedule->krylov != FP_KRYLOV_FCG)
    return serverFail(S, FP_EINVAL, "krylov must be FP_KRYLOV_NONE or FP_KRYLOV_FCG.");
  if (schedule->topology != 0 && schedule->topology != 1) return serverFail(S, FP_EINVAL, "topology must be 0 or 1.");
  if (vcycles < 1 || vcycles > FP_MAX_VCYCLES)
    return serverFail(S, FP_EINVAL, "vcycles must be from 1 to " + std::to_string(FP_MAX_VCYCLES) + ".");
  if (!std::isfinite(tolerance) || tolerance < 0.f)
    return serverFail(S, FP_EINVAL, "tolerance must be finite and nonnegative.");
  // The red-black limits are checked per session at admission (they depend on its levels).
  std::lock_guard<std::mutex> lk(S->mu);
  S->schedule = *schedule;
  if (schedule->smoother == FP_SMOOTHER_JACOBI)
    S->schedule.levels = S->schedule.pre_sweeps = S->schedule.post_sweeps = S->schedule.bottom_sweeps = 0;
  S->vcycles = vcycles;
  S->tolerance = tolerance;
  return FP_OK;
}

int fp_server_close(fp_server* S, uint32_t session) {
  if (!S) return fp_set_error(FP_EINVAL, "null server");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    Session* s = sessionOf(S, session);
    if (!s || s->state == FP_SESSION_CLOSED) {
      S->error = "no open session " + std::to_string(session);
      return FP_EINVAL;
    }
    if (s->state == FP_SESSION_WAITING || s->state == FP_SESSION_FAILED) {
      for (Request* r : s->queue) delete r;
      S->queued -= s->queue.size();
      s->queue.clear();
      s->state = FP_SESSION_CLOSED;  // never admitted: nothing to free
    } else {
      s->state = FP_SESSION_CLOSING;
    }
  }
  S->work.notify_all();
  return FP_OK;
}

int fp_server_session_state(fp_server* S, uint32_t session, int* state) {
  if (!S || !state) return fp_set_error(FP_EINVAL, "fp_server_session_state needs a server and an output.");
  std::lock_guard<std::mutex> lk(S->mu);
  Session* s = sessionOf(S, session);
  if (!s) {
    S->error = "no session " + std::to_string(session);
    return FP_EINVAL;
  }
  *state = s->state;
  return FP_OK;
}

int fp_server_submit(fp_server* S, uint32_t session, const fp_frame* frame, float dt, uint64_t* ticket) {
  if (!S || !frame) return fp_set_error(FP_EINVAL, "fp_server_submit needs a server and a frame.");
  if ((frame->source_count && !frame->sources) || (frame->force_count && !frame->forces) ||
      (frame->collider_count && !frame->colliders) || (frame->force_target_count && !frame->force_targets) ||
      (frame->collider_mask_words && !frame->collider_masks) || (frame->mesh_source_count && !frame->mesh_sources) ||
      (frame->target_cell_count && (!frame->target_cells || !frame->target_cell_ranges)))
    return serverFail(S, FP_EINVAL, "frame arrays are null but their counts are not");
  if (!std::isfinite(dt) || dt <= 0 || dt > 1.f / 30.f)
    return serverFail(S, FP_EINVAL, "Simulation step must be in (0, 1/30]. Use fixed substeps.");
  Request* r = new (std::nothrow) Request{};
  if (!r) return serverFail(S, FP_ENOMEM, "out of host memory");
  r->frame.assign(*frame);
  r->dt = dt;
  r->session = session;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    Session* s = sessionOf(S, session);
    if (!s || s->state == FP_SESSION_CLOSING || s->state == FP_SESSION_CLOSED || s->state == FP_SESSION_FAILED) {
      delete r;
      S->error = "session " + std::to_string(session) + " takes no steps";
      return FP_EINVAL;
    }
    r->ticket = S->nextTicket++;
    r->submitMs = S->now();
    s->queue.push_back(r);
    S->queued++;
    if (ticket) *ticket = r->ticket;
  }
  S->work.notify_all();
  return FP_OK;
}

int fp_server_poll(fp_server* S, fp_completion* out, uint32_t capacity, uint32_t* count, int wait_ms) {
  if (!S || !count || (capacity && !out)) return fp_set_error(FP_EINVAL, "fp_server_poll needs a server and outputs.");
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->completed.empty() && wait_ms > 0)
    S->done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !S->completed.empty(); });
  uint32_t n = 0;
  while (n < capacity && !S->completed.empty()) {
    out[n++] = S->completed.front();
    S->completed.pop_front();
  }
  *count = n;
  return FP_OK;
}

int fp_server_drain(fp_server* S, int wait_ms) {
  if (!S) return fp_set_error(FP_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  // Steps queued by sessions that wait for admission count: they run once admitted.
  bool ok = S->done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !S->queued && !S->inFlight; });
  if (!ok) {
    S->error = "drain: steps still queued after " + std::to_string(wait_ms) + " ms";
    return FP_ETIMEOUT;
  }
  return FP_OK;
}

int fp_server_read_stats(fp_server* S, fp_server_stats* out) {
  if (!S || !out) return fp_set_error(FP_EINVAL, "fp_server_read_stats needs a server and an output.");
  std::vector<double> lat;
  std::vector<fp::Engine*> engines;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(out, 0, sizeof(*out));
    out->live = S->live;
    out->waiting = 0;
    for (Session* s : S->sessions)
      if (s && s->state == FP_SESSION_WAITING) out->waiting++;
    out->queued_steps = (uint32_t)S->queued;
    out->memory_bytes = S->memory;
    out->steps_done = S->stepsDone;
    out->launches = S->launches;
    out->voxel_steps = S->voxelSteps;
    out->elapsed_ms = S->now();
    out->mean_batch = S->launches ? (double)S->batchSessions / (double)S->launches : 0.0;
    lat = S->latencies;
    for (Session* s : S->sessions)
      if (s && s->engine) engines.push_back(s->engine);
  }
  {
    std::lock_guard<std::mutex> g(S->gpu);
    for (fp::Engine* e : engines) out->device_bytes += e->memoryBytes();
  }
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    out->latency_p50_ms = lat[lat.size() / 2];
    out->latency_p99_ms = lat[std::min(lat.size() - 1, (size_t)std::llround(0.99 * (double)(lat.size() - 1)))];
  }
  return FP_OK;
}

// A live session with no step queued or in flight: its Engine, with the GPU lock held by the
// caller (the scheduler only touches an Engine under that lock).
static fp::Engine* idleEngine(fp_server* S, uint32_t session, std::string& why) {
  std::lock_guard<std::mutex> lk(S->mu);
  Session* s = sessionOf(S, session);
  if (!s || s->state != FP_SESSION_LIVE || !s->engine) {
    why = "session " + std::to_string(session) + " is not live";
    return nullptr;
  }
  if (!s->queue.empty() || s->inflight) {
    why = "session " + std::to_string(session) + " has steps queued or running";
    return nullptr;
  }
  return s->engine;
}

// A live session's Engine, looked up with the GPU lock held (the scheduler deletes the Engines
// of closed sessions under it, and takes the GPU lock before the session lock, as here).
static fp::Engine* liveEngine(fp_server* S, uint32_t session) {
  std::lock_guard<std::mutex> lk(S->mu);
  Session* s = sessionOf(S, session);
  return s && (s->state == FP_SESSION_LIVE || s->state == FP_SESSION_CLOSING) ? s->engine : nullptr;
}

int fp_server_session_stats(fp_server* S, uint32_t session, fp_stats* out) {
  if (!S || !out) return fp_set_error(FP_EINVAL, "fp_server_session_stats needs a server and an output.");
  std::unique_lock<std::mutex> g(S->gpu);
  fp::Engine* e = liveEngine(S, session);
  if (!e) {
    g.unlock();
    return serverFail(S, FP_EINVAL, "session " + std::to_string(session) + " is not live");
  }
  int rc = e->stats(out);
  if (rc) return serverFail(S, rc, e->error());
  return FP_OK;
}

int fp_server_snapshot(fp_server* S, uint32_t session, void** blob, size_t* bytes) {
  if (!S || !blob || !bytes) return fp_set_error(FP_EINVAL, "fp_server_snapshot needs a server and outputs.");
  std::unique_lock<std::mutex> g(S->gpu);
  std::string why;
  fp::Engine* e = idleEngine(S, session, why);
  if (!e) {
    g.unlock();
    return serverFail(S, FP_EINVAL, why);
  }
  std::vector<uint8_t> v;
  int rc = e->snapshot(v);
  if (rc) return serverFail(S, rc, e->error());
  void* p = std::malloc(v.size() ? v.size() : 1);
  if (!p) return serverFail(S, FP_ENOMEM, "out of host memory for the snapshot");
  std::memcpy(p, v.data(), v.size());
  *blob = p;
  *bytes = v.size();
  return FP_OK;
}

int fp_server_restore(fp_server* S, uint32_t session, const void* blob, size_t bytes) {
  if (!S || !blob) return fp_set_error(FP_EINVAL, "fp_server_restore needs a server and a snapshot.");
  std::unique_lock<std::mutex> g(S->gpu);
  std::string why;
  fp::Engine* e = idleEngine(S, session, why);
  if (!e) {
    g.unlock();
    return serverFail(S, FP_EINVAL, why);
  }
  int rc = e->restore(static_cast<const uint8_t*>(blob), bytes);
  if (rc) return serverFail(S, rc, e->error());
  return FP_OK;
}

int fp_server_read_field(fp_server* S, uint32_t session, int field, float* host, size_t bytes) {
  if (!S || !host) return fp_set_error(FP_EINVAL, "fp_server_read_field needs a server and a buffer.");
  std::unique_lock<std::mutex> g(S->gpu);
  fp::Engine* e = liveEngine(S, session);
  if (!e) {
    g.unlock();
    return serverFail(S, FP_EINVAL, "session " + std::to_string(session) + " is not live");
  }
  int rc = e->readField(field, host, bytes);
  if (rc) return serverFail(S, rc, e->error());
  return FP_OK;
}

}  // extern "C"
