// Stepper: one launch steps any number of simulations (fp_engine.hpp). Per step it
//   1. waits for the previous launch's measurement (read right after field evolution, so the
//      host prepares while the GPU finishes the previous step) and hands it out;
//   2. checks every frame, then lets each simulation do its host work;
//   3. writes the work rows, every simulation's SimParams and scene into one pinned upload
//      and copies it with one cudaMemcpyAsync;
//   4. replays the CUDA graph of the step's kernels (captured once per combination of the
//      optional launches: grids are fixed and buffers are read from SimParams, so growth of
//      any simulation keeps the graph valid).
#include <algorithm>
#include <chrono>
#include <cstring>

#include "fp_engine.hpp"
#include "fp_launch.h"

namespace fp {

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

Stepper::Stepper(int device, int brickSize) : device_(device), B_(brickSize) {
  brickLevels_ = B_ == 8 ? 3 : (B_ == 16 ? 4 : 5);
  bottom_ = brickLevels_ + 2;
}

Stepper::~Stepper() {
  if (stream_) cudaStreamSynchronize(stream_);
  clearGraphs();
  if (arenaH_) cudaFreeHost(arenaH_);
  if (arenaD_) cudaFree(arenaD_);
  if (readH_) cudaFreeHost(readH_);
  if (noise_) cudaFree(noise_);
  if (readEvent_) cudaEventDestroy(readEvent_);
  for (cudaEvent_t e : {forkTopo_, joinTopo_, forkCurl_, joinCurl_, joinSmoke_})
    if (e) cudaEventDestroy(e);
  if (side_) cudaStreamDestroy(side_);
  for (Phase& ph : phases_) {
    if (ph.a) cudaEventDestroy(ph.a);
    if (ph.b) cudaEventDestroy(ph.b);
  }
  if (stream_) cudaStreamDestroy(stream_);
}

int Stepper::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FP_OK;
  error_ = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? FP_ENOMEM : FP_EDEVICE;
}

int Stepper::initialize() {
  int rc;
  if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return rc;
  if ((rc = check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate"))) return rc;
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  if ((rc = check(cudaEventCreateWithFlags(&readEvent_, cudaEventDisableTiming), "cudaEventCreate"))) return rc;
  if ((rc = check(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking), "cudaStreamCreate"))) return rc;
  for (cudaEvent_t* e : {&forkTopo_, &joinTopo_, &forkCurl_, &joinCurl_, &joinSmoke_})
    if ((rc = check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate"))) return rc;
  // The curl-noise table (CurlNoise.ts:5-51), once, shared by the simulations.
  if ((rc = check(cudaMalloc(&noise_, 64 * 64 * 64 * sizeof(float4)), "cudaMalloc"))) return rc;
  fp_launch_noise((float4*)noise_, stream_);
  // Shared-memory limits before any capture.
  fp_mg_configure(B_);
  fp_step_configure(B_);
  // Room for a few hundred simulations' parameters and scenes from the start: growing the
  // upload later waits for the stream and captures the graphs again.
  if ((rc = reserve(4 << 20, 256, 1 << 16))) return rc;
  return check(cudaStreamSynchronize(stream_), "initialize");
}

FpBatch Stepper::batch() const {
  FpBatch b;
  b.sims = reinterpret_cast<const SimParams*>(arenaD_ + align256((size_t)(1 + FP_WORK_KINDS * (maxSims_ + 1)) * 4));
  b.work = reinterpret_cast<uint32_t*>(arenaD_);
  b.stride = maxSims_ + 1;
  return b;
}

// Room for an upload of `arenaBytes` with `sims` simulations and `readWords` measurement
// words. Growing either waits for the stream; a new upload buffer drops the captured graphs
// (their kernels hold its address).
int Stepper::reserve(size_t arenaBytes, int sims, size_t readWords) {
  if (sims > maxSims_ || arenaBytes > arenaCap_) {
    cudaStreamSynchronize(stream_);
    clearGraphs();
    int nextSims = std::max(sims, maxSims_ * 2);
    size_t header = align256((size_t)(1 + FP_WORK_KINDS * (nextSims + 1)) * 4) + (size_t)nextSims * sizeof(SimParams);
    size_t cap = std::max(arenaBytes + header, arenaCap_ * 2);
    if (arenaH_) cudaFreeHost(arenaH_);
    if (arenaD_) cudaFree(arenaD_);
    arenaH_ = arenaD_ = nullptr;
    arenaCap_ = 0;
    if (cudaMallocHost(&arenaH_, cap) != cudaSuccess || cudaMalloc(&arenaD_, cap) != cudaSuccess) {
      error_ = "out of memory for the step's upload";
      return FP_ENOMEM;
    }
    arenaCap_ = cap;
    maxSims_ = nextSims;
  }
  if (readWords > readCap_) {
    cudaStreamSynchronize(stream_);
    if (readH_) cudaFreeHost(readH_);
    readH_ = nullptr;
    size_t cap = std::max(readWords, readCap_ * 2);
    void* dev = nullptr;
    if (cudaHostAlloc(&readH_, cap * 4, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&dev, readH_, 0) != cudaSuccess) {
      readCap_ = 0;
      error_ = "out of pinned memory for the measurement";
      return FP_ENOMEM;
    }
    readD_ = (uint32_t*)dev;
    readCap_ = cap;
  }
  return FP_OK;
}

void Stepper::clearGraphs() {
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
  graphs_.clear();
}

int Stepper::consume() {
  if (!pendingRead_) return FP_OK;
  auto t0 = std::chrono::steady_clock::now();
  int rc = check(cudaEventSynchronize(readEvent_), "step");
  hostWaitMs_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (rc) return rc;
  pendingRead_ = false;
  double voxels = 0;
  for (auto& pe : pending_) {
    voxels += (double)reinterpret_cast<const FpCounters*>(readH_ + pe.second)->active * B_ * B_ * B_;
    pe.first->applyReadback(readH_ + pe.second);
  }
  pending_.clear();
  if (profilePending_) {
    // The phases after the measurement may still run: wait for the step's last one.
    for (int k = PH_COUNT - 1; k >= 0; k--)
      if (phases_[k].used) {
        cudaEventSynchronize(phases_[k].b);
        break;
      }
    for (Phase& ph : phases_) {
      if (!ph.used) continue;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ph.a, ph.b);
      ph.ms += ms;
      ph.launches += ph.stepLaunches;
      ph.voxels += voxels;
      ph.used = false;
    }
    profilePending_ = false;
  }
  return FP_OK;
}

void Stepper::forget(const Engine* e) {
  pending_.erase(std::remove_if(pending_.begin(), pending_.end(),
                                [e](const std::pair<Engine*, size_t>& pe) { return pe.first == e; }),
                 pending_.end());
}

int Stepper::synchronize() { return check(cudaStreamSynchronize(stream_), "synchronize"); }

int Stepper::step(Engine* const* sims, const fp_frame* const* frames, const float* dts, int count) {
  auto t0 = std::chrono::steady_clock::now();
  double wait0 = hostWaitMs_;
  int rc = FP_OK;
  auto done = [&](int code) {
    double all = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    hostPrepareMs_ += all - (hostWaitMs_ - wait0);
    return code;
  };
  if (count <= 0) return done(FP_OK);
  // Messages name the simulation's position when the launch holds more than one.
  auto who = [&](int i) { return count > 1 ? "simulation " + std::to_string(i) + ": " : std::string(); };
  for (int i = 0; i < count; i++)
    if (sims[i]->brickSize() != B_) {
      error_ = who(i) + "brick size differs from the batch's";
      return done(FP_EINVAL);
    }
  // The velocity lattice's brick levels are the launch's: one velocity divisor a stepper.
  if (vd_ == 0) {
    vd_ = sims[0]->velocityDivisor();
    brickLevels_ = 0;
    while ((1 << brickLevels_) < B_ / vd_) brickLevels_++;
    bottom_ = brickLevels_ + 2;
  }
  for (int i = 0; i < count; i++)
    if (sims[i]->velocityDivisor() != vd_) {
      error_ = who(i) + "velocity divisor differs from the batch's";
      return done(FP_EINVAL);
    }
  // One launch runs one pressure-solve schedule.
  for (int i = 1; i < count; i++)
    if (std::memcmp(&sims[i]->schedule(), &sims[0]->schedule(), sizeof(fp_solver_schedule)) != 0) {
      error_ = who(i) + "solver schedule differs from the batch's";
      return done(FP_EINVAL);
    }
  for (int i = 0; i < count; i++)
    if ((rc = sims[i]->validate(*frames[i], dts[i]))) {
      error_ = who(i) + sims[i]->error();
      return done(rc);
    }
  if ((rc = check(cudaSetDevice(device_), "cudaSetDevice"))) return done(rc);
  if ((rc = consume())) return done(rc);
  for (int i = 0; i < count; i++)
    if ((rc = sims[i]->prepare(*frames[i], dts[i]))) {
      error_ = who(i) + sims[i]->error();
      return done(rc);
    }
  // Layout of the upload and of the measurement words.
  size_t scene = 0, words = 0;
  for (int i = 0; i < count; i++) {
    scene += sims[i]->sceneBytes();
    words += sims[i]->readbackWords();
  }
  size_t header = align256((size_t)(1 + FP_WORK_KINDS * (std::max(count, maxSims_) + 1)) * 4) +
                  (size_t)std::max(count, maxSims_) * sizeof(SimParams);
  if ((rc = reserve(header + scene, count, words))) return done(rc);
  FpBatch bt = batch();
  size_t paramsOff = (size_t)((const uint8_t*)bt.sims - arenaD_);
  size_t off = paramsOff + (size_t)maxSims_ * sizeof(SimParams);
  uint32_t* work = reinterpret_cast<uint32_t*>(arenaH_);
  work[0] = (uint32_t)count;
  uint32_t* rowBlocks = work + 1 + FP_WORK_IDBLOCKS * bt.stride;
  uint32_t* rowTiles = work + 1 + FP_WORK_TILES * bt.stride;
  uint32_t* rowIds = work + 1 + FP_WORK_IDS * bt.stride;
  uint32_t blocks = 0, tiles = 0, ids = 0;
  size_t word = 0;
  bool solidsFresh = false, solidsAll = false, topoAll = false, curl = false, measure = false;
  schedule_ = sims[0]->schedule();
  int vcycles = 1;
  fusedCoarse_ = true;
  anySmoke_ = false;
  smokeDiv_ = 0;
  pending_.clear();
  for (int i = 0; i < count; i++) {
    Engine* e = sims[i];
    uint32_t cap = (uint32_t)e->capacity();
    fusedCoarse_ = fusedCoarse_ && fp_coarse_fits(e->liveTiles());
    anySmoke_ = anySmoke_ || e->smokeDivisor() > 1;
    if (e->smokeDivisor() > 1 && (smokeDiv_ == 0 || e->smokeDivisor() < smokeDiv_)) smokeDiv_ = e->smokeDivisor();
    rowBlocks[i] = blocks;
    rowTiles[i] = tiles;
    rowIds[i] = ids;
    blocks += (cap * 64 + 255) / 256;
    tiles += (uint32_t)e->liveTiles();  // the tile-level kernels walk the live tiles
    ids += cap * 64;
    SimParams* P = reinterpret_cast<SimParams*>(arenaH_ + paramsOff) + i;
    e->writeStep(*P, arenaH_, arenaD_, off, *frames[i], dts[i], readD_ + word, noise());
    off += e->sceneBytes();
    pending_.push_back({e, word});
    word += e->readbackWords();
    solidsFresh = solidsFresh || (e->buildSolids() && !e->solidsAll());
    solidsAll = solidsAll || e->solidsAll();
    topoAll = topoAll || e->topoAll();
    curl = curl || frames[i]->simulation.vorticity != 0.f;
    vcycles = std::max(vcycles, e->vcycles());
    measure = measure || e->measures();
  }
  rowBlocks[count] = blocks;
  rowTiles[count] = tiles;
  rowIds[count] = ids;
  if ((rc = check(cudaMemcpyAsync(arenaD_, arenaH_, off, cudaMemcpyHostToDevice, stream_), "upload"))) return done(rc);
  lastUpload_ = off;
  lastReadback_ = word * 4;

  int latest = 0;
  if (profiling_) {
    // Eager launches with an event pair around each phase.
    uint64_t n = 0;
    enqueue(solidsFresh, solidsAll, topoAll, curl, vcycles, measure, latest, n);
    launches_ += n;
  } else {
    uint64_t key = (uint64_t)solidsFresh | ((uint64_t)solidsAll << 1) | ((uint64_t)topoAll << 2) | ((uint64_t)curl << 3) |
                   ((uint64_t)measure << 4) | ((uint64_t)vcycles << 5) | ((uint64_t)fusedCoarse_ << 16) |
                   ((uint64_t)anySmoke_ << 17) | ((uint64_t)schedule_.smoother << 18) |
                   ((uint64_t)schedule_.krylov << 19) | ((uint64_t)schedule_.levels << 20) |
                   ((uint64_t)schedule_.pre_sweeps << 24) | ((uint64_t)schedule_.post_sweeps << 28) |
                   ((uint64_t)schedule_.bottom_sweeps << 32) | ((uint64_t)smokeDiv_ << 40);
    auto it = graphs_.find(key);
    if (it == graphs_.end()) {
      GraphEntry ge{};
      if ((rc = check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture")))
        return done(rc);
      enqueue(solidsFresh, solidsAll, topoAll, curl, vcycles, measure, ge.latest, ge.launches);
      cudaGraph_t g = nullptr;
      rc = check(cudaStreamEndCapture(stream_, &g), "cudaStreamEndCapture");
      if (rc) return done(rc);
      rc = check(cudaGraphInstantiate(&ge.exec, g, 0), "cudaGraphInstantiate");
      cudaGraphDestroy(g);
      if (rc) return done(rc);
      it = graphs_.emplace(key, ge).first;
    }
    if ((rc = check(cudaGraphLaunch(it->second.exec, stream_), "cudaGraphLaunch"))) return done(rc);
    latest = it->second.latest;
    launches_ += it->second.launches;
  }
  pendingRead_ = true;
  for (int i = 0; i < count; i++) sims[i]->launched(dts[i], latest);
  return done(check(cudaGetLastError(), "step launch"));
}

void Stepper::phaseBegin(int id) {
  if (profiling_) cudaEventRecord(phases_[id].a, stream_);
}
void Stepper::phaseEnd(int id, int launches) {
  if (!profiling_) return;
  Phase& ph = phases_[id];
  cudaEventRecord(ph.b, stream_);
  ph.stepLaunches = (uint64_t)launches;
  ph.used = true;
  profilePending_ = true;
}

int Stepper::setProfiling(bool on) {
  int rc = consume();
  if (rc) return rc;
  for (Phase& ph : phases_) {
    if (!ph.a && (rc = check(cudaEventCreate(&ph.a), "cudaEventCreate"))) return rc;
    if (!ph.b && (rc = check(cudaEventCreate(&ph.b), "cudaEventCreate"))) return rc;
    if (on) {
      ph.launches = 0;
      ph.ms = 0;
      ph.voxels = 0;
    }
    ph.used = false;
  }
  profiling_ = on;
  return FP_OK;
}

int Stepper::readProfile(fp_phase* out, uint32_t* count) {
  static const char* names[PH_COUNT] = {"allocation", "topology", "predict", "correct", "evolve", "smoke",
                                        "curl", "forces", "divergence", "multigrid", "project"};
  int rc = consume();
  if (rc) return rc;
  uint32_t cap = *count;
  *count = PH_COUNT;
  if (!out || cap < PH_COUNT) {
    error_ = "profile buffer too small";
    return FP_ELIMIT;
  }
  for (int i = 0; i < PH_COUNT; i++) {
    std::memset(&out[i], 0, sizeof(fp_phase));
    std::strncpy(out[i].name, names[i], sizeof(out[i].name) - 1);
    out[i].launches = phases_[i].launches;
    out[i].ms = phases_[i].ms;
    out[i].voxels = phases_[i].voxels;
  }
  return FP_OK;
}

// One V-cycle of PressureSolver.plan (PressureSolver.ts:276-365); `cur` holds each level's
// current pressure buffer. The finest level's first iterate was written with the divergence.
void Stepper::vcycle(int level, int cur[], uint64_t& launches) {
  auto sel = [](int l, int which) { return fp_mg_sel(l, which); };
  bool tiles = level >= brickLevels_;
  if (fusedCoarse_ && level == brickLevels_ + 1) {
    // Two relaxations, restriction, the bottom, prolongation, three relaxations: an even
    // number of flips leaves the result in the buffer of the first iterate.
    MgSel S{level, sel(level, 2), sel(level, cur[level]), -1, sel(level, cur[level]), sel(bottom_, 0), cycle_};
    fp_launch_coarse(batch(), S, 19, sms_, stream_);
    launches++;
    cur[bottom_] = 0;
    return;
  }
  if (level == bottom_) {
    MgSel S{level, sel(level, 2), sel(level, cur[level]), -1, sel(level, 1 - cur[level]), -1, cycle_};
    fp_launch_bottom(batch(), S, 19, sms_, stream_);
    launches++;
    cur[level] = 1 - cur[level];
    return;
  }
  auto relax = [&](int n) {
    for (int i = 0; i < n; i++) {
      MgSel S{level, level == 0 ? rhs0Sel_ : sel(level, 2), sel(level, cur[level]), -1, sel(level, 1 - cur[level]), -1, cycle_};
      fp_launch_relax(batch(), S, tiles, B_ / vd_, sms_, stream_);
      launches++;
      cur[level] = 1 - cur[level];
    }
  };
  if (level > 0) relax(2);
  int coarse = level + 1;
  MgSel R{coarse, level == 0 ? rhs0Sel_ : sel(level, 2), sel(level, cur[level]), -1, sel(coarse, 2), sel(coarse, 1), cycle_};
  fp_launch_restrict(batch(), R, coarse >= brickLevels_, B_ / vd_, sms_, stream_);
  launches++;
  cur[coarse] = 1;
  vcycle(coarse, cur, launches);
  MgSel Pr{level, -1, sel(level, cur[level]), sel(coarse, cur[coarse]), sel(level, 1 - cur[level]), -1, cycle_};
  fp_launch_prolong(batch(), Pr, tiles, B_ / vd_, sms_, stream_);
  launches++;
  cur[level] = 1 - cur[level];
  relax(3);
}

// One V-cycle of the red-black schedule (fp_solver_schedule) from `level` down: every level in
// place in its first buffer, `pre_sweeps` before each restriction, the coarse level from zero,
// prolongation in place, `post_sweeps` (odd cells first) after it; the coarsest of the
// schedule's levels takes `bottom_sweeps` (the bottom level in one CTA per simulation). The
// restriction's first iterate of the coarse level goes to its second buffer, unused.
void Stepper::vcycleRB(int level, bool zero, uint64_t& launches) {
  auto sel = [](int l, int which) { return fp_mg_sel(l, which); };
  const fp_solver_schedule& sc = schedule_;
  const int coarsest = sc.levels > 0 ? std::min(sc.levels - 1, bottom_) : bottom_;
  const bool tiles = level >= brickLevels_;
  const int rhs = level == 0 ? rhs0Sel_ : sel(level, 2), buf = sel(level, 0);
  auto half = [&](int parity, bool fromZero) {
    MgSel S{level, rhs, fromZero ? -1 : buf, -1, buf, -1, cycle_, parity + 1};
    fp_launch_relax(batch(), S, tiles, B_ / vd_, sms_, stream_);
    launches++;
  };
  auto sweeps = [&](int n, bool fromZero, bool post) {
    for (int i = 0; i < n; i++) {
      const int first = post ? 1 : 0;
      half(first, fromZero && i == 0);
      half(1 - first, false);
    }
  };
  if (level == coarsest) {
    if (level == bottom_) {
      MgSel S{level, rhs, zero ? -1 : buf, -1, buf, -1, cycle_, 1};
      fp_launch_bottom_rb(batch(), S, sc.bottom_sweeps, sms_, stream_);
      launches++;
    } else {
      sweeps(sc.bottom_sweeps, zero, false);
    }
    return;
  }
  sweeps(sc.pre_sweeps, zero, false);
  const int coarse = level + 1;
  MgSel R{coarse, rhs, buf, -1, sel(coarse, 2), sel(coarse, 1), cycle_, 0};
  fp_launch_restrict(batch(), R, coarse >= brickLevels_, B_ / vd_, sms_, stream_);
  launches++;
  vcycleRB(coarse, true, launches);
  MgSel Pr{level, -1, buf, sel(coarse, 0), buf, -1, cycle_, 0};
  fp_launch_prolong(batch(), Pr, tiles, B_ / vd_, sms_, stream_);
  launches++;
  sweeps(sc.post_sweeps, false, true);
}

// The step's kernels, measurement and its event, enqueued on the stream (eagerly, or under
// capture into a graph). `latest` receives the finest level's buffer holding the solution.
void Stepper::enqueue(bool solidsFresh, bool solidsAll, bool topoAll, bool curl, int vcycles, bool measure, int& latest,
                      uint64_t& launches) {
  FpBatch bt = batch();
  launches = 0;
  phaseBegin(PH_ALLOC);
  fp_launch_allocation(bt, solidsFresh, solidsAll, sms_, stream_);
  int n = fp_allocation_launches(solidsFresh, solidsAll);
  launches += n;
  phaseEnd(PH_ALLOC, n);
  // Topology of the slots granted this step, or of everything after the geometry changed.
  // Topology reads the allocation's tables and solids and writes only the multigrid's flags and
  // masks, which nothing reads before the divergence: beside the transport kernels when not
  // profiling.
  const bool fork = !profiling_;
  if (fork) {
    cudaEventRecord(forkTopo_, stream_);
    cudaStreamWaitEvent(side_, forkTopo_, 0);
    fp_launch_topology(bt, topoAll, sms_, side_);
    cudaEventRecord(joinTopo_, side_);
    // Coarse smoke's advection reads the start-of-step state only: beside the fine transport,
    // joined before the coarse evolution.
    if (anySmoke_) {
      fp_launch_smoke_advect(bt, B_, vd_, smokeDiv_, sms_, side_);
      cudaEventRecord(joinSmoke_, side_);
    }
  } else {
    phaseBegin(PH_TOPO);
    fp_launch_topology(bt, topoAll, sms_, stream_);
    phaseEnd(PH_TOPO, topoAll ? 4 : 2);
  }
  launches += topoAll ? 4 : 2;
  phaseBegin(PH_PREDICT);
  fp_launch_predict(bt, B_, vd_, sms_, stream_);
  phaseEnd(PH_PREDICT, 1);
  phaseBegin(PH_CORRECT);
  fp_launch_correct(bt, B_, vd_, sms_, stream_);
  phaseEnd(PH_CORRECT, 1);
  // The curl reads only the corrected velocity, and only the forces read it: beside evolution.
  if (fork && curl) {
    cudaEventRecord(forkCurl_, stream_);
    cudaStreamWaitEvent(side_, forkCurl_, 0);
    fp_launch_curl(bt, B_, vd_, sms_, side_);
    cudaEventRecord(joinCurl_, side_);
  }
  phaseBegin(PH_EVOLVE);
  fp_launch_evolve(bt, B_, vd_, sms_, stream_);
  phaseEnd(PH_EVOLVE, 1);
  // Coarse smoke evolves after the fine fields, whose source production it averages, and
  // records content before the measurement.
  if (anySmoke_) {
    phaseBegin(PH_SMOKE);
    if (fork)
      cudaStreamWaitEvent(stream_, joinSmoke_, 0);
    else
      fp_launch_smoke_advect(bt, B_, vd_, smokeDiv_, sms_, stream_);
    fp_launch_smoke_evolve(bt, B_, vd_, smokeDiv_, sms_, stream_);
    phaseEnd(PH_SMOKE, 2);
  }
  launches += anySmoke_ ? 5 : 3;

  // Measurement: counters and the tiles' content flags are final once evolution ran, so they
  // are read here; the next step waits for this event only and prepares while the GPU runs
  // the rest of this step. Failed allocations count from one measurement to the next.
  fp_launch_readback(bt, sms_, stream_);
  launches++;
  // Under capture, external: an event-record node the graph replays.
  if (profiling_)
    cudaEventRecord(readEvent_, stream_);
  else
    cudaEventRecordWithFlags(readEvent_, stream_, cudaEventRecordExternal);

  if (curl) {
    if (fork) {
      cudaStreamWaitEvent(stream_, joinCurl_, 0);
    } else {
      phaseBegin(PH_CURL);
      fp_launch_curl(bt, B_, vd_, sms_, stream_);
      phaseEnd(PH_CURL, 1);
    }
    launches++;
  }
  phaseBegin(PH_FORCES);
  fp_launch_forces(bt, B_, vd_, sms_, stream_);
  launches++;
  phaseEnd(PH_FORCES, 1);
  // Cold start every step: the divergence writes the first iterate into p0[1].
  int cur[FP_MAX_LEVELS] = {0};
  if (fork) cudaStreamWaitEvent(stream_, joinTopo_, 0);  // the first iterate reads the topology
  phaseBegin(PH_DIVERGENCE);
  fp_launch_divergence(bt, 1, vd_, sms_, stream_);
  launches++;
  phaseEnd(PH_DIVERGENCE, 1);
  cur[0] = 1;
  phaseBegin(PH_MULTIGRID);
  uint64_t mg = 0;
  rhs0Sel_ = fp_mg_sel(0, 2);
  const bool redBlack = schedule_.smoother == FP_SMOOTHER_REDBLACK;
  if (schedule_.krylov == FP_KRYLOV_FCG) {
    // Flexible CG: V-cycle 0 from the divergence gives the start x (the CG iterate, p0[2]);
    // each later V-cycle, from zero on the residual s (level 0's selector 3), gives z, the next
    // direction and step. Simulations that converged skip the later cycles' work.
    cycle_ = 0;
    int x0 = 0;
    if (redBlack) {
      vcycleRB(0, true, mg);
    } else {
      vcycle(0, cur, mg);
      x0 = cur[0];
    }
    fp_launch_fcg_begin(bt, x0, sms_, stream_);
    mg += 2;
    rhs0Sel_ = fp_mg_sel(0, 3);
    for (int c = 1; c < vcycles; c++) {
      cycle_ = c;
      int z = 0;
      if (redBlack) {
        vcycleRB(0, true, mg);
      } else {
        // The first iterate from zero (as the divergence kernel writes it for V-cycle 0).
        MgSel S{0, rhs0Sel_, -1, -1, fp_mg_sel(0, 1), -1, cycle_, 0};
        fp_launch_relax(bt, S, false, B_ / vd_, sms_, stream_);
        mg++;
        cur[0] = 1;
        vcycle(0, cur, mg);
        z = cur[0];
      }
      fp_launch_fcg_iterate(bt, z, c, sms_, stream_);
      mg += fp_fcg_iterate_launches(c);
    }
    rhs0Sel_ = fp_mg_sel(0, 2);
    latest = 2;
  } else if (redBlack) {
    // In place in p0[0]; a later V-cycle corrects the current iterate (a converged simulation
    // skips it and keeps its result in the same buffer).
    for (int c = 0; c < vcycles; c++) {
      cycle_ = c;
      vcycleRB(0, c == 0, mg);
      if (vcycles > 1 || measure) {
        fp_launch_residual(bt, 0, c, sms_, stream_);
        mg += 2;
      }
    }
    latest = 0;
  } else {
    // Up to `vcycles` V-cycles. Each leaves the finest level's result in the buffer it started
    // from (four flips: prolongation and three sweeps), so a simulation that converged and
    // skips the later cycles ends in the same buffer. After each cycle, when measured, the
    // FP64 residual decides convergence.
    for (int c = 0; c < vcycles; c++) {
      cycle_ = c;
      vcycle(0, cur, mg);
      if (vcycles > 1 || measure) {
        fp_launch_residual(bt, cur[0], c, sms_, stream_);
        mg += 2;
      }
    }
    latest = cur[0];
  }
  cycle_ = 0;
  launches += mg;
  phaseEnd(PH_MULTIGRID, (int)mg);
  phaseBegin(PH_PROJECT);
  fp_launch_project(bt, latest, vd_, sms_, stream_);
  launches++;
  if (measure) {
    fp_launch_post_divergence(bt, sms_, stream_);
    launches++;
  }
  phaseEnd(PH_PROJECT, measure ? 2 : 1);
}

}  // namespace fp
