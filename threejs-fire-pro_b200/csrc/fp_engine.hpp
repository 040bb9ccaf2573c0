// Host engine of one simulation: the C++ counterpart of the reference's `FluidSimulation`
// (src/engine/FluidSimulation.ts) and `TileDirectory` (src/engine/TileDirectory.ts). It owns
// every device buffer, keeps the tile directory, packs each step's scene and enqueues the
// step's kernels on the simulation's stream.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/firepro.h"
#include "fp_types.h"

namespace fp {

// The directory of tiles (TileDirectory.ts:61-186): 4x4x4 bricks each, created around
// sources and content, lingering 60 steps after nothing needs them, slots reused lowest first.
class TileDirectory {
 public:
  struct Tile {
    int x, y, z;
    int64_t needed;
    bool closing;
    bool alive;
  };
  bool ground = true;
  bool dirty = true;

  void need(int lx, int ly, int lz, int hx, int hy, int hz, int64_t step);
  void retire(int64_t step);
  void clear();
  int slotAt(int x, int y, int z) const;
  int slotsUsed() const { return (int)slots_.size(); }
  int count() const { return (int)index_.size(); }
  const std::vector<Tile>& slots() const { return slots_; }
  std::vector<int> takeCreated();

 private:
  static uint64_t key(int x, int y, int z) {
    return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) |
           (uint64_t)(uint32_t)(z + (1 << 20));
  }
  std::vector<Tile> slots_;
  std::unordered_map<uint64_t, int> index_;
  std::vector<int> created_;
};

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

class Engine {
 public:
  Engine(const fp_grid& grid, int device);
  ~Engine();

  int initialize();
  int step(const fp_frame& frame, float dt);
  int stepBody(const fp_frame& frame, float dt);
  int reset();
  int setRuntime(float cutoff, double budget, int ground);
  int synchronize();
  int stats(fp_stats* out);
  int readField(int field, float* host, size_t bytes);
  int readTable(int table, void* host, size_t* bytes);
  int readBricks(float* boxes, uint32_t* count);
  int setProfiling(bool on);
  int readProfile(fp_phase* out, uint32_t* count);
  cudaStream_t stream() const { return stream_; }
  const std::string& error() const { return error_; }
  int fail(int code, const std::string& message) {
    error_ = message;
    return code;
  }

 private:
  // configuration
  int device_;
  int B_, shift_, N_, W_, brickLevels_, bottom_;
  float h_;
  bool maccormack_;
  int precision_;
  double budget_;
  float cutoff_ = 0.f;
  bool ground_ = true;
  int sms_ = 148;
  cudaStream_t stream_ = nullptr;
  std::string error_;

  // host state
  TileDirectory dir_;
  int capacity_ = 0;
  std::vector<int4> tileRec_;
  std::vector<int> tileNbr_;
  std::vector<int4> hash_;
  double time_ = 0;
  int64_t steps_ = 0;
  bool mayHaveFlame_ = false;
  bool solidsStale_ = true;
  bool geometryDirty_ = true;
  int colliderCount_ = 0;
  std::vector<uint8_t> prevColliders_;
  std::vector<uint32_t> prevMasks_;
  std::vector<std::pair<int4, uint32_t>> contentTiles_;
  uint32_t activeBricks_ = 0, usedSlots_ = 0, lastFailures_ = 0;
  bool poolLimited_ = false;
  int latest_ = 0;  // index of the latest pressure solution
  uint32_t slots_ = 0;
  bool pendingRead_ = false;
  int64_t readStep_ = -1;

  // device memory
  std::vector<DeviceBuffer*> owned_;
  DeviceBuffer pages_, entries_, state_, activity_, records_, blockCounts_, active_, zeroList_;
  DeviceBuffer freeStack_, counters_;
  DeviceBuffer vel_[4], curl_, fld_[3], expn_, div_, vmin_, vmax_, sb_, donors_, solids_;
  DeviceBuffer p0_[2], topo_[FP_MAX_LEVELS], lp_[FP_MAX_LEVELS][2], lrhs_[FP_MAX_LEVELS];
  DeviceBuffer tileRecD_, tileNbrD_, hashD_;
  DeviceBuffer emittersD_, collidersD_, masksD_, forcesD_, regionsD_, tileListsD_;
  DeviceBuffer noise_, paramsD_;
  int velIdx_[4] = {0, 1, 2, 3};  // start, predictor/projected, corrected, forced
  int fldIdx_[3] = {0, 1, 2};     // start, predictor, evolved

  // pinned host staging
  SimParams* paramsH_ = nullptr;
  uint8_t* stageH_ = nullptr;  // pinned arena of the step's host-to-device copies
  size_t stageCap_ = 0, stageUsed_ = 0;
  uint32_t* readH_ = nullptr;
  size_t readWords_ = 0;
  cudaEvent_t readEvent_ = nullptr;

  // per-phase device timing (GpuProfiler.ts), and the launch count
  enum PhaseId { PH_ALLOC, PH_TOPO, PH_PREDICT, PH_CORRECT, PH_EVOLVE, PH_CURL, PH_FORCES, PH_DIVERGENCE,
                 PH_MULTIGRID, PH_PROJECT, PH_COUNT };
  struct Phase {
    uint64_t launches = 0, stepLaunches = 0;
    double ms = 0, voxels = 0;
    bool used = false;
    cudaEvent_t a = nullptr, b = nullptr;
  };
  Phase phases_[PH_COUNT];
  bool profiling_ = false;
  bool profilePending_ = false;
  uint64_t launches_ = 0;
  uint64_t h2d_ = 0, d2h_ = 0, stepH2d_ = 0, stepD2h_ = 0;
  double hostPrepareMs_ = 0, hostWaitMs_ = 0;
  void phaseBegin(int id);
  void phaseEnd(int id, int launches);

  // The step's launch sequence as CUDA graphs, one per shape (capacity, solids, topology
  // rebuild, curl, pressure buffer parity). Kernel arguments hold buffer addresses, so any
  // reallocation clears the cache.
  struct GraphEntry {
    cudaGraphExec_t exec;
    int latest;
    uint64_t launches;
  };
  std::unordered_map<uint64_t, GraphEntry> graphs_;
  void enqueueKernels(bool solids, bool topoAll, bool curl, int& latest, uint64_t& launches);
  void clearGraphs();

  // per-step scene (host)
  std::vector<FpEmitter> emitters_;
  std::vector<FpCollider> colliders_;
  std::vector<uint32_t> masks_;
  std::vector<FpForce> forces_;
  std::vector<FpRegion> regions_;
  std::vector<uint32_t> tileLists_;
  FpFlame flame_;

  bool alloc(DeviceBuffer& b, size_t bytes, bool zero = true);
  bool grow(DeviceBuffer& b, size_t bytes, int fill);  // keeps contents
  bool upload(DeviceBuffer& b, const void* src, size_t bytes);
  void freeAll();
  int check(cudaError_t e, const char* what);
  uint32_t slotLimit() const;
  int levelShift(int level) const { return level < brickLevels_ ? brickLevels_ - level : brickLevels_ + 2 - level; }
  int levelCells(int level) const { int s = levelShift(level); return 1 << (3 * s); }

  int allocatePools(uint32_t slots);
  int growPool(uint32_t target);
  int setCapacity(int capacity);
  int applyTiles();
  void updateTiles(const fp_frame& f);
  int packFlame(const fp_combustion& c, float dt);
  bool packScene(const fp_frame& f);
  void bin(int kind, int index, const double* lo, const double* hi, std::vector<std::vector<uint32_t>>& lists);
  int uploadScene();
  void fillParams(const fp_frame& f, float dt);
  int consumeReadback();
  void vcycle(int level, int cur[]);
  float* P0(int k) { return (float*)p0_[k].ptr; }
  float* LP(int level, int k) { return level == 0 ? P0(k) : (float*)lp_[level][k].ptr; }
  float* RHS(int level) { return level == 0 ? (float*)div_.ptr : (float*)lrhs_[level].ptr; }
  SimParams* dParams() { return (SimParams*)paramsD_.ptr; }
};

}  // namespace fp
