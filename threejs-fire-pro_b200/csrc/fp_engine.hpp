// Host side of the step.
//
// `Engine` is one simulation: the C++ counterpart of the reference's `FluidSimulation`
// (src/engine/FluidSimulation.ts) and `TileDirectory` (src/engine/TileDirectory.ts). It owns
// the simulation's device pools and tables, keeps the tile directory and packs each step's
// scene on the host.
//
// `Stepper` launches steps. One step of any number of simulations (all with the same brick
// size) is one host-to-device copy of their parameters and scenes, then one CUDA graph whose
// kernels each cover every simulation's bricks (fp_launch.h). A single simulation is a batch
// of one; the batch and serving front ends step many at once.
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
class Engine;

class TileDirectory {
  friend class Engine;  // a snapshot saves and restores the directory whole

 public:
  struct Tile {
    int x, y, z;
    int64_t needed;
    bool closing;
    bool alive;
    uint64_t seq;  // creation order (the reference's Map keeps tiles in insertion order)
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
  uint64_t nextSeq_ = 0;
};

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

class Stepper;

class Engine {
 public:
  Engine(const fp_grid& grid, Stepper* owner);
  ~Engine();

  // Device pools of the whole voxel budget and an empty directory (FluidSimulation.ts:496-549).
  int initialize();
  int reset();
  int setRuntime(float cutoff, double budget, int ground);
  int stats(fp_stats* out);
  int readField(int field, float* host, size_t bytes);
  int readTable(int table, void* host, size_t* bytes);
  int readBricks(float* boxes, uint32_t* count);
  const std::string& error() const { return error_; }
  int fail(int code, const std::string& message) {
    error_ = message;
    return code;
  }
  int brickSize() const { return B_; }
  // Device bytes a simulation of this grid holds once its pools exist, with `tiles` tile
  // slots (for admission).
  static uint64_t estimateBytes(const fp_grid& grid, uint32_t tiles = 0);
  static uint32_t tilesForBudget(double budget, int cells);
  int reserveTiles(uint32_t tiles);
  uint64_t memoryBytes() const;

  // ---- the Stepper's side of a step
  // Checks the frame and dt without changing any state (FluidSimulation.ts:1367-1369,
  // flame.ts:43-87).
  int validate(const fp_frame& frame, float dt);
  // Host work before the launch: pool growth, tiles, scene packing.
  int prepare(const fp_frame& frame, float dt);
  // Bytes the packed scene takes in the launch's upload, 256-byte aligned blobs.
  size_t sceneBytes() const;
  // Copy the packed scene into the upload at `off` and fill the step's SimParams.
  void writeStep(SimParams& P, uint8_t* hostBase, uint8_t* devBase, size_t off, const fp_frame& frame, float dt,
                 uint32_t* readback, const float4* noise);
  bool buildSolids() const { return colliderCount_ > 0 || solidsStale_; }
  bool solidsAll() const { return solidsStale_; }
  bool topoAll() const { return geometryDirty_ || schedule_.topology != 0; }
  int capacity() const { return capacity_; }
  int liveTiles() const { return (int)liveTiles_.size(); }
  int smokeDivisor() const { return smokeDiv_; }
  int velocityDivisor() const { return vd_; }
  size_t readbackWords() const { return (sizeof(FpCounters) + sizeof(FpSolver)) / 4 + (size_t)capacity_; }
  // Pressure solve (no reference counterpart; the reference runs one V-cycle): up to
  // `vcycles` V-cycles a step, stopping at a relative FP64 residual of `tolerance` (0: all).
  int setSolver(int vcycles, float tolerance);
  int readSolver(fp_solver_stats* out);
  int readBounds(fp_bounds* out);
  // The whole state between steps, host and device, as one blob (fp_sim_snapshot), and back
  // into a simulation of the same grid (fp_sim_restore).
  int snapshot(std::vector<uint8_t>& out);
  int restore(const uint8_t* data, size_t bytes);
  // The solve's smoother, levels, sweeps and Krylov wrapper (fp_sim_set_schedule).
  int setSchedule(const fp_solver_schedule& schedule);
  const fp_solver_schedule& schedule() const { return schedule_; }
  // Volume rendering of the latest state (fp_render.cu) into device memory `image` (enqueued),
  // or into host memory `host` (waits).
  int render(const fp_camera& camera, const fp_render_settings& settings, float* image, float* host);
  // Scene-light sums of the latest state (fp_sim_collect_lights), into host `sums`.
  int collectLights(const fp_render_settings& settings, const float* anchors, uint32_t count, float* sums);
  int vcycles() const { return vcycles_; }
  // Whether the step measures the residual and the post-projection divergence.
  bool measures() const { return vcycles_ > 1 || tolerance_ > 0.f || measure_; }
  // After the launch: buffers rotate, time advances; the measurement is pending.
  void launched(float dt, int latest);
  // The measurement this simulation's last launch wrote (readActivity, FluidSimulation.ts:1701-1746).
  void applyReadback(const uint32_t* words);

 private:
  Stepper* owner_;
  // configuration
  int B_, shift_, N_, W_, brickLevels_, bottom_;
  int vd_, VB_, vshift_, VN_;  // the velocity lattice: velocityDivisor d, B/d cells a side
  float h_;
  bool maccormack_;
  int precision_;
  double budget_;
  float cutoff_ = 0.f;
  bool ground_ = true;
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
  uint64_t bricksStepped_ = 0;  // computing bricks summed over the measured steps
  bool poolLimited_ = false;
  int latest_ = 0;  // index of the latest pressure solution
  int vcycles_ = 1;
  float tolerance_ = 0.f;
  fp_solver_schedule schedule_{};  // zeroed: the reference's Jacobi V-cycle
  // The CG buffers (p0_[2], kry_) for `slots` slots when the schedule wraps the V-cycle in CG.
  int krylovPools(uint32_t slots);
  bool measure_ = false;
  FpSolver lastSolver_{};
  uint32_t slots_ = 0;
  uint64_t stepH2d_ = 0, stepD2h_ = 0;

  // device memory
  DeviceBuffer pages_, entries_, state_, activity_, records_, blockCounts_, active_, zeroList_;
  DeviceBuffer freeStack_, counters_;
  DeviceBuffer vel_[4], curl_, fld_[3], expn_, div_, sb_, donors_, solids_;
  DeviceBuffer p0_[3], topo_[FP_MAX_LEVELS], lp_[FP_MAX_LEVELS][2], lrhs_[FP_MAX_LEVELS];
  DeviceBuffer kry_[3];  // flexible CG: residual, direction, A direction (p0_[2] its iterate)
  DeviceBuffer tileRecD_, tileNbrD_, hashD_, solver_, tileMask_, liveTilesD_, tileIndexD_;
  DeviceBuffer bounds_;  // FpBounds: the bounds-checked build's record
  std::vector<int> liveTiles_, tileIndex_;  // live tile slots ascending; slot -> position or -1
  int velIdx_[4] = {0, 1, 2, 3};  // start, predictor/projected, corrected, forced
  int fldIdx_[3] = {0, 1, 2};     // start, predictor, evolved
  // Coarse smoke (smoke_divisor d > 1): SB_ = B/d cells a side (2^sshift_), SN_ a slot; the
  // pools trade like the scalars' (start, predictor, evolved), the donor range beside them.
  int smokeDiv_ = 1, SB_ = 0, sshift_ = 0, SN_ = 0;
  DeviceBuffer smoke_[3], smokeBnd_;
  int smokeIdx_[3] = {0, 1, 2};
  // Mesh emission: the records (0: none), per brick id its table (-1 none) then the tables'
  // record indices; rebuilt when the records or the tiles (tileVersion_) change.
  std::vector<FpMeshSource> meshRecords_;
  std::vector<int> meshTables_;
  DeviceBuffer meshTablesD_, meshSourcesD_;
  int meshCount_ = 0;
  uint64_t tileVersion_ = 0, meshVersion_ = ~0ull;
  // Mesh force targets' coverage of velocity cells by brick (force-fields.wgsl:13-47): the
  // table, and the targets (force index, cell count, cells) it was built from.
  std::vector<uint32_t> coverage_;
  std::vector<int32_t> coverageTargets_;
  DeviceBuffer coverageD_;
  bool coverageOn_ = false;
  uint64_t coverageVersion_ = ~0ull;
  bool sceneUploadFailed_ = false;

  // rendering: the box in bricks (inclusive) from the latest step's content and sources, the
  // render pools and the parameters of a render
  // TileDirectory.clusters (TileDirectory.ts:189-237), built with the tables: each tile slot's
  // cluster (-1 none) and each cluster's box of tiles (lo xyz, hi xyz); the render boxes of the
  // latest step in bricks (lo xyz, hi xyz inclusive), one per cluster with content or sources.
  std::vector<int> clusterOf_, clusterBoxes_, renderBoxes_;
  void buildClusters();
  std::vector<int> sourceBoxes_;  // lo xyz, hi xyz per source
  DeviceBuffer renderField_, renderSmoke_, sceneDepth_, slices_, lighting_, occupancy_, lut_, renderParams_, image_, anchors_, lightSums_, renderBoxesD_;
  SimParams* renderParamsH_ = nullptr;
  // The blackbody table and the render parameters of the latest state (device).
  int renderInputs();
  void updateRenderBox();

  // pinned staging of the directory tables' copies
  uint8_t* stageH_ = nullptr;
  size_t stageCap_ = 0, stageUsed_ = 0;
  uint64_t h2d_ = 0;

  // per-step scene (host)
  std::vector<FpEmitter> emitters_;
  std::vector<FpCollider> colliders_;
  std::vector<uint32_t> masks_;
  std::vector<FpForce> forces_;
  std::vector<FpRegion> regions_;
  std::vector<uint32_t> tileLists_;
  FpFlame flame_;

  cudaStream_t stream() const;
  // Bytes a value of the scalar pools and of the coarse multigrid levels takes.
  size_t scalarBytes() const { return precision_ == FP_PRECISION_MIXED ? 2 : 4; }
  size_t coarseBytes() const { return precision_ == FP_PRECISION_MIXED ? 2 : 4; }
  bool alloc(DeviceBuffer& b, size_t bytes, bool zero = true);
  bool grow(DeviceBuffer& b, size_t bytes, int fill);  // keeps contents
  bool upload(DeviceBuffer& b, const void* src, size_t bytes);
  void freeAll();
  int check(cudaError_t e, const char* what);
  int consume();
  uint32_t slotLimit() const;
  int levelShift(int level) const { return level < brickLevels_ ? brickLevels_ - level : brickLevels_ + 2 - level; }
  int levelCells(int level) const { int s = levelShift(level); return 1 << (3 * s); }

  int allocatePools(uint32_t slots);
  int growPool(uint32_t target);
  int setCapacity(int capacity);
  int applyTiles();
  void updateTiles(const fp_frame& f);
  int packFlame(const fp_combustion& c, float dt, FpFlame& out);
  bool packScene(const fp_frame& f);
  void bin(int kind, int index, const double* lo, const double* hi, std::vector<std::vector<uint32_t>>& lists);
};

class Stepper {
 public:
  Stepper(int device, int brickSize);
  ~Stepper();
  int initialize();
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }
  int brickSize() const { return B_; }
  const std::string& error() const { return error_; }

  // One step of `count` simulations in one launch. Every frame and dt is checked before any
  // simulation changes; a failure names the simulation's position.
  int step(Engine* const* sims, const fp_frame* const* frames, const float* dts, int count);
  // Wait for the last launch's measurement and hand it to its simulations.
  int consume();
  // A simulation leaves: its pending measurement is dropped.
  void forget(const Engine* e);
  int synchronize();
  int setProfiling(bool on);
  int readProfile(fp_phase* out, uint32_t* count);
  uint64_t launches() const { return launches_; }
  double hostPrepareMs() const { return hostPrepareMs_; }
  double hostWaitMs() const { return hostWaitMs_; }
  // Host-mapped measurement words of the i-th simulation of the last launch: its counters
  // (FpCounters), then its tile words. Valid once the launch's measurement completed, until
  // the next launch.
  const uint32_t* lastReadback(int i) const { return readH_ + pending_[i].second; }
  uint64_t lastUploadBytes() const { return lastUpload_; }
  uint64_t lastReadbackBytes() const { return lastReadback_; }
  const float4* noise() const { return (const float4*)noise_; }

 private:
  int device_, B_, brickLevels_, bottom_;
  int vd_ = 0;  // the simulations' velocity divisor, from the first step
  int sms_ = 148;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t readEvent_ = nullptr;
  // A second stream the step forks work onto where nothing on the main stream depends on it yet:
  // the multigrid topology (joined before the divergence) beside the transport kernels, the curl
  // (joined before the forces) beside evolution. Not while profiling (phases stay serial).
  cudaStream_t side_ = nullptr;
  cudaEvent_t forkTopo_ = nullptr, joinTopo_ = nullptr, forkCurl_ = nullptr, joinCurl_ = nullptr, joinSmoke_ = nullptr;
  std::string error_;
  void* noise_ = nullptr;

  // The launch's upload: work rows, then SimParams per simulation, then the scenes.
  uint8_t* arenaH_ = nullptr;
  uint8_t* arenaD_ = nullptr;
  size_t arenaCap_ = 0;
  int maxSims_ = 0;  // simulations the work rows and parameters have room for
  // Host-mapped measurement words of every simulation of the launch.
  uint32_t* readH_ = nullptr;
  uint32_t* readD_ = nullptr;  // its device alias
  size_t readCap_ = 0;
  std::vector<std::pair<Engine*, size_t>> pending_;  // simulation, word offset
  bool pendingRead_ = false;

  uint64_t launches_ = 0, lastUpload_ = 0, lastReadback_ = 0;
  double hostPrepareMs_ = 0, hostWaitMs_ = 0;

  // per-phase device timing (GpuProfiler.ts)
  enum PhaseId { PH_ALLOC, PH_TOPO, PH_PREDICT, PH_CORRECT, PH_EVOLVE, PH_SMOKE, PH_CURL, PH_FORCES, PH_DIVERGENCE,
                 PH_MULTIGRID, PH_PROJECT, PH_COUNT };  // in the order the step runs them
  struct Phase {
    uint64_t launches = 0, stepLaunches = 0;
    double ms = 0, voxels = 0;
    bool used = false;
    cudaEvent_t a = nullptr, b = nullptr;
  };
  Phase phases_[PH_COUNT];
  bool profiling_ = false;
  bool profilePending_ = false;
  void phaseBegin(int id);
  void phaseEnd(int id, int launches);

  // The step's launch sequence as CUDA graphs, one per combination of the optional launches.
  struct GraphEntry {
    cudaGraphExec_t exec;
    int latest;
    uint64_t launches;
  };
  std::unordered_map<uint64_t, GraphEntry> graphs_;
  void clearGraphs();
  FpBatch batch() const;
  void enqueue(bool solidsFresh, bool solidsAll, bool topoAll, bool curl, int vcycles, bool measure, int& latest,
               uint64_t& launches);
  int cycle_ = 0;             // the V-cycle being enqueued
  bool fusedCoarse_ = false;  // the V-cycle below the first tile level runs as k_coarse
  bool anySmoke_ = false;     // a simulation of the launch keeps coarse smoke
  int smokeDiv_ = 0;          // the finest coarse smoke grid's divisor among them (0: none)
  fp_solver_schedule schedule_{};  // the launch's pressure-solve schedule (its simulations')
  int rhs0Sel_ = 2;           // the finest level's right-hand side: the divergence, or the CG residual
  void vcycle(int level, int cur[], uint64_t& launches);
  // One red-black V-cycle from `level` down, in place; from zero when `zero`.
  void vcycleRB(int level, bool zero, uint64_t& launches);
  int check(cudaError_t e, const char* what);
  int reserve(size_t arenaBytes, int sims, size_t readWords);
};

}  // namespace fp
