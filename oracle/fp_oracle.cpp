// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU oracle of Fire Pro's sparse-brick simulation step: a restatement, operation for
// operation, of the reference's WGSL kernels and of the TypeScript engine host that drives
// them. Templated on the real type: double is the FP64 error oracle; float is the FP32
// CPU baseline (OpenMP over bricks). Storage rounding restates the reference's
// half-precision pools when asked (mode "half"), or the mixed mode of this build.
//
// Only tests/, bench.py's `cpu_baseline` leg and __graft_entry__.smoke() may load this.
// Parity unpinned: the reference ships no tests, golden vectors or CPU path, and cannot
// run in this environment (TypeScript without Node; WGSL without a WebGPU device).
//
// Layout. Pools are slot-major: [slot][channel][cell], cells x fastest within a brick.
// The reference keeps each slot in a 3D texture with a one-texel apron that copies the
// first layer of the following bricks; reads through that apron equal reads of the
// neighbour's cells (zero where the neighbour has no slot), so this oracle reads the
// neighbour cells directly. Samples are trilinear with exact weights.
//
// Citations are path:line in the reference project.

#include <algorithm>
#include <array>
#include <functional>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/firepro.h"
#include "fp_oracle_common.hpp"

namespace orc {

// ---------------------------------------------------------------------------------------
// Tile directory: src/engine/TileDirectory.ts:61-186.
// ---------------------------------------------------------------------------------------
static const int TILE_BRICKS = 4;
static const int LINGER_STEPS = 60;  // TileDirectory.ts:8
static const int MIN_TILES = 16;     // FluidSimulation.ts:72
static const int32_t FRESH_ENTRY = 0x2000000;  // tiles.wgsl:138
static const int RECORD_WORDS = 28;            // FluidSimulation.ts:139

struct Tile {
  I3 coord;
  int slot;
  int64_t needed;
  bool closing;
};

struct Directory {
  // Insertion-ordered, like the JS Map of TileDirectory.ts:62.
  std::map<uint64_t, Tile> bySeq;
  std::unordered_map<uint64_t, uint64_t> byCoord;  // packed coordinates -> sequence
  std::unordered_map<uint64_t, int> slotOf;         // packed coordinates -> tile slot
  uint64_t nextSeq = 0;
  static uint64_t key(int x, int y, int z) {
    return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) |
           (uint64_t)(uint32_t)(z + (1 << 20));
  }
  std::vector<int> slotUsed;  // -1 free, else 1 (TileDirectory.ts:63 `slots`)
  std::vector<int> created;
  bool dirty = true;
  bool ground = true;
  int version = 0;

  int count() const { return (int)bySeq.size(); }
  Tile* find(int x, int y, int z) {
    auto it = byCoord.find(key(x, y, z));
    if (it == byCoord.end()) return nullptr;
    return &bySeq[it->second];
  }
  // TileDirectory.ts:86-108
  void need(I3 lo, I3 hi, int64_t step) {
    for (int z = lo[2]; z <= hi[2]; z++)
      for (int y = ground ? std::max(0, lo[1]) : lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++) {
          Tile* t = find(x, y, z);
          if (t) {
            t->needed = step;
            if (t->closing) {
              t->closing = false;
              dirty = true;
            }
            continue;
          }
          int slot = -1;
          for (size_t i = 0; i < slotUsed.size(); i++)
            if (slotUsed[i] < 0) {
              slot = (int)i;
              break;
            }
          if (slot < 0) {
            slot = (int)slotUsed.size();
            slotUsed.push_back(-1);
          }
          slotUsed[slot] = 1;
          uint64_t seq = nextSeq++;
          bySeq[seq] = Tile{i3(x, y, z), slot, step, false};
          byCoord[key(x, y, z)] = seq;
          slotOf[key(x, y, z)] = slot;
          created.push_back(slot);
          dirty = true;
        }
  }
  // TileDirectory.ts:111-123
  void retire(int64_t step) {
    for (auto it = bySeq.begin(); it != bySeq.end();) {
      Tile& t = it->second;
      if (t.closing) {
        slotUsed[t.slot] = -1;
        byCoord.erase(key(t.coord[0], t.coord[1], t.coord[2]));
        slotOf.erase(key(t.coord[0], t.coord[1], t.coord[2]));
        it = bySeq.erase(it);
        dirty = true;
        continue;
      }
      if (step - t.needed > LINGER_STEPS) {
        t.closing = true;
        dirty = true;
      }
      ++it;
    }
    while (!slotUsed.empty() && slotUsed.back() < 0) slotUsed.pop_back();
  }
  void clear() {
    bySeq.clear();
    byCoord.clear();
    slotOf.clear();
    slotUsed.clear();
    created.clear();
    dirty = true;
  }
  int slotAt(int x, int y, int z) const {
    auto it = slotOf.find(key(x, y, z));
    return it == slotOf.end() ? -1 : it->second;
  }
  std::vector<int> takeCreated() {
    std::vector<int> out;
    for (int s : created)
      if (s < (int)slotUsed.size() && slotUsed[s] >= 0) out.push_back(s);
    created.clear();
    return out;
  }
};

// ---------------------------------------------------------------------------------------
// Packed scene records (fluid-common.wgsl:34-51; FluidSimulation.ts:1150-1366).
// ---------------------------------------------------------------------------------------
template <class R>
struct Emitter {
  R pos[3];
  bool enabled;
  R size[3];
  bool box;
  R flame, heat, smoke, response;  // rates.xyzw
  R vel[3];
  R outward;                       // velocity.w
  R period, strength, fuel;        // variation.xyz
};

template <class R>
struct Collider {
  int kind;  // 0 ellipsoid, 1 box, 2 mesh
  R center[3];
  R extent[3];
  R axes[3][3];  // columns
  int lo[3];
  int size[3];
  uint32_t first;  // word offset of the mask
};

template <class R>
struct Force {
  R axis[3];
  R strength;
  R center[3];
  int kind;
  R scale, lift, inward;
  int regionFirst, regionCount;
  bool targeted;
  bool hasMesh;
};
template <class R>
struct Region {
  R center[3];
  bool box;
  R size[3];
};

template <class R>
struct FlameP {
  R dt, lifespan, smoke, heat, expansion;
  int counts[3];
  R knots[3][8][2];
};

struct Prec {
  int vel = STORE_EXACT, scal = STORE_EXACT, expn = STORE_EXACT, p0 = STORE_EXACT, pc = STORE_EXACT;
  int curl = STORE_EXACT, bounds = STORE_EXACT;
  bool truncate = false;  // truncateHalf at the reference's hand-offs
};

// Activity flags (fluid-content.wgsl:11-13).
static const uint32_t CONTENT = 1u, EXPANDS = 2u, MAY_EXPAND = 4u;
static const uint32_t BRICK_FREES = 8u, BRICK_REQUESTS = 16u;  // fluid-allocation.wgsl:40-41
static const uint8_t STORED_SOLID = 64u;                       // pressure.wgsl:159
static const uint32_t SOLID = 1024u;                           // pressure.wgsl:168

static inline int neighborIndex(int dx, int dy, int dz) { return (dz + 1) * 9 + (dy + 1) * 3 + dx + 1; }

template <class R>
struct Sim {
  // --- configuration
  int B, shift, N, W;  // brick cells per side, log2, cells per brick, solid words per slot
  // The velocity and pressure lattice (velocityDivisor d, FluidSimulation.ts:365-373): B/d
  // cells a brick side at spacing h d, the brick footprint shared with the field lattice.
  int vd = 1, VB, vshift, VN;
  R vh;
  R h;                 // voxel size (float value)
  bool maccormack;
  Prec prec;
  int brickLevels, bottom;
  double voxelBudget = 8e6;
  float cutoff = 0.0f;
  bool ground = true;

  // --- host state (FluidSimulation.ts fields)
  Directory dir;
  int capacity = 0;  // tile slots
  std::vector<I3> snapshot;  // tile coordinates per slot at the last tables build
  std::vector<int> snapshotState;
  std::vector<int32_t> tileNeighbors;  // 27 per tile slot
  double time = 0;
  int64_t steps = 0;
  bool mayHaveFlame = false;
  bool solidsStale = true;
  bool geometryDirty = true;
  int colliderCount = 0;
  std::vector<Collider<R>> prevColliders;
  std::vector<uint32_t> prevMasks;
  std::vector<std::pair<I3, uint32_t>> contentTiles;  // tile coord, brick bits
  uint32_t activeBrickCount = 0, usedSlots = 0, lastFailures = 0;
  bool poolLimited = false;

  // --- per brick id (capacity * 64)
  std::vector<int32_t> pages, entries, records;
  std::vector<uint32_t> state, activity;  // activity: bricks then tile slots

  // --- pool
  uint32_t slots = 0;
  std::vector<uint32_t> freeStack;
  int32_t freeCount = 0;
  uint32_t failures = 0;
  std::vector<R> vel, velP, velC, velF, curl;  // [slot][3 or 4][N]
  std::vector<R> fld, fldP, fldN;              // [slot][4][N]
  std::vector<R> expn, div;                    // [slot][N]
  std::vector<R> vmin, vmax;                   // velocity donor bounds [slot][3][N]
  std::vector<R> sb;                           // scalar bounds [slot][8][N]
  std::vector<int32_t> vdonor;                 // velocity donor bases [slot][3][N][3]
  std::vector<uint32_t> solids;                // [slot][W]
  // Coarse smoke (smokeDivisor d > 1, smoke.wgsl): density on its own grid of SB = B/d cells
  // a brick side at spacing sp = h d; smk the state, smkP the predictor, smkN the evolved,
  // smkBnd the donors' min and max [slot][2][SN].
  int smokeDiv = 1, SB = 0, sshift = 0, SN = 0;
  R sp = 0;
  std::vector<R> smk, smkP, smkN, smkBnd;
  // multigrid: per level p (ping-pong), rhs, topology
  struct Level {
    std::vector<R> p[2], rhs;
    std::vector<uint8_t> topo;
    int current = 0;
  };
  std::vector<Level> levels;
  std::vector<R> pres[2];  // level 0 pressures
  int latest = 0;
  int vcycles = 1;  // V-cycles a step; later ones are defect corrections of the finest level
  // The solve's schedule (fp_solver_schedule): the reference's Jacobi V-cycle, or red-black
  // Gauss-Seidel on the `mgLevels` finest levels; optionally flexible CG around either.
  int smoother = FP_SMOOTHER_JACOBI, mgLevels = 0, preSweeps = 2, postSweeps = 2, bottomSweeps = 8;
  int krylov = FP_KRYLOV_NONE;
  int topologyEachStep = 0;  // the schedule's topology 1: every brick's topology rebuilt each step
  float tolerance = 0;  // CG: stop once RMS residual <= tolerance x RMS right-hand side
  std::vector<R>* rhs0 = nullptr;  // the finest level's right-hand side: the divergence, or the CG residual
  std::vector<R> kx, ks, kd, kq;   // CG: iterate, residual (rhs + A x), direction, A direction
  std::vector<double> cgRes2;      // CG: the residual's sum of squares after each V-cycle

  // --- per step scene
  std::vector<Emitter<R>> emitters;
  std::vector<Collider<R>> colliders;
  std::vector<uint32_t> masks;
  std::vector<Force<R>> forces;
  std::vector<Region<R>> regions;
  std::set<std::array<int, 4>> coverage;  // (force, x, y, z) of the velocity cells mesh targets cover
  std::vector<std::vector<int>> lists[3];  // per kind, per tile slot
  FlameP<R> flame;
  std::vector<V3<float>> noiseTable;  // 64^3 curl noise (built once)
  // uniforms of the step
  R dt, buoyancy, coolingK, smokeWeight, damping, dissipation, vorticity;
  R timeU, seedU;
  uint32_t seedBits;
  bool lifetimeZero;
  bool fuelEnabled;
  R ignition, burnRate;
  int held = 0;
  bool solidsAll = false;

  // --- step-local lists
  std::vector<uint32_t> active;                      // brick ids
  std::vector<std::pair<uint32_t, uint32_t>> zeroed;  // id, slot | fresh<<31

  // ================================================================================
  Sim(const fp_grid& g, Prec p) {
    B = g.brick_size;
    shift = B == 8 ? 3 : (B == 16 ? 4 : 5);
    N = B * B * B;
    W = N / 32;
    h = (R)(float)g.voxel_size;
    maccormack = g.scalar_maccormack != 0;
    prec = p;
    smokeDiv = g.smoke_divisor > 1 ? g.smoke_divisor : 1;
    SB = B / smokeDiv;
    sshift = 0;
    while ((1 << sshift) < SB) sshift++;
    SN = SB * SB * SB;
    sp = h * (R)smokeDiv;  // voxelSize x smokeDivisor: a power of two, exact
    vd = g.velocity_divisor > 1 ? g.velocity_divisor : 1;
    VB = B / vd;
    vshift = 0;
    while ((1 << vshift) < VB) vshift++;
    VN = VB * VB * VB;
    vh = h * (R)vd;  // velocityGrid = voxelSize x velocityDivisor: a power of two, exact
    brickLevels = vshift;  // the pressure lives on the velocity lattice
    bottom = brickLevels + 2;
    if (g.voxel_budget > 0) voxelBudget = g.voxel_budget;
    buildNoise();
    allocate();
  }

  uint32_t slotLimit() const {
    double v = std::floor(voxelBudget / (double)N);
    return (uint32_t)std::max(1.0, v);
  }
  int levelShift(int level) const { return level < brickLevels ? brickLevels - level : brickLevels + 2 - level; }
  int levelSide(int level) const { return 1 << levelShift(level); }
  int levelCells(int level) const { int s = levelSide(level); return s * s * s; }

  // FluidSimulation.ts:496-549 — empty pools and no tiles. The pool holds the whole
  // voxel budget at once; it grows only when the budget does.
  void allocate() {
    slots = slotLimit();
    freeStack.assign(slots, 0);
    for (uint32_t i = 0; i < slots; i++) freeStack[i] = slots - 1 - i;  // pops slot 0 first
    freeCount = (int32_t)slots;
    failures = 0;
    resizePools(slots);
    dir.clear();
    contentTiles.clear();
    capacity = 0;
    setCapacity(MIN_TILES);
    applyTiles();
    solidsStale = true;
    geometryDirty = true;
    usedSlots = 0;
    poolLimited = false;
  }
  void resizePools(uint32_t n) {
    size_t s = n;
    vel.resize(s * 3 * VN, 0); velP.resize(s * 3 * VN, 0); velC.resize(s * 3 * VN, 0); velF.resize(s * 3 * VN, 0);
    curl.resize(s * 4 * VN, 0);
    fld.resize(s * 4 * N, 0); fldP.resize(s * 4 * N, 0); fldN.resize(s * 4 * N, 0);
    expn.resize(s * N, 0); div.resize(s * VN, 0);
    vmin.resize(s * 3 * VN, 0); vmax.resize(s * 3 * VN, 0);
    sb.resize(s * 8 * N, 0);
    vdonor.resize(s * 3 * VN * 3, 0);
    solids.resize(s * W, 0);
    if (smokeDiv > 1) {
      smk.resize(s * SN, 0); smkP.resize(s * SN, 0); smkN.resize(s * SN, 0);
      smkBnd.resize(s * 2 * SN, 0);
    }
    pres[0].resize(s * VN, 0); pres[1].resize(s * VN, 0);
    levels.resize(bottom + 1);
    levels[0].topo.resize(s * VN, 0);
    for (int l = 1; l < brickLevels; l++) {
      size_t c = s * levelCells(l);
      levels[l].p[0].resize(c, 0); levels[l].p[1].resize(c, 0); levels[l].rhs.resize(c, 0);
      levels[l].topo.resize(c, 0);
    }
  }
  // Grow the pool after the voxel budget rose: new slots go under the free stack
  // (FluidSimulation.ts:1013-1093, fluid-pool-growth.wgsl:12-21).
  void growPool(uint32_t target) {
    if (target <= slots) return;
    uint32_t added = target - slots;
    std::vector<uint32_t> next(target, 0);
    for (uint32_t i = 0; i < added; i++) next[i] = slots + added - 1 - i;
    for (uint32_t i = 0; i < slots; i++) next[added + i] = freeStack[i];
    freeStack.swap(next);
    freeCount += (int32_t)added;
    resizePools(target);
    slots = target;
    geometryDirty = true;
  }
  void setCapacity(int cap) {
    int old = capacity;
    capacity = cap;
    size_t bricks = (size_t)cap * 64;
    pages.resize(bricks, -1);
    entries.resize(bricks, -1);
    records.resize(bricks * RECORD_WORDS, -1);
    state.resize(bricks, 0);
    std::vector<uint32_t> act(bricks + cap, 0);
    for (size_t i = 0; i < (size_t)old * 64 && i < activity.size(); i++) act[i] = activity[i];
    activity.swap(act);
    for (int l = brickLevels; l <= bottom; l++) {
      size_t c = (size_t)cap * levelCells(l);
      levels[l].p[0].resize(c, 0); levels[l].p[1].resize(c, 0); levels[l].rhs.resize(c, 0);
      levels[l].topo.resize(c, 0);
    }
    snapshot.resize(cap, i3(0, 0, 0));
    snapshotState.resize(cap, 0);
    tileNeighbors.resize((size_t)cap * 27, -1);
  }
  // FluidSimulation.ts:629-678 applyTiles and TileDirectory.ts:151-186 tables.
  void applyTiles() {
    int needed = std::max(MIN_TILES, (int)dir.slotUsed.size());
    if (needed > capacity) {
      int cap = capacity;
      while (cap < needed) cap *= 2;
      setCapacity(cap);
    }
    std::fill(snapshotState.begin(), snapshotState.end(), 0);
    std::fill(tileNeighbors.begin(), tileNeighbors.end(), -1);
    for (int s = 0; s < capacity; s++) snapshot[s] = i3(0, 0, 0);
    for (auto& kv : dir.bySeq) {
      const Tile& t = kv.second;
      snapshot[t.slot] = t.coord;
      snapshotState[t.slot] = t.closing ? 2 : 1;
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            Tile* n = dir.find(t.coord[0] + dx, t.coord[1] + dy, t.coord[2] + dz);
            if (n) tileNeighbors[(size_t)t.slot * 27 + neighborIndex(dx, dy, dz)] = n->slot;
          }
    }
    dir.dirty = false;
    dir.version++;
    for (int slot : dir.takeCreated()) {
      for (int k = 0; k < 64; k++) {
        size_t id = (size_t)slot * 64 + k;
        pages[id] = -1;
        state[id] = 0;
        activity[id] = 0;
        entries[id] = -1;
      }
    }
    geometryDirty = true;  // PressureSolver.setBricks -> resetPlans
    lookupGen = nextGen();
  }

  // ---------------------------------------------------------------- addressing (tiles.wgsl)
  int tileAt(int x, int y, int z) { return dir.slotAt(x, y, z); }
  static int floordiv(int a, int s) { return a >> s; }
  // The id of world brick b, or -1 (tiles.wgsl:266-272).
  int brickId(int bx, int by, int bz) {
    int t = tileAt(bx >> 2, by >> 2, bz >> 2);
    if (t < 0) return -1;
    return t * 64 + (((bz & 3) * 4 + (by & 3)) * 4 + (bx & 3));
  }
  // The last brick each thread looked up, valid while `lookupGen` is unchanged: entries and
  // tiles change only between the step's phases, when the generation moves on.
  struct LookupCache {
    const void* sim;
    uint64_t gen;
    int bx, by, bz;
    int32_t entry;
  };
  static uint64_t nextGen() {
    static std::atomic<uint64_t> counter{1};
    return ++counter;
  }
  uint64_t lookupGen = nextGen();
  int32_t brickEntry(int bx, int by, int bz) {
    static thread_local LookupCache cache = {nullptr, 0, 0, 0, 0, -1};
    if (cache.sim == this && cache.gen == lookupGen && cache.bx == bx && cache.by == by && cache.bz == bz)
      return cache.entry;
    int id = brickId(bx, by, bz);
    int32_t e = id < 0 ? -1 : entries[id];
    cache = LookupCache{this, lookupGen, bx, by, bz, e};
    return e;
  }
  static int entryPage(int32_t e) { return e < 0 ? -1 : (e & 0xffffff); }
  int brickSlot(int bx, int by, int bz) { return entryPage(brickEntry(bx, by, bz)); }
  I3 brickOf(uint32_t id) {
    I3 t = snapshot[id >> 6];
    int l = id & 63;
    return i3(t[0] * 4 + (l & 3), t[1] * 4 + ((l >> 2) & 3), t[2] * 4 + (l >> 4));
  }
  int local(int x, int y, int z) const { return ((z & (B - 1)) * B + (y & (B - 1))) * B + (x & (B - 1)); }
  // Cell p of a pool of `ch` channels: zero in a brick without a slot (fluid-sampling.wgsl:68-75).
  R cellAt(const std::vector<R>& pool, int ch, int c, int x, int y, int z) {
    int s = brickSlot(x >> shift, y >> shift, z >> shift);
    if (s < 0) return 0;
    return pool[((size_t)s * ch + c) * N + local(x, y, z)];
  }
  // Trilinear sample at `pos` in cell units, centres at .5 (fluid-sampling.wgsl:85-114).
  R sampleCells(const std::vector<R>& pool, int ch, int c, R px, R py, R pz) {
    R q[3] = {px - R(0.5), py - R(0.5), pz - R(0.5)};
    int b[3];
    R f[3];
    for (int a = 0; a < 3; a++) {
      b[a] = floori((double)q[a]);
      f[a] = q[a] - (R)b[a];
    }
    R value = 0;
    for (int z = 0; z < 2; z++)
      for (int y = 0; y < 2; y++)
        for (int x = 0; x < 2; x++) {
          R w = (x ? f[0] : R(1) - f[0]) * (y ? f[1] : R(1) - f[1]) * (z ? f[2] : R(1) - f[2]);
          value += cellAt(pool, ch, c, b[0] + x, b[1] + y, b[2] + z) * w;
        }
    return value;
  }
  // The coarse smoke grid (fluid-sampling.wgsl:4-20: each grid shares the brick footprint,
  // with its own cells per side): cell (x,y,z) of a [slot][SN] pool, zero without a slot, and
  // the trilinear sample at `q` in its cell units, centres at .5.
  R coarseCell(const std::vector<R>& pool, int x, int y, int z) {
    int slot = brickSlot(x >> sshift, y >> sshift, z >> sshift);
    if (slot < 0) return 0;
    int m = SB - 1;
    return pool[(size_t)slot * SN + ((z & m) * SB + (y & m)) * SB + (x & m)];
  }
  R coarseSample(const std::vector<R>& pool, R px, R py, R pz) {
    R q[3] = {px - R(0.5), py - R(0.5), pz - R(0.5)};
    int b[3];
    R f[3];
    for (int a = 0; a < 3; a++) {
      b[a] = floori((double)q[a]);
      f[a] = q[a] - (R)b[a];
    }
    R value = 0;
    for (int z = 0; z < 2; z++)
      for (int y = 0; y < 2; y++)
        for (int x = 0; x < 2; x++) {
          R w = (x ? f[0] : R(1) - f[0]) * (y ? f[1] : R(1) - f[1]) * (z ? f[2] : R(1) - f[2]);
          value += coarseCell(pool, b[0] + x, b[1] + y, b[2] + z) * w;
        }
    return value;
  }
  // Solid test of field cell c (solids.wgsl:15-31).
  bool solidCell(int x, int y, int z) {
    if (ground && y < 0) return true;
    if (colliderCount == 0) return false;
    int s = brickSlot(x >> shift, y >> shift, z >> shift);
    if (s < 0) return false;
    int bit = local(x, y, z);
    return ((solids[(size_t)s * W + (bit >> 5)] >> (bit & 31)) & 1u) != 0;
  }
  // fieldCell (solids.wgsl:7-9): the quarter-cell bias picks one cell on shared corners.
  bool solidAt(R wx, R wy, R wz) {
    return solidCell(floori((double)(wx / h + R(0.25))), floori((double)(wy / h + R(0.25))),
                     floori((double)(wz / h + R(0.25))));
  }
  V3<R> center(int x, int y, int z) { return v3<R>((R(x) + R(0.5)) * h, (R(y) + R(0.5)) * h, (R(z) + R(0.5)) * h); }

  // ---------------------------------------------------------------- velocity sampling
  // The velocity lattice (fluid-sampling.wgsl:4-13: each grid shares the brick footprint with
  // its own cells per side): cell offset, cell of a [slot][ch][VN] pool, trilinear sample in its
  // cell units, a cell's centre.
  int vlocal(int x, int y, int z) const { return ((z & (VB - 1)) * VB + (y & (VB - 1))) * VB + (x & (VB - 1)); }
  R vcell(const std::vector<R>& pool, int ch, int c, int x, int y, int z) {
    int s = brickSlot(x >> vshift, y >> vshift, z >> vshift);
    if (s < 0) return 0;
    return pool[((size_t)s * ch + c) * VN + vlocal(x, y, z)];
  }
  R vsample(const std::vector<R>& pool, int ch, int c, R px, R py, R pz) {
    R q[3] = {px - R(0.5), py - R(0.5), pz - R(0.5)};
    int b[3];
    R f[3];
    for (int a = 0; a < 3; a++) {
      b[a] = floori((double)q[a]);
      f[a] = q[a] - (R)b[a];
    }
    R value = 0;
    for (int z = 0; z < 2; z++)
      for (int y = 0; y < 2; y++)
        for (int x = 0; x < 2; x++) {
          R w = (x ? f[0] : R(1) - f[0]) * (y ? f[1] : R(1) - f[1]) * (z ? f[2] : R(1) - f[2]);
          value += vcell(pool, ch, c, b[0] + x, b[1] + y, b[2] + z) * w;
        }
    return value;
  }
  V3<R> vcenter(int x, int y, int z) { return v3<R>((R(x) + R(0.5)) * vh, (R(y) + R(0.5)) * vh, (R(z) + R(0.5)) * vh); }
  // velocityCellAverage (fluid-sampling.wgsl:268-285): the box average of the field cells under
  // velocity cell (x,y,z), each linear sample on the shared corner of a 2x2x2 block.
  R fieldAverage(const std::vector<R>& pool, int ch, int c, int x, int y, int z) {
    if (vd == 1) return cellAt(pool, ch, c, x, y, z);
    int blocks = vd / 2;
    R sum = 0;
    for (int k = 0; k < blocks; k++)
      for (int j = 0; j < blocks; j++)
        for (int i = 0; i < blocks; i++)
          sum += sampleCells(pool, ch, c, R(x * vd + 1 + 2 * i), R(y * vd + 1 + 2 * j), R(z * vd + 1 + 2 * k));
    return sum / R(blocks * blocks * blocks);
  }
  // fluid-advection.wgsl:9-15: the MAC component at world position `p`.
  R velComp(const std::vector<R>& pool, V3<R> p, int c) {
    V3<R> q = p;
    q[c] -= R(0.5) * vh;
    return vsample(pool, 3, c, q[0] / vh, q[1] / vh, q[2] / vh);
  }
  V3<R> velocityAt(V3<R> p) { return v3<R>(velComp(vel, p, 0), velComp(vel, p, 1), velComp(vel, p, 2)); }
  // fluid-advection.wgsl:26-44
  V3<R> velocityOnFace(int x, int y, int z, int c, V3<R> orig) {
    R fp[3] = {R(x) + R(0.5), R(y) + R(0.5), R(z) + R(0.5)};
    fp[c] += R(0.5);
    V3<R> r;
    for (int k = 0; k < 3; k++) {
      if (k == c) {
        r[k] = orig[k];
        continue;
      }
      R q[3] = {fp[0], fp[1], fp[2]};
      q[k] -= R(0.5);
      r[k] = vsample(vel, 3, k, q[0], q[1], q[2]);
    }
    return r;
  }

  // ---------------------------------------------------------------- scene packing
  void checkFinite(float v, const char* name) {
    if (!std::isfinite(v)) throw std::string(name) + " must be finite in f32.";
  }
  // flame.ts:43-87 packFlameStep
  void packFlame(const fp_combustion& c, float dtf) {
    float step = dtf, lifespan = c.lifespan;
    checkFinite(step, "Flame timestep");
    checkFinite(lifespan, "Flame lifespan");
    if (step <= 0 || lifespan <= 0) throw std::string("Flame timestep and lifespan must be positive in f32.");
    checkFinite(step / lifespan, "Lifetime decrement");
    checkFinite(c.smoke_rate, "Smoke rate");
    checkFinite(c.heat_rate, "Heat rate");
    checkFinite(c.expansion_rate, "Expansion rate");
    if (c.smoke_rate < 0 || c.heat_rate < 0) throw std::string("Smoke and heat rates must be nonnegative.");
    const char* names[3] = {"smoke", "heat", "expansion"};
    flame.dt = step; flame.lifespan = lifespan; flame.smoke = c.smoke_rate; flame.heat = c.heat_rate;
    flame.expansion = c.expansion_rate;
    for (int ch = 0; ch < 3; ch++) {
      const fp_flame_ramp& r = c.ramps[ch];
      if (r.count < 2 || r.count > 8) throw std::string(names[ch]) + " ramp needs 2–8 knots.";
      float prev = -1;
      for (uint32_t i = 0; i < r.count; i++) {
        float x = r.knots[i][0], y = r.knots[i][1];
        if (!std::isfinite(x)) throw std::string(names[ch]) + " lifetime must be finite in f32.";
        if (!std::isfinite(y)) throw std::string(names[ch]) + " response must be finite in f32.";
        if (x < 0 || x > 1 || y < 0 || y > 1 || x <= prev)
          throw std::string(names[ch]) + " knots must increase in f32 with coordinates in [0,1].";
        if ((i == 0 && x != 0) || (i == r.count - 1 && x != 1))
          throw std::string(names[ch]) + " ramp must span lifetime 0–1.";
        flame.knots[ch][i][0] = x;
        flame.knots[ch][i][1] = y;
        prev = x;
      }
      flame.counts[ch] = (int)r.count;
    }
  }
  // Every tile within the world box, or every tile (FluidSimulation.ts:1163-1188). The
  // reference's host arithmetic is JavaScript's: double precision, whatever the oracle's R.
  void bin(int kind, int index, bool hasBox, const double* lo, const double* hi) {
    double tileSize = double(TILE_BRICKS * B) * (double)h;
    if (!hasBox) {
      for (int s = 0; s < capacity; s++)
        if (snapshotState[s] != 0) lists[kind][s].push_back(index);
      return;
    }
    int l[3], u[3];
    for (int a = 0; a < 3; a++) {
      l[a] = floori(lo[a] / tileSize);
      u[a] = floori(hi[a] / tileSize);
    }
    for (int z = l[2]; z <= u[2]; z++)
      for (int y = l[1]; y <= u[1]; y++)
        for (int x = l[0]; x <= u[0]; x++) {
          int s = dir.slotAt(x, y, z);
          if (s >= 0) lists[kind][s].push_back(index);
        }
  }
  bool packScene(const fp_frame& f) {
    for (int k = 0; k < 3; k++) lists[k].assign(capacity, {});
    double brick = double(B) * (double)h;
    emitters.clear();
    for (uint32_t i = 0; i < f.source_count; i++) {
      const fp_source& s = f.sources[i];
      if (s.shape == FP_SHAPE_MESH) continue;
      Emitter<R> e;
      for (int a = 0; a < 3; a++) {
        e.pos[a] = s.position[a];
        e.size[a] = s.size[a];
        e.vel[a] = s.velocity[a];
      }
      e.enabled = true;
      e.box = s.shape == FP_SHAPE_BOX;
      e.flame = s.flame; e.heat = s.heat_rate; e.smoke = s.smoke_rate; e.response = s.velocity_response;
      e.outward = s.outward_speed;
      e.period = s.has_variation ? s.variation_period : 0.5f;
      e.strength = s.has_variation ? s.variation_strength : 0.0f;
      e.fuel = s.fuel_rate;
      int index = (int)emitters.size();
      emitters.push_back(e);
      double lo[3], hi[3];
      for (int a = 0; a < 3; a++) {
        double ext = std::max((double)s.size[a], 0.03);
        lo[a] = (double)s.position[a] - ext - 2 * brick;
        hi[a] = (double)s.position[a] + ext + 2 * brick;
      }
      bin(0, index, true, lo, hi);
    }
    // Colliders (FluidSimulation.ts:1216-1295).
    colliders.clear();
    masks.assign(f.collider_masks, f.collider_masks + f.collider_mask_words);
    for (uint32_t i = 0; i < f.collider_count; i++) {
      const fp_collider& c = f.colliders[i];
      Collider<R> k{};
      double lo[3], hi[3];
      if (c.shape == FP_SHAPE_MESH) {
        k.kind = 2;
        for (int a = 0; a < 3; a++) {
          k.lo[a] = c.lo[a];
          k.size[a] = c.dims[a];
          lo[a] = (double)c.lo[a] * (double)h;
          hi[a] = (double)(c.lo[a] + c.dims[a]) * (double)h;
        }
        k.first = c.mask_offset;
      } else {
        k.kind = c.shape == FP_SHAPE_BOX ? 1 : 0;
        for (int a = 0; a < 3; a++) {
          k.center[a] = c.position[a];
          k.extent[a] = c.size[a];
          for (int b = 0; b < 3; b++) k.axes[a][b] = c.axes[a][b];
        }
        for (int a = 0; a < 3; a++) {
          double ext = c.size[a];
          if (k.kind == 1)
            ext = std::fabs((double)c.axes[0][a]) * (double)c.size[0] +
                  std::fabs((double)c.axes[1][a]) * (double)c.size[1] +
                  std::fabs((double)c.axes[2][a]) * (double)c.size[2];
          lo[a] = (double)c.position[a] - ext;
          hi[a] = (double)c.position[a] + ext;
        }
      }
      colliders.push_back(k);
      bin(2, (int)i, true, lo, hi);
    }
    bool changed = colliders.size() != prevColliders.size() || masks != prevMasks;
    for (size_t i = 0; !changed && i < colliders.size(); i++)
      changed = std::memcmp(&colliders[i], &prevColliders[i], sizeof(Collider<R>)) != 0;
    prevColliders = colliders;
    prevMasks = masks;
    colliderCount = (int)colliders.size();
    // Forces (ForceFields.ts:41-114).
    forces.clear();
    regions.clear();
    coverage.clear();
    for (uint32_t i = 0; i < f.force_count; i++) {
      const fp_force& s = f.forces[i];
      Force<R> k{};
      for (int a = 0; a < 3; a++) {
        k.axis[a] = s.vector[a];
        k.center[a] = s.center[a];
      }
      k.strength = s.strength;
      k.kind = s.type;
      k.scale = s.scale; k.lift = s.lift; k.inward = s.inward;
      k.targeted = s.targeted != 0;
      k.regionFirst = (int)regions.size();
      k.regionCount = 0;
      bool hasReach = false;
      double lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
      if (k.targeted) {
        for (uint32_t t = 0; t < s.target_count; t++) {
          const fp_source& src = f.force_targets[s.first_target + t];
          if (src.shape == FP_SHAPE_MESH) {
            // A mesh target covers the cells its samples reach; the reach grows by the
            // samples' bounds (position lo, size hi) and a velocity cell (ForceFields.ts:97-107).
            k.hasMesh = true;
            uint32_t ti = s.first_target + t;
            if (!f.target_cell_ranges || f.target_cell_ranges[2 * ti + 1] == 0) continue;
            for (int a = 0; a < 3; a++) {
              double l = (double)src.position[a] - (double)vh, u = (double)src.size[a] + (double)vh;
              if (!hasReach) { lo[a] = l; hi[a] = u; } else { lo[a] = std::min(lo[a], l); hi[a] = std::max(hi[a], u); }
            }
            hasReach = true;
            uint32_t first = f.target_cell_ranges[2 * ti], n = f.target_cell_ranges[2 * ti + 1];
            for (uint32_t c = 0; c < n; c++) {
              const int32_t* cell = f.target_cells + 3 * ((size_t)first + c);
              coverage.insert({(int)i, cell[0], cell[1], cell[2]});
            }
            continue;
          }
          Region<R> r;
          for (int a = 0; a < 3; a++) {
            r.center[a] = src.position[a];
            r.size[a] = src.size[a];
          }
          r.box = src.shape == FP_SHAPE_BOX;
          regions.push_back(r);
          k.regionCount++;
          for (int a = 0; a < 3; a++) {
            double ext = std::max((double)src.size[a], 0.03);
            double l = (double)src.position[a] - ext, u = (double)src.position[a] + ext;
            if (!hasReach) { lo[a] = l; hi[a] = u; } else { lo[a] = std::min(lo[a], l); hi[a] = std::max(hi[a], u); }
          }
          hasReach = true;
        }
      }
      forces.push_back(k);
      if (!k.targeted) {
        bin(1, (int)i, false, nullptr, nullptr);
      } else {
        double l[3], u[3];
        for (int a = 0; a < 3; a++) {
          l[a] = lo[a] - brick;
          u[a] = hi[a] + brick;
        }
        bin(1, (int)i, true, l, u);
      }
    }
    return changed;
  }

  // ---------------------------------------------------------------- host step
  // Mesh emission (FluidSimulation.ts:1318-1351): records from 1 (record 0 is none); per
  // brick id its table, numbered in the records' order, and per table a record a cell.
  std::vector<fp_mesh_source> meshRecords;
  std::vector<int> meshTables;
  void buildMeshTables(const fp_frame& f) {
    meshRecords.assign(1, fp_mesh_source{});
    meshRecords.insert(meshRecords.end(), f.mesh_sources, f.mesh_sources + f.mesh_source_count);
    meshTables.clear();
    if (f.mesh_source_count == 0) return;
    const size_t bricks = (size_t)capacity * 64;
    std::map<int, int> tables;
    std::vector<std::pair<size_t, int>> placed;
    for (int r = 1; r < (int)meshRecords.size(); r++) {
      const int* cell = meshRecords[r].cell;
      int id = brickId(cell[0] >> shift, cell[1] >> shift, cell[2] >> shift);
      if (id < 0) continue;
      auto it = tables.find(id);
      if (it == tables.end()) it = tables.emplace(id, (int)tables.size()).first;
      size_t index = ((((size_t)it->second * B + (cell[2] & (B - 1))) * B + (cell[1] & (B - 1))) * B) + (cell[0] & (B - 1));
      placed.push_back({index, r});
    }
    meshTables.assign(bricks + tables.size() * (size_t)N, 0);
    std::fill(meshTables.begin(), meshTables.begin() + bricks, -1);
    for (auto& t : tables) meshTables[t.first] = t.second;
    for (auto& p : placed) meshTables[bricks + p.first] = p.second;
  }
  int meshTable(int id) const { return meshTables.empty() || id < 0 ? -1 : meshTables[id]; }
  // meshSourceAt (fluid-sources.wgsl:9-22) for field cell (x,y,z): its record (0: none).
  const fp_mesh_source& meshSourceAt(int x, int y, int z) {
    if (meshTables.empty()) return meshRecords[0];
    int table = meshTable(brickId(x >> shift, y >> shift, z >> shift));
    if (table < 0) return meshRecords[0];
    size_t index = (((size_t)table * B + (z & (B - 1))) * B + (y & (B - 1))) * B + (x & (B - 1));
    return meshRecords[meshTables[(size_t)capacity * 64 + index]];
  }
  void needBox(const double* lo, const double* hi, double margin) {
    double size = double(TILE_BRICKS * B) * (double)h;
    I3 l, u;
    for (int a = 0; a < 3; a++) {
      l[a] = floori((lo[a] - margin) / size);
      u[a] = floori((hi[a] + margin) / size);
    }
    dir.need(l, u, steps);
  }
  // FluidSimulation.ts:873-912 updateTiles
  void updateTiles(const fp_frame& f) {
    dir.retire(steps);
    double reach = double(2 * B) * (double)h;
    double margin = reach + double(TILE_BRICKS * B) * (double)h;
    for (uint32_t i = 0; i < f.source_count; i++) {
      const fp_source& s = f.sources[i];
      if (s.shape == FP_SHAPE_MESH) {
        // The samples' bounds, a voxel more margin (FluidSimulation.ts:879-893).
        double lo[3] = {(double)s.position[0], (double)s.position[1], (double)s.position[2]};
        double hi[3] = {(double)s.size[0], (double)s.size[1], (double)s.size[2]};
        needBox(lo, hi, margin + (double)h);
        continue;
      }
      double ext = std::max(std::max(std::max((double)s.size[0], (double)s.size[1]), (double)s.size[2]), 0.03) +
                   (double)s.outward_speed * 0.25;
      double lo[3], hi[3];
      for (int a = 0; a < 3; a++) {
        lo[a] = (double)s.position[a] - ext;
        hi[a] = (double)s.position[a] + ext;
      }
      needBox(lo, hi, margin);
    }
    for (auto& ct : contentTiles)
      dir.need(i3(ct.first[0] - 1, ct.first[1] - 1, ct.first[2] - 1),
               i3(ct.first[0] + 1, ct.first[1] + 1, ct.first[2] + 1), steps);
    if (dir.dirty) applyTiles();
    // The sources' bricks (bricksOver, FluidSimulation.ts:862-868) and the render box.
    sourceBoxes.clear();
    double brick = double(B) * (double)h;
    for (uint32_t i = 0; i < f.source_count; i++) {
      const fp_source& s = f.sources[i];
      if (s.shape == FP_SHAPE_MESH) {
        for (int a = 0; a < 3; a++) sourceBoxes.push_back((int)std::floor((double)s.position[a] / brick));
        for (int a = 0; a < 3; a++) sourceBoxes.push_back((int)std::floor((double)s.size[a] / brick));
        continue;
      }
      double ext = std::max(std::max(std::max((double)s.size[0], (double)s.size[1]), (double)s.size[2]), 0.03) +
                   (double)s.outward_speed * 0.25;
      for (int a = 0; a < 3; a++) sourceBoxes.push_back((int)std::floor(((double)s.position[a] - ext) / brick));
      for (int a = 0; a < 3; a++) sourceBoxes.push_back((int)std::floor(((double)s.position[a] + ext) / brick));
    }
    updateRenderBox();
  }

  // ---------------------------------------------------------------- rendering (test oracle)
  // TileDirectory.clusters (TileDirectory.ts:189-237) and updateBoxes (FluidSimulation.ts:
  // 916-957): tiles grouped by touch in insertion order, groups boxed, overlapping boxes merged
  // until none overlap; then per cluster the content and source bricks whose centre's tile lies
  // in it, two bricks of margin, within the cluster's tiles. Boxes in cluster order, six ints
  // each (lo xyz, hi xyz in bricks, inclusive).
  std::vector<int> renderBoxes;
  std::vector<int> sourceBoxes;
  void updateRenderBox() {
    std::map<uint64_t, int> group;  // tile key -> group
    std::vector<std::array<int, 6>> boxes;
    for (auto& kv : dir.bySeq) {
      const Tile& first = kv.second;
      uint64_t fk = Directory::key(first.coord[0], first.coord[1], first.coord[2]);
      if (group.count(fk)) continue;
      int index = (int)boxes.size();
      std::array<int, 6> box = {first.coord[0], first.coord[1], first.coord[2], first.coord[0], first.coord[1], first.coord[2]};
      group[fk] = index;
      std::vector<I3> stack = {first.coord};
      while (!stack.empty()) {
        I3 c = stack.back();
        stack.pop_back();
        for (int a = 0; a < 3; a++) {
          box[a] = std::min(box[a], c[a]);
          box[3 + a] = std::max(box[3 + a], c[a]);
        }
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              Tile* n = dir.find(c[0] + dx, c[1] + dy, c[2] + dz);
              if (!n) continue;
              uint64_t nk = Directory::key(n->coord[0], n->coord[1], n->coord[2]);
              if (group.count(nk)) continue;
              group[nk] = index;
              stack.push_back(n->coord);
            }
      }
      boxes.push_back(box);
    }
    std::vector<int> into(boxes.size());
    for (size_t i = 0; i < into.size(); i++) into[i] = (int)i;
    std::function<int(int)> root = [&](int i) { return into[i] == i ? i : (into[i] = root(into[i])); };
    auto overlaps = [](const std::array<int, 6>& a, const std::array<int, 6>& b) {
      for (int k = 0; k < 3; k++)
        if (!(a[k] <= b[3 + k] && b[k] <= a[3 + k])) return false;
      return true;
    };
    for (bool merged = true; merged;) {
      merged = false;
      for (size_t i = 0; i < boxes.size(); i++)
        for (size_t j = i + 1; j < boxes.size(); j++) {
          int a = root((int)i), b = root((int)j);
          if (a == b || !overlaps(boxes[a], boxes[b])) continue;
          for (int k = 0; k < 3; k++) {
            boxes[a][k] = std::min(boxes[a][k], boxes[b][k]);
            boxes[a][3 + k] = std::max(boxes[a][3 + k], boxes[b][3 + k]);
          }
          into[b] = a;
          merged = true;
        }
    }
    std::vector<int> renumbered(boxes.size(), -1);
    std::vector<std::array<int, 6>> clusters;
    for (size_t i = 0; i < boxes.size(); i++)
      if (root((int)i) == (int)i) {
        renumbered[i] = (int)clusters.size();
        clusters.push_back(boxes[i]);
      }
    std::map<int, std::array<int, 6>> found;
    auto include = [&](const int* l, const int* u) {
      int c[3];
      for (int a = 0; a < 3; a++) c[a] = (int)std::floor(((double)l[a] + (double)u[a]) / 2.0);
      if (ground) c[1] = std::max(0, c[1]);
      int t[3] = {(int)std::floor(c[0] / 4.0), (int)std::floor(c[1] / 4.0), (int)std::floor(c[2] / 4.0)};
      auto g = group.find(Directory::key(t[0], t[1], t[2]));
      if (g == group.end()) return;
      int cluster = renumbered[root(g->second)];
      auto it = found.find(cluster);
      if (it == found.end()) {
        found[cluster] = {l[0], l[1], l[2], u[0], u[1], u[2]};
        return;
      }
      for (int a = 0; a < 3; a++) {
        it->second[a] = std::min(it->second[a], l[a]);
        it->second[3 + a] = std::max(it->second[3 + a], u[a]);
      }
    };
    for (auto& ct : contentTiles) {
      int l[3], u[3];
      bool ok = true;
      for (int a = 0; a < 3 && ok; a++) {
        uint32_t used = (ct.second >> (a * 4)) & 15u;
        if (!used) {
          ok = false;
          break;
        }
        int low = 0, high = 0;
        while (!((used >> low) & 1u)) low++;
        for (int b = 0; b < 4; b++)
          if ((used >> b) & 1u) high = b;
        l[a] = ct.first[a] * 4 + low;
        u[a] = ct.first[a] * 4 + high;
      }
      if (ok) include(l, u);
    }
    for (size_t k = 0; k + 6 <= sourceBoxes.size(); k += 6) include(&sourceBoxes[k], &sourceBoxes[k + 3]);
    renderBoxes.clear();
    for (auto& kv : found) {
      const std::array<int, 6>& tiles = clusters[kv.first];
      for (int a = 0; a < 3; a++) renderBoxes.push_back(std::max(kv.second[a] - 2, tiles[a] * 4));
      for (int a = 0; a < 3; a++) renderBoxes.push_back(std::min(kv.second[3 + a] + 2, (tiles[3 + a] + 1) * 4 - 1));
    }
  }
  // The box a render thread samples in (its pages and clamps): per thread.
  static int* curBox() {
    static thread_local int b[6] = {0, 0, 0, -1, -1, -1};
    return b;
  }
  void useBox(int k) {
    for (int a = 0; a < 6; a++) curBox()[a] = renderBoxes[(size_t)6 * k + a];
  }
  int boxOf(int bx, int by, int bz) const {
    for (size_t k = 0; k + 6 <= renderBoxes.size(); k += 6) {
      const int* b = &renderBoxes[k];
      if (bx >= b[0] && bx <= b[3] && by >= b[1] && by <= b[4] && bz >= b[2] && bz <= b[5]) return (int)(k / 6);
    }
    return -1;
  }

  // The render (lighting.wgsl, volume-march.wgsl, fire-emission.wgsl,
  // volume-reconstruction.wgsl) in R, cell by cell: the render field, occupancy and lighting
  // of every boxed brick with a slot, then a march per pixel.
  struct Render {
    const fp_camera* cam;
    const fp_render_settings* rs;
    std::vector<float> lut;
    int lightShift;
    std::unordered_map<uint64_t, int> index;  // boxed slotted brick -> row
    std::vector<R> field;                     // [row][4][N]
    std::vector<R> smoke;                     // coarse smoke: [row][SN], smoothed
    std::vector<uint8_t> occupancy;           // [row][blocks]
    std::vector<R> light;                     // [row][4][L^3]
  };
  static uint64_t brickKey(int x, int y, int z) {
    return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) |
           (uint64_t)(uint32_t)(z + (1 << 20));
  }
  bool boxed(int bx, int by, int bz) const {
    const int* b = curBox();
    return bx >= b[0] && bx <= b[3] && by >= b[1] && by <= b[4] && bz >= b[2] && bz <= b[5];
  }
  // The render row of brick b when it lies in the current box.
  template <class G_>
  int rowOf(G_& G, int bx, int by, int bz) {
    if (!boxed(bx, by, bz)) return -1;
    auto it = G.index.find(brickKey(bx, by, bz));
    return it == G.index.end() ? -1 : it->second;
  }
  int boxSlot(int bx, int by, int bz) { return boxed(bx, by, bz) ? brickSlot(bx, by, bz) : -1; }
  static R glowOf(R life) { return std::min(std::max(life * R(5), R(0)), R(1)); }
  R rawSmoke(int x, int y, int z) {
    int s = boxSlot(x >> shift, y >> shift, z >> shift);
    return s < 0 ? R(0) : fld[(size_t)s * 4 * N + local(x, y, z)];
  }
  void clampBox(R q[3], int per) {
    for (int a = 0; a < 3; a++)
      q[a] = std::min(std::max(q[a], R(curBox()[a]) * R(per) + R(.5)), R(curBox()[3 + a] + 1) * R(per) - R(.5));
  }
  R smokeSample(R qx, R qy, R qz) {
    R q[3] = {qx, qy, qz};
    clampBox(q, B);
    R g[3], fr[3];
    int b[3];
    for (int a = 0; a < 3; a++) {
      g[a] = q[a] - R(.5);
      b[a] = (int)std::floor(g[a]);
      fr[a] = g[a] - R(b[a]);
    }
    R v = 0;
    for (int k = 0; k < 8; k++) {
      int d[3] = {k & 1, (k >> 1) & 1, k >> 2};
      R w = (d[0] ? fr[0] : 1 - fr[0]) * (d[1] ? fr[1] : 1 - fr[1]) * (d[2] ? fr[2] : 1 - fr[2]);
      v += rawSmoke(b[0] + d[0], b[1] + d[1], b[2] + d[2]) * w;
    }
    return v;
  }
  R smoothedSmoke(int x, int y, int z) {
    R d = 0;
    for (int k = 0; k < 8; k++) d += smokeSample(R(x + (k & 1)), R(y + ((k >> 1) & 1)), R(z + (k >> 2)));
    return std::max(R(0), d * R(.125));
  }
  // The coarse smoke grid (lighting.wgsl smoothCoarseSmoke :104-129, cachedSmokeCell :133-156,
  // volume-common.wgsl renderSmokeAt :74-78), SB cells a brick side.
  R rawCoarse(int x, int y, int z) {
    int s = boxSlot(x >> sshift, y >> sshift, z >> sshift);
    if (s < 0) return R(0);
    int m = SB - 1;
    return smk[(size_t)s * SN + ((z & m) * SB + (y & m)) * SB + (x & m)];
  }
  R coarseRenderSample(R qx, R qy, R qz) {
    R q[3] = {qx, qy, qz};
    clampBox(q, SB);
    R g[3], fr[3];
    int b[3];
    for (int a = 0; a < 3; a++) {
      g[a] = q[a] - R(.5);
      b[a] = (int)std::floor(g[a]);
      fr[a] = g[a] - R(b[a]);
    }
    R v = 0;
    for (int k = 0; k < 8; k++) {
      int d[3] = {k & 1, (k >> 1) & 1, k >> 2};
      R w = (d[0] ? fr[0] : 1 - fr[0]) * (d[1] ? fr[1] : 1 - fr[1]) * (d[2] ? fr[2] : 1 - fr[2]);
      v += rawCoarse(b[0] + d[0], b[1] + d[1], b[2] + d[2]) * w;
    }
    return v;
  }
  R smoothedCoarse(int x, int y, int z) {
    R d = 0;
    for (int k = 0; k < 8; k++) d += coarseRenderSample(R(x + (k & 1)), R(y + ((k >> 1) & 1)), R(z + (k >> 2)));
    return std::max(R(0), d * R(.125));
  }
  R renderSmokeCell(Render& G, int x, int y, int z, bool apron) {
    int row = rowOf(G, x >> sshift, y >> sshift, z >> sshift);
    int m = SB - 1;
    if (row >= 0) return G.smoke[(size_t)row * SN + ((z & m) * SB + (y & m)) * SB + (x & m)];
    return apron ? smoothedCoarse(x, y, z) : R(0);
  }
  R renderSmokeAt(Render& G, R qx, R qy, R qz) {
    R q[3] = {qx, qy, qz};
    clampBox(q, SB);
    R g[3], fr[3];
    int b[3];
    for (int a = 0; a < 3; a++) {
      g[a] = q[a] - R(.5);
      b[a] = (int)std::floor(g[a]);
      fr[a] = g[a] - R(b[a]);
    }
    bool based = rowOf(G, b[0] >> sshift, b[1] >> sshift, b[2] >> sshift) >= 0;
    R v = 0;
    for (int k = 0; k < 8; k++) {
      int d[3] = {k & 1, (k >> 1) & 1, k >> 2};
      R w = (d[0] ? fr[0] : 1 - fr[0]) * (d[1] ? fr[1] : 1 - fr[1]) * (d[2] ? fr[2] : 1 - fr[2]);
      v += renderSmokeCell(G, b[0] + d[0], b[1] + d[1], b[2] + d[2], based) * w;
    }
    return v;
  }
  R cachedSmokeCell(Render& G, int x, int y, int z) {
    int m = SB - 1, b[3] = {x >> sshift, y >> sshift, z >> sshift}, l[3] = {x & m, y & m, z & m};
    int row = rowOf(G, b[0], b[1], b[2]);
    if (row >= 0) return G.smoke[(size_t)row * SN + (l[2] * SB + l[1]) * SB + l[0]];
    for (int k = 1; k < 8; k++) {
      if (((k & 1) && l[0] != 0) || ((k & 2) && l[1] != 0) || ((k & 4) && l[2] != 0)) continue;
      if (rowOf(G, b[0] - (k & 1), b[1] - ((k >> 1) & 1), b[2] - ((k >> 2) & 1)) >= 0)
        return smoothedCoarse(x, y, z);
    }
    return R(0);
  }
  std::array<R, 4> renderCell(Render& G, int x, int y, int z, bool apron) {
    int row = rowOf(G, x >> shift, y >> shift, z >> shift);
    if (row >= 0) {
      size_t o = (size_t)row * 4 * N + local(x, y, z);
      return {G.field[o], G.field[o + N], G.field[o + 2 * N], G.field[o + 3 * N]};
    }
    // With coarse smoke the render reads the simulation's fields, whose apron holds zero where
    // no neighbour slot is.
    if (!apron || smokeDiv > 1) return {0, 0, 0, 0};
    return {smoothedSmoke(x, y, z), 0, 0, 0};
  }
  std::array<R, 4> renderSample(Render& G, R qx, R qy, R qz) {
    R q[3] = {qx, qy, qz};
    clampBox(q, B);
    R g[3], fr[3];
    int b[3];
    for (int a = 0; a < 3; a++) {
      g[a] = q[a] - R(.5);
      b[a] = (int)std::floor(g[a]);
      fr[a] = g[a] - R(b[a]);
    }
    bool based = rowOf(G, b[0] >> shift, b[1] >> shift, b[2] >> shift) >= 0;
    std::array<R, 4> v = {0, 0, 0, 0};
    for (int k = 0; k < 8; k++) {
      int d[3] = {k & 1, (k >> 1) & 1, k >> 2};
      R w = (d[0] ? fr[0] : 1 - fr[0]) * (d[1] ? fr[1] : 1 - fr[1]) * (d[2] ? fr[2] : 1 - fr[2]);
      auto c = renderCell(G, b[0] + d[0], b[1] + d[1], b[2] + d[2], based);
      for (int ch = 0; ch < 4; ch++) v[ch] += c[ch] * w;
    }
    return v;
  }
  std::array<R, 4> reconstruct(Render& G, R px, R py, R pz, int mode) {
    if (mode == 0) return renderSample(G, px, py, pz);
    R pos[2][3], wt[2][3], p[3] = {px, py, pz};
    for (int a = 0; a < 3; a++) {
      R g = p[a] - R(.5);
      if (mode == 1) {
        R center = std::floor(g + R(.5)), delta = g - center;
        R w0 = R(.5) * (R(.5) - delta) * (R(.5) - delta), w1 = R(.75) - delta * delta,
          w2 = R(.5) * (R(.5) + delta) * (R(.5) + delta);
        wt[0][a] = w0 + w1;
        wt[1][a] = w2;
        pos[0][a] = center - R(.5) + w1 / wt[0][a];
        pos[1][a] = center + R(1.5);
      } else {
        R base = std::floor(g), q = g - base, inv = 1 - q;
        R w0 = inv * inv * inv / 6, w1 = (3 * q * q * q - 6 * q * q + 4) / 6, w2 = (-3 * q * q * q + 3 * q * q + 3 * q + 1) / 6,
          w3 = q * q * q / 6;
        wt[0][a] = w0 + w1;
        wt[1][a] = w2 + w3;
        pos[0][a] = base - R(.5) + w1 / wt[0][a];
        pos[1][a] = base + R(1.5) + w3 / wt[1][a];
      }
    }
    std::array<R, 4> v = {0, 0, 0, 0};
    for (int i = 0; i < 8; i++) {
      int ix = (i >> 2) & 1, iy = (i >> 1) & 1, iz = i & 1;
      auto s = renderSample(G, pos[ix][0], pos[iy][1], pos[iz][2]);
      R w = wt[ix][0] * wt[iy][1] * wt[iz][2];
      for (int ch = 0; ch < 4; ch++) v[ch] += w * s[ch];
    }
    for (int ch = 0; ch < 4; ch++) v[ch] = std::max(v[ch], R(0));
    return v;
  }
  R extinctionOf(Render& G, const std::array<R, 4>& f) {
    return std::max(R(0), f[0]) * R(G.rs->optical[0]) + glowOf(f[2]) * R(G.rs->flame_opacity);
  }
  std::array<R, 3> emissionOf(Render& G, const std::array<R, 4>& f) {
    const fp_render_settings& S = *G.rs;
    if (S.optical[1] <= 0) return {0, 0, 0};
    R s = std::max(R(0), f[0]) * R(S.optical[0]), flame = glowOf(f[2]) * R(S.flame_opacity);
    R source[3];
    for (int c = 0; c < 3; c++) source[c] = (1 - R(S.smoke[c])) * s * R(S.smoke[3]) + flame;
    if (source[0] == 0 && source[1] == 0 && source[2] == 0) return {0, 0, 0};
    R heat = std::max(R(0), f[1]);
    R kelvin = R(800) + heat / (heat + 2) * (R(S.fire[3]) - 800);
    R u = std::min(std::max((kelvin - 500) / 9500, R(0)), R(1)) * R(511);
    int i0 = (int)std::floor(u), i1 = std::min(i0 + 1, 511);
    R fr = u - R(i0), spec[4];
    for (int c = 0; c < 4; c++) spec[c] = R(G.lut[i0 * 4 + c]) * (1 - fr) + R(G.lut[i1 * 4 + c]) * fr;
    R scale = std::exp2(std::min(std::max(spec[3], R(-24)), R(10)));
    R thermal[3] = {spec[0] * scale, spec[1] * scale, spec[2] * scale};
    R tintPeak = std::max(R(S.fire[0]), std::max(R(S.fire[1]), R(S.fire[2])));
    R sat = 1 - std::min(R(S.fire[0]), std::min(R(S.fire[1]), R(S.fire[2]))) / std::max(tintPeak, R(1e-6));
    R peak = std::max(thermal[0], std::max(thermal[1], thermal[2]));
    std::array<R, 3> out;
    for (int c = 0; c < 3; c++)
      out[c] = (thermal[c] * tintPeak * (1 - sat) + R(S.fire[c]) * peak * sat) * source[c] * R(S.optical[1]);
    return out;
  }
  std::array<R, 4> sampleWorld(Render& G, R px, R py, R pz) {
    R size = R(B) * h, p[3] = {px, py, pz};
    for (int a = 0; a < 3; a++)
      if (p[a] < R(curBox()[a]) * size || p[a] > R(curBox()[3 + a] + 1) * size) return {0, 0, 0, 0};
    auto f = renderSample(G, px / h, py / h, pz / h);
    if (smokeDiv > 1) f[0] = renderSmokeAt(G, px / h / R(smokeDiv), py / h / R(smokeDiv), pz / h / R(smokeDiv));
    return f;
  }
  std::array<R, 4> incidentLight(Render& G, R px, R py, R pz) {
    const fp_render_settings& S = *G.rs;
    auto lf = sampleWorld(G, px, py, pz);
    if (lf[0] + glowOf(lf[2]) < R(1e-5)) return {0, 0, 0, 1};
    R ln = std::sqrt(R(S.light[0]) * S.light[0] + R(S.light[1]) * S.light[1] + R(S.light[2]) * S.light[2]);
    R sun[3] = {R(S.light[0]) / ln, R(S.light[1]) / ln, R(S.light[2]) / ln}, p[3] = {px, py, pz};
    R size = R(B) * h, exit = R(1e30);
    for (int a = 0; a < 3; a++) {
      if (!(std::fabs(sun[a]) > R(1e-6))) continue;
      R edge = (sun[a] > 0 ? R(curBox()[3 + a] + 1) : R(curBox()[a])) * size;
      exit = std::min(exit, (edge - p[a]) / sun[a]);
    }
    exit = std::max(R(0), exit);
    int count = (int)S.shadow_samples;
    R ds = exit / R(count), depth = 0;
    if (S.light[3] > 0)
      for (int i = 0; i < count; i++) {
        R t = (R(i) + R(.5)) * ds;
        auto f = sampleWorld(G, px + sun[0] * t, py + sun[1] * t, pz + sun[2] * t);
        depth += (std::max(R(0), f[0]) * R(S.optical[2]) + glowOf(f[2]) * R(S.flame_opacity)) * ds;
        if (depth > 9) break;
      }
    const R dirs[6][3] = {{.36, .48, -.8}, {-.36, -.48, .8}, {-.8, .6, 0}, {.8, -.6, 0}, {.48, .64, .6}, {-.48, -.64, -.6}};
    R glow[3] = {0, 0, 0};
    if (S.optical[1] > 0 && lf[0] > R(1e-5))
      for (int d = 0; d < 6; d++) {
        R t = 0, interval = R(.075), transmission = 1;
        for (int s = 0; s < 6; s++) {
          R q = t + interval * R(.5);
          auto f = sampleWorld(G, px + dirs[d][0] * q, py + dirs[d][1] * q, pz + dirs[d][2] * q);
          R ext = extinctionOf(G, f), att = std::exp(-ext * interval), depth2 = ext * interval;
          R integ = depth2 < R(.001) ? interval * (1 - R(.5) * depth2 + depth2 * depth2 / 6) : (1 - att) / ext;
          auto e = emissionOf(G, f);
          for (int c = 0; c < 3; c++) glow[c] += transmission * e[c] * integ / 6;
          transmission *= att;
          t += interval;
          interval *= R(1.65);
        }
      }
    return {glow[0], glow[1], glow[2], std::exp(-depth)};
  }
  std::array<R, 4> lightSample(Render& G, R qx, R qy, R qz) {
    const int L = 1 << G.lightShift, L3 = L * L * L;
    R texel = h * R(B >> G.lightShift), q[3] = {qx, qy, qz};
    clampBox(q, L);
    R g[3], fr[3];
    int b[3];
    for (int a = 0; a < 3; a++) {
      g[a] = q[a] - R(.5);
      b[a] = (int)std::floor(g[a]);
      fr[a] = g[a] - R(b[a]);
    }
    if (rowOf(G, b[0] >> G.lightShift, b[1] >> G.lightShift, b[2] >> G.lightShift) < 0) return {0, 0, 0, 1};
    std::array<R, 4> v = {0, 0, 0, 0};
    for (int k = 0; k < 8; k++) {
      int d[3] = {k & 1, (k >> 1) & 1, k >> 2};
      int x = b[0] + d[0], y = b[1] + d[1], z = b[2] + d[2];
      R w = (d[0] ? fr[0] : 1 - fr[0]) * (d[1] ? fr[1] : 1 - fr[1]) * (d[2] ? fr[2] : 1 - fr[2]);
      int row = rowOf(G, x >> G.lightShift, y >> G.lightShift, z >> G.lightShift);
      std::array<R, 4> t;
      if (row >= 0) {
        int m = L - 1;
        size_t o = (size_t)row * 4 * L3 + (((z & m) * L + (y & m)) * L + (x & m));
        t = {G.light[o], G.light[o + L3], G.light[o + 2 * L3], G.light[o + 3 * L3]};
      } else {
        t = incidentLight(G, (R(x) + R(.5)) * texel, (R(y) + R(.5)) * texel, (R(z) + R(.5)) * texel);
      }
      for (int c = 0; c < 4; c++) v[c] += t[c] * w;
    }
    return v;
  }
  static R jitterOf(uint32_t px, uint32_t py, float time) {
    uint32_t s0 = px * 1664525u + 1013904223u, s1 = py * 1664525u + 1013904223u,
             s2 = (uint32_t)(time * 60.f) * 1664525u + 1013904223u;
    s0 += s1 * s2;
    s1 += s2 * s0;
    s2 += s0 * s1;
    s0 ^= s0 >> 16u;
    s1 ^= s1 >> 16u;
    s2 ^= s2 >> 16u;
    s0 += s1 * s2;
    return R((float)(s0 >> 8u) / 16777216.f);
  }
  // collectLights (scene-lights.wgsl:37-106): every computing brick samples its cells on a 4^3
  // lattice (stride B/4, at the stride's middle), and adds to the anchor nearest its centre
  // (height above an anchor counting a quarter; ties to the first) the luminance of their
  // emission, its luminance-weighted offset from the anchor and its RGB: 8 floats an anchor.
  void collectLights(const fp_render_settings& rs, const float* lut, const float* anchors, int count, double* sums) {
    Render G;
    G.rs = &rs;
    G.lut.assign(lut, lut + 512 * 4);
    const int stride = B / 4;
    const double side = (double)B * (double)h;
    for (int i = 0; i < count * 8; i++) sums[i] = 0;
    if (count == 0) return;
    for (uint32_t id : active) {
      int slot = entryPage(entries[id]);
      if (slot < 0) continue;
      I3 b = brickOf(id);
      double c[3] = {((double)b[0] + .5) * side, ((double)b[1] + .5) * side, ((double)b[2] + .5) * side};
      int best = 0;
      double bestD = 1e300;
      for (int k = 0; k < count; k++) {
        double d[3] = {c[0] - anchors[3 * k], c[1] - anchors[3 * k + 1], c[2] - anchors[3 * k + 2]};
        double rise = d[1] > 0 ? d[1] * .25 : d[1];
        double dist = d[0] * d[0] + d[2] * d[2] + rise * rise;
        if (dist < bestD) {
          bestD = dist;
          best = k;
        }
      }
      double acc[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int lane = 0; lane < 64; lane++) {
        int l[3] = {(lane & 3) * stride + stride / 2, ((lane >> 2) & 3) * stride + stride / 2, (lane >> 4) * stride + stride / 2};
        size_t o = (size_t)slot * 4 * N + (size_t)((l[2] * B + l[1]) * B + l[0]);
        std::array<R, 4> f = {fld[o], fld[o + N], fld[o + 2 * N], fld[o + 3 * N]};
        if (smokeDiv > 1) {  // the coarse density at the cell's centre; taps before the brick read zero
          R q[3], fr[3], v = 0;
          int c0[3];
          for (int a = 0; a < 3; a++) {
            q[a] = (R(l[a]) + R(.5)) / R(smokeDiv) - R(.5);
            c0[a] = (int)std::floor(q[a]);
            fr[a] = q[a] - R(c0[a]);
          }
          for (int k = 0; k < 8; k++) {
            int d[3] = {k & 1, (k >> 1) & 1, k >> 2}, cl[3] = {c0[0] + d[0], c0[1] + d[1], c0[2] + d[2]};
            if (cl[0] < 0 || cl[1] < 0 || cl[2] < 0) continue;
            int s = brickSlot(b[0] + (cl[0] >> sshift), b[1] + (cl[1] >> sshift), b[2] + (cl[2] >> sshift));
            if (s < 0) continue;
            int m = SB - 1;
            R w = (d[0] ? fr[0] : 1 - fr[0]) * (d[1] ? fr[1] : 1 - fr[1]) * (d[2] ? fr[2] : 1 - fr[2]);
            v += smk[(size_t)s * SN + ((cl[2] & m) * SB + (cl[1] & m)) * SB + (cl[0] & m)] * w;
          }
          f[0] = v;
        }
        std::array<R, 3> rgb = emissionOf(G, f);
        double lum = .2126 * (double)rgb[0] + .7152 * (double)rgb[1] + .0722 * (double)rgb[2];
        acc[0] += lum;
        for (int a = 0; a < 3; a++) {
          double p = ((double)(b[a] * B + l[a]) + .5) * (double)h;
          acc[1 + a] += (p - (double)anchors[3 * best + a]) * lum;
          acc[4 + a] += (double)rgb[a];
        }
      }
      for (int k = 0; k < 7; k++) sums[best * 8 + k] += acc[k];
    }
  }
  void render(const fp_camera& cam, const fp_render_settings& rs, const float* lut, float* image) {
    Render G;
    G.cam = &cam;
    G.rs = &rs;
    G.lut.assign(lut, lut + 512 * 4);
    int divShift = rs.lighting_divisor == 1 ? 0 : (rs.lighting_divisor == 2 ? 1 : 2);
    G.lightShift = shift - divShift;
    const int L = 1 << G.lightShift, L3 = L * L * L, per = B / 8, blocks = per * per * per;
    // Every slotted computing brick inside a box (boxes never overlap), with its box.
    std::vector<I3> bricks;
    std::vector<int> boxOfRow;
    if (steps > 0)
      for (uint32_t id : active) {
        I3 b = brickOf(id);
        int k = boxOf(b[0], b[1], b[2]);
        if (k < 0 || brickSlot(b[0], b[1], b[2]) < 0) continue;
        G.index[brickKey(b[0], b[1], b[2])] = (int)bricks.size();
        bricks.push_back(b);
        boxOfRow.push_back(k);
      }
    size_t nb = bricks.size();
    G.field.assign(nb * 4 * N, 0);
    if (smokeDiv > 1) G.smoke.assign(nb * SN, 0);
    G.occupancy.assign(nb * blocks, 0);
    G.light.assign(nb * 4 * L3, 0);
#pragma omp parallel for schedule(dynamic)
    for (long r = 0; r < (long)nb; r++) {
      const I3& b = bricks[r];
      useBox(boxOfRow[r]);
      int s = boxSlot(b[0], b[1], b[2]);
      for (int k = 0; k < N; k++) {
        int x = b[0] * B + (k & (B - 1)), y = b[1] * B + ((k >> shift) & (B - 1)), z = b[2] * B + (k >> (2 * shift));
        size_t o = (size_t)r * 4 * N + k;
        G.field[o] = smokeDiv > 1 ? fld[(size_t)s * 4 * N + k] : smoothedSmoke(x, y, z);
        for (int c = 1; c < 4; c++) G.field[o + c * N] = fld[((size_t)s * 4 + c) * N + k];
      }
      if (smokeDiv > 1)
        for (int k = 0; k < SN; k++) {
          int x = b[0] * SB + (k & (SB - 1)), y = b[1] * SB + ((k >> sshift) & (SB - 1)), z = b[2] * SB + (k >> (2 * sshift));
          G.smoke[(size_t)r * SN + k] = smoothedCoarse(x, y, z);
        }
    }
#pragma omp parallel for schedule(dynamic)
    for (long r = 0; r < (long)nb; r++) {
      const I3& b = bricks[r];
      useBox(boxOfRow[r]);
      for (int blk = 0; blk < blocks; blk++) {
        int o[3] = {b[0] * B + (blk % per) * 8 - 2, b[1] * B + ((blk / per) % per) * 8 - 2,
                    b[2] * B + (blk / (per * per)) * 8 - 2};
        int flags = 0;
        const bool coarse = smokeDiv > 1;
        R glowMax = 0, smokeMax = 0;
        for (int u = 0; u < 216; u++) {
          int ux = o[0] + (u % 6) * 2, uy = o[1] + ((u / 6) % 6) * 2, uz = o[2] + (u / 36) * 2;
          if (rowOf(G, ux >> shift, uy >> shift, uz >> shift) < 0) continue;
          for (int k = 0; k < 8; k++) {
            auto f = renderCell(G, ux + (k & 1), uy + ((k >> 1) & 1), uz + (k >> 2), true);
            R g = glowOf(f[2]);
            flags |= (g > R(.002) ? 1 : 0) | ((coarse ? R(0) : f[0]) + g > R(.002) ? 2 : 0);
            glowMax = std::max(glowMax, g);
          }
        }
        if (coarse) {  // every trilinear donor of coarse density in the block and halo
          R ratio = R(smokeDiv);
          int lo[3], hi[3];
          for (int a = 0; a < 3; a++) {
            lo[a] = (int)std::floor(R(o[a]) / ratio - R(.5));
            hi[a] = (int)std::floor(R(o[a] + 12) / ratio - R(.5)) + 1;
          }
          for (int z = lo[2]; z <= hi[2]; z++)
            for (int y = lo[1]; y <= hi[1]; y++)
              for (int x = lo[0]; x <= hi[0]; x++) {
                int q[3] = {x, y, z};
                for (int a = 0; a < 3; a++) q[a] = std::min(std::max(q[a], curBox()[a] * SB), (curBox()[3 + a] + 1) * SB - 1);
                smokeMax = std::max(smokeMax, cachedSmokeCell(G, q[0], q[1], q[2]));
              }
          if (smokeMax + glowMax > R(.002)) flags |= 2;
        }
        G.occupancy[(size_t)r * blocks + blk] = (uint8_t)flags;
      }
      R texel = h * R(B >> G.lightShift);
      for (int k = 0; k < L3; k++) {
        int lx = k % L, ly = (k / L) % L, lz = k / (L * L);
        auto li = incidentLight(G, (R(b[0] * L + lx) + R(.5)) * texel, (R(b[1] * L + ly) + R(.5)) * texel,
                                (R(b[2] * L + lz) + R(.5)) * texel);
        for (int c = 0; c < 4; c++) G.light[(size_t)r * 4 * L3 + c * L3 + k] = li[c];
      }
    }
    const int W = (int)cam.width, Hh = (int)cam.height;
    // A ray of viewport point (ux, uy) (fireProRay, fireProSpan) and what its march keeps.
    struct Ray {
      R ro[3], rd[3], safe[3], exitSide[3], lo, hi, stepSize, jitter, direct[3];
    };
    const R brickSize = h * R(B), lightRatio = R(B >> G.lightShift);
    const int boxCount = steps > 0 ? (int)(renderBoxes.size() / 6) : 0;
    // fireProHit: entry and exit of box k (the exit first when it misses).
    auto boxHit = [&](const Ray& r, int k, R* hit) {
      const int* bx = &renderBoxes[(size_t)6 * k];
      R lo = 0, hi = R(1e30);
      for (int a = 0; a < 3; a++) {
        R ta = (R(bx[a]) * brickSize - r.ro[a]) / r.safe[a], tb = (R(bx[3 + a] + 1) * brickSize - r.ro[a]) / r.safe[a];
        lo = std::max(lo, std::min(ta, tb));
        hi = std::min(hi, std::max(ta, tb));
      }
      hit[0] = lo;
      hit[1] = hi;
    };
    // fireProEnter: the box the ray is in at t, or enters next, becomes the current one.
    auto enterBox = [&](const Ray& r, R& t, R& exit) -> bool {
      R entry = R(1e30), out = 0;
      int best = -1;
      for (int k = 0; k < boxCount; k++) {
        R hit[2];
        boxHit(r, k, hit);
        if (hit[1] > hit[0] && hit[1] > t && hit[0] < entry) {
          entry = hit[0];
          out = hit[1];
          best = k;
        }
      }
      if (best < 0) return false;
      useBox(best);
      exit = out;
      t = std::max(t, entry);
      return true;
    };
    auto rayOf = [&](R ux, R uy, Ray& r) -> bool {
      R cx = ux * 2 - 1, cy = 1 - uy * 2;
      const float* M = cam.inverse_view_projection;
      R nh[4], fh[4];
      for (int k = 0; k < 4; k++) {
        nh[k] = R(M[k]) * cx + R(M[4 + k]) * cy + R(M[12 + k]);
        fh[k] = R(M[k]) * cx + R(M[4 + k]) * cy + R(M[8 + k]) * R(.99999f) + R(M[12 + k]);
      }
      for (int a = 0; a < 3; a++) {
        r.ro[a] = nh[a] / nh[3];
        r.rd[a] = fh[a] / fh[3] - r.ro[a];
      }
      R rl = std::sqrt(r.rd[0] * r.rd[0] + r.rd[1] * r.rd[1] + r.rd[2] * r.rd[2]);
      for (int a = 0; a < 3; a++) r.rd[a] /= rl;
      for (int a = 0; a < 3; a++) {
        r.safe[a] = std::fabs(r.rd[a]) > R(1e-6) ? r.rd[a] : R(1e-6);
        r.exitSide[a] = r.rd[a] > 0 ? 1 : 0;
      }
      // fireProSpan: first entry, last exit, length inside every box.
      r.lo = R(1e30);
      r.hi = 0;
      R length = 0;
      for (int k = 0; k < boxCount; k++) {
        R hit[2];
        boxHit(r, k, hit);
        if (hit[1] > hit[0]) {
          r.lo = std::min(r.lo, hit[0]);
          r.hi = std::max(r.hi, hit[1]);
          length += hit[1] - hit[0];
        }
      }
      if (!(r.hi > r.lo)) return false;
      r.stepSize = std::max(h * R(.5), length / R(rs.ray_steps));
      R ln = std::sqrt(R(rs.light[0]) * rs.light[0] + R(rs.light[1]) * rs.light[1] + R(rs.light[2]) * rs.light[2]);
      R g = rs.optical[3];
      R mu = (r.rd[0] * rs.light[0] + r.rd[1] * rs.light[1] + r.rd[2] * rs.light[2]) / ln;
      R phase = (1 - g * g) / std::pow(std::max(R(.05), 1 + g * g - 2 * g * mu), R(1.5));
      R dk = R(rs.light[3]) * (R(.35) + phase * R(.3));
      for (int c = 0; c < 3; c++) r.direct[c] = R(rs.scene_light[c]) * dk;
      return true;
    };
    // One step of fireProMarch at t, ds long; returns the next t.
    auto marchStep = [&](const Ray& r, R t, R ds, R exit, R& trans, R* rad) -> R {
      R tt = t + r.jitter * ds;
      R p[3] = {r.ro[0] + r.rd[0] * tt, r.ro[1] + r.rd[1] * tt, r.ro[2] + r.rd[2] * tt};
      R cell[3] = {p[0] / h, p[1] / h, p[2] / h};
      int ci[3] = {(int)std::floor(cell[0]), (int)std::floor(cell[1]), (int)std::floor(cell[2])};
      int row = rowOf(G, ci[0] >> shift, ci[1] >> shift, ci[2] >> shift);
      R size = brickSize;
      int flags = 0;
      if (row >= 0) {
        int m = B - 1;
        int block = ((((ci[2] & m) >> 3) * per) + ((ci[1] & m) >> 3)) * per + ((ci[0] & m) >> 3);
        flags = G.occupancy[(size_t)row * blocks + block];
        size = h * 8;
      }
      if (!(flags & 2)) {
        R dist = R(1e30);
        for (int a = 0; a < 3; a++) dist = std::min(dist, ((std::floor(p[a] / size) + r.exitSide[a]) * size - p[a]) / r.safe[a]);
        return std::min(t + std::max(R(1), std::floor(dist / r.stepSize) + 1) * r.stepSize, exit);
      }
      auto f = reconstruct(G, cell[0], cell[1], cell[2], (flags & 1) ? rs.filter : 0);
      if (smokeDiv > 1) f[0] = renderSmokeAt(G, cell[0] / R(smokeDiv), cell[1] / R(smokeDiv), cell[2] / R(smokeDiv));
      if (f[0] + glowOf(f[2]) > R(.002)) {
        auto glow = emissionOf(G, f);
        R density = std::max(R(0), f[0]) * R(rs.optical[0]), sc[3] = {0, 0, 0};
        if (density > 0) {
          auto inc = lightSample(G, cell[0] / lightRatio, cell[1] / lightRatio, cell[2] / lightRatio);
          for (int c = 0; c < 3; c++)
            sc[c] = R(rs.smoke[c]) * (R(rs.ambient_light[c]) + r.direct[c] * inc[3] + inc[c] * R(.65)) * density;
        }
        R ext = extinctionOf(G, f), tau = ext * ds;
        R integral = ds * (1 - R(.5) * tau + tau * tau / 6);
        if (tau >= R(.001)) integral = (1 - std::exp(-tau)) / ext;
        for (int c = 0; c < 3; c++) rad[c] += trans * (sc[c] + glow[c]) * integral;
        trans *= 1 - std::min(R(1), ext * integral);
      }
      return t + ds;
    };
    // buildSlices (volume-slices.wgsl:28-122) at half resolution.
    const int SW = std::max(1, (W + 1) / 2), SH = std::max(1, (Hh + 1) / 2), NS = 8;
    std::vector<R> slices;
    const bool half = cam.half_resolution != 0 && boxCount > 0;
    if (half) {
      slices.assign((size_t)SW * SH * NS * 4, 0);
#pragma omp parallel for schedule(dynamic)
      for (long pix = 0; pix < (long)SW * SH; pix++) {
        int px = (int)(pix % SW), py = (int)(pix / SW);
        R* out = &slices[(size_t)pix * NS * 4];
        R trans = 1, rad[3] = {0, 0, 0};
        int recorded = 0;
        Ray r;
        if (rayOf((R(px) + R(.5)) / R(SW), (R(py) + R(.5)) / R(SH), r)) {
          r.jitter = jitterOf((uint32_t)px, (uint32_t)py, cam.time);
          R spacing = std::max(r.hi - r.lo, R(0)) / R(NS), t = r.lo, depth = r.lo + spacing, exit = t;
          while (recorded < NS && t < r.hi && trans >= R(.008)) {
            if (t >= exit) {
              if (!enterBox(r, t, exit)) break;
            } else {
              R ds = std::min(r.stepSize, std::min(depth, exit) - t);
              t = marchStep(r, t, ds, exit, trans, rad);
            }
            while (recorded < NS && t >= depth) {
              R v[4] = {rad[0], rad[1], rad[2], 1 - trans};
              for (int c = 0; c < 4; c++) out[recorded * 4 + c] = v[c];
              recorded++;
              depth = r.lo + spacing * R(recorded + 1);
            }
          }
        }
        for (; recorded < NS; recorded++) {
          R v[4] = {rad[0], rad[1], rad[2], 1 - trans};
          for (int c = 0; c < 4; c++) out[recorded * 4 + c] = v[c];
        }
      }
    }
#pragma omp parallel for schedule(dynamic)
    for (long pix = 0; pix < (long)W * Hh; pix++) {
      int px = (int)(pix % W), py = (int)(pix / W);
      float* out = image + pix * 4;
      out[0] = out[1] = out[2] = out[3] = 0.f;
      if (boxCount == 0) continue;
      R ux = (R(px) + R(.5)) / R(W), uy = (R(py) + R(.5)) / R(Hh);
      Ray r;
      if (!rayOf(ux, uy, r)) continue;
      // fireProSceneDistance (volume-march.wgsl:76-89)
      R end = r.hi;
      if (cam.scene_depth && cam.scene_depth[pix] < .999999f) {
        const float* M = cam.inverse_view_projection;
        R cx = ux * 2 - 1, cy = 1 - uy * 2, d = cam.scene_depth[pix], hit[4], dist = 0;
        for (int k = 0; k < 4; k++) hit[k] = R(M[k]) * cx + R(M[4 + k]) * cy + R(M[8 + k]) * d + R(M[12 + k]);
        for (int a = 0; a < 3; a++) dist += (hit[a] / hit[3] - r.ro[a]) * r.rd[a];
        end = std::min(end, dist);
      }
      if (end <= r.lo) continue;
      r.jitter = jitterOf((uint32_t)px, (uint32_t)py, cam.time);
      R t = r.lo, trans = 1, rad[3] = {0, 0, 0};
      if (half) {  // resume from the last slice in front of the scene (scene-volume.wgsl:146-160)
        R slice = std::floor((end - r.lo) / (r.hi - r.lo) * R(NS));
        if (slice >= 1) {
          int layer = (int)std::min(slice, R(NS)) - 1;
          R gx = ux * R(SW) - R(.5), gy = uy * R(SH) - R(.5);
          R fx0 = std::floor(gx), fy0 = std::floor(gy), wx = gx - fx0, wy = gy - fy0;
          int x0 = (int)fx0, y0 = (int)fy0;
          int xs[2] = {std::min(std::max(x0, 0), SW - 1), std::min(std::max(x0 + 1, 0), SW - 1)};
          int ys[2] = {std::min(std::max(y0, 0), SH - 1), std::min(std::max(y0 + 1, 0), SH - 1)};
          R v[4] = {0, 0, 0, 0};
          for (int k = 0; k < 4; k++) {
            int ix = k & 1, iy = k >> 1;
            R w = (ix ? wx : 1 - wx) * (iy ? wy : 1 - wy);
            const R* sv4 = &slices[(((size_t)ys[iy] * SW + xs[ix]) * NS + layer) * 4];
            for (int c = 0; c < 4; c++) v[c] += sv4[c] * w;
          }
          t = r.lo + (r.hi - r.lo) * std::min(slice, R(NS)) / R(NS);
          trans = 1 - v[3];
          for (int c = 0; c < 3; c++) rad[c] = v[c];
        }
      }
      R exit = t;  // fireProMarch's cursor starts exited: the first pass enters the box at t
      while (t < end && trans >= R(.008)) {
        if (t >= exit) {
          if (!enterBox(r, t, exit)) break;
          continue;
        }
        R ds = std::min(r.stepSize, std::min(end, exit) - t);
        t = marchStep(r, t, ds, exit, trans, rad);
      }
      out[0] = (float)rad[0];
      out[1] = (float)rad[1];
      out[2] = (float)rad[2];
      out[3] = (float)(1 - trans);
    }
  }

  std::string step(const fp_frame& f, float dtf) {
    if (!std::isfinite(dtf) || dtf <= 0 || dtf > 1.0f / 30.0f)
      return "Simulation step must be in (0, 1/30]. Use fixed substeps.";
    try {
      packFlame(f.combustion, dtf);
    } catch (const std::string& e) {
      return e;
    }
    if (dir.ground != ground) {
      dir.ground = ground;
      geometryDirty = true;
    }
    uint32_t limit = slotLimit();
    if (limit > slots) growPool(limit);
    updateTiles(f);
    if (packScene(f)) {
      solidsStale = true;
      geometryDirty = true;
    }
    buildMeshTables(f);
    mayHaveFlame = mayHaveFlame || f.fuel.enabled;
    for (uint32_t i = 0; i < f.source_count; i++) mayHaveFlame = mayHaveFlame || f.sources[i].flame > 0;
    dt = (R)dtf;
    buoyancy = f.simulation.buoyancy; coolingK = f.simulation.cooling; smokeWeight = f.simulation.smoke_weight;
    damping = f.simulation.velocity_damping; dissipation = f.simulation.dissipation;
    vorticity = f.simulation.vorticity;
    timeU = (R)(float)time;
    float seedf = (float)f.simulation.seed;
    seedU = (R)seedf;
    std::memcpy(&seedBits, &seedf, 4);
    lifetimeZero = !mayHaveFlame;
    fuelEnabled = f.fuel.enabled != 0;
    ignition = f.fuel.ignition_heat;
    burnRate = f.fuel.burn_rate;
    held = (int)std::max<int64_t>(0, (int64_t)slots - (int64_t)slotLimit());
    solidsAll = solidsStale;
    for (int s = 0; s < capacity; s++) activity[(size_t)capacity * 64 + s] = 0;
    allocation();
    solidsStale = false;
    zeroFresh();
    transport();
    forcesStep();
    solvePressure();
    projectStep();
    readActivity();
    time += dtf;
    steps++;
    return "";
  }

  // ---------------------------------------------------------------- allocation
  // sourceNear (fluid-allocation.wgsl:90-108), in the kernel's f32 arithmetic: its result is
  // an integer decision that must match the device's bit for bit.
  bool sourceNear(I3 b, int tile) {
    float hf = (float)h, dtf = (float)dt;
    float size = (float)B * hf;
    float lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = (float)b[a] * size;
      hi[a] = ((float)b[a] + 1.f) * size;
    }
    for (int i : lists[0][tile]) {
      const Emitter<R>& e = emitters[i];
      if (!e.enabled) continue;
      bool inside = true;
      for (int a = 0; a < 3; a++) {
        float motion = std::fabs((float)e.vel[a]) + std::fabs((float)e.outward);
        float pad = std::min(size, 2.f * (float)vh + motion * dtf);
        float extent = std::max((float)e.size[a], 0.03f) + pad;
        float pos = (float)e.pos[a];
        if (!(pos + extent > lo[a] && pos - extent < hi[a])) inside = false;
      }
      if (inside) return true;
    }
    return false;
  }
  // buildBricks, freeBricks, allocateBricks, linkBricks, finishBricks, buildSolids
  // (fluid-allocation.wgsl:129-387), serially in brick-id order.
  void allocation() {
    size_t count = (size_t)capacity * 64;
    std::vector<uint32_t> st(count, 0);
    std::vector<uint32_t> freeRank(count, 0), reqRank(count, 0);
    uint32_t frees = 0, requests = 0;
    for (size_t index = 0; index < count; index++) {
      uint32_t s = 0;
      int tile = (int)(index >> 6);
      if (snapshotState[tile] != 0) {
        I3 b = brickOf((uint32_t)index);
        bool open = snapshotState[tile] != 2;
        bool listed = false;
        for (int z = -1; z <= 1 && open && !listed; z++)
          for (int y = -1; y <= 1 && !listed; y++)
            for (int x = -1; x <= 1 && !listed; x++) {
              int nb = brickId(b[0] + x, b[1] + y, b[2] + z);
              if (nb < 0) continue;
              int toward = neighborIndex(-x, -y, -z);
              listed = ((activity[nb] >> 3u) & (1u << toward)) != 0u || meshTable(nb) >= 0;
            }
        if (open && !listed) listed = sourceNear(b, tile);
        int32_t page = pages[index];
        bool wasListed = (state[index] & 1u) != 0;
        s = (uint32_t)listed | ((uint32_t)wasListed << 2);
        if (!listed && page >= 0) s |= BRICK_FREES;
        if (listed && page < 0) s |= BRICK_REQUESTS;
      }
      st[index] = s;
      if (s & BRICK_FREES) freeRank[index] = frees++;
      if (s & BRICK_REQUESTS) reqRank[index] = requests++;
    }
    zeroed.clear();
    // freeBricks
    for (size_t index = 0; index < count; index++) {
      if (!(st[index] & BRICK_FREES)) continue;
      int32_t page = pages[index];
      freeStack[freeCount + freeRank[index]] = (uint32_t)page;
      if (st[index] & 4u) zeroed.push_back({(uint32_t)index, (uint32_t)page});
      pages[index] = -1;
    }
    // allocateBricks
    active.clear();
    for (size_t index = 0; index < count; index++) {
      uint32_t s = st[index];
      int32_t page = pages[index];
      bool fresh = false;
      if (s & BRICK_REQUESTS) {
        int32_t top = freeCount + (int32_t)frees - (int32_t)reqRank[index];
        if (top > held) {
          page = (int32_t)freeStack[top - 1];
          pages[index] = page;
          zeroed.push_back({(uint32_t)index, (uint32_t)page | 0x80000000u});
          fresh = true;
        }
      }
      if (page >= 0) active.push_back((uint32_t)index);
      state[index] = (uint32_t)(page >= 0);
      entries[index] = page >= 0 ? (page | (fresh ? FRESH_ENTRY : 0)) : -1;
      uint32_t flags = activity[index];
      activity[index] = (flags & EXPANDS) ? MAY_EXPAND : 0u;
    }
    // The zero list holds frees, then grants, in brick order within each; its order is
    // immaterial to the step.
    // linkBricks
    for (size_t index = 0; index < count; index++) {
      if (entries[index] < 0) continue;
      I3 b = brickOf((uint32_t)index);
      int32_t* w = &records[index * RECORD_WORDS];
      for (int k = 0; k < 27; k++) {
        int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
        int nb = brickId(b[0] + dx, b[1] + dy, b[2] + dz);
        w[k] = nb >= 0 ? entries[nb] : -1;
      }
      int unknowns = 1;
      for (int k = 0; k < 8; k++) {
        int dx = -(k & 1), dy = -((k >> 1) & 1), dz = -((k >> 2) & 1);
        if (ground && b[1] + dy < 0) continue;
        if (w[neighborIndex(dx, dy, dz)] < 0) unknowns = 0;
      }
      w[27] = unknowns;
    }
    lookupGen = nextGen();
    // finishBricks
    int32_t fr = freeCount + (int32_t)frees;
    int32_t granted = std::min((int32_t)requests, std::max(fr - held, 0));
    freeCount = fr - granted;
    failures += requests - (uint32_t)granted;
    // buildSolids
    if (colliderCount > 0 || solidsAll) buildSolids();
  }
  bool insideCollider(const Collider<R>& c, int x, int y, int z) {
    if (c.kind == 2) {
      int q[3] = {x - c.lo[0], y - c.lo[1], z - c.lo[2]};
      for (int a = 0; a < 3; a++)
        if (q[a] < 0 || q[a] >= c.size[a]) return false;
      uint32_t index = (uint32_t)((q[2] * c.size[1] + q[1]) * c.size[0] + q[0]);
      return ((masks[c.first + (index >> 5)] >> (index & 31u)) & 1u) != 0;
    }
    // f32, as buildSolids computes it: the bits must match the device's exactly.
    float hf = (float)h;
    float w[3] = {((float)x + 0.5f) * hf, ((float)y + 0.5f) * hf, ((float)z + 0.5f) * hf};
    float d[3];
    for (int a = 0; a < 3; a++) {
      // transpose(axes) * (w - center): row a = column a of axes.
      float s = (float)c.axes[a][0] * (w[0] - (float)c.center[0]);
      s = s + (float)c.axes[a][1] * (w[1] - (float)c.center[1]);
      s = s + (float)c.axes[a][2] * (w[2] - (float)c.center[2]);
      d[a] = std::fabs(s / (float)c.extent[a]);
    }
    if (c.kind == 1) return d[0] < 1.f && d[1] < 1.f && d[2] < 1.f;
    float r = d[0] * d[0];
    r = r + d[1] * d[1];
    r = r + d[2] * d[2];
    return r < 1.f;
  }
  void buildSolidsBrick(uint32_t id, int slot) {
    I3 b = brickOf(id);
    int tile = (int)(id >> 6);
    for (int word = 0; word < W; word++) {
      uint32_t bits = 0;
      for (int k = 0; k < 32; k++) {
        int bit = word * 32 + k;
        int x = b[0] * B + (bit & (B - 1)), y = b[1] * B + ((bit >> shift) & (B - 1)), z = b[2] * B + (bit >> (2 * shift));
        for (int i : lists[2][tile])
          if (insideCollider(colliders[i], x, y, z)) {
            bits |= 1u << k;
            break;
          }
      }
      solids[(size_t)slot * W + word] = bits;
    }
  }
  void buildSolids() {
    if (solidsAll) {
      for (size_t id = 0; id < (size_t)capacity * 64; id++) {
        int slot = entryPage(entries[id]);
        if (slot >= 0) buildSolidsBrick((uint32_t)id, slot);
      }
    } else {
      for (auto& z : zeroed)
        if (z.second & 0x80000000u) buildSolidsBrick(z.first, (int)(z.second & 0xffffffu));
    }
  }
  // fluid-zeroing.wgsl: a fresh slot starts as still, empty air. Pools every step
  // rewrites before reading need no clearing.
  void zeroFresh() {
    for (auto& z : zeroed) {
      if (!(z.second & 0x80000000u)) continue;
      size_t s = z.second & 0xffffffu;
      std::fill(vel.begin() + s * 3 * VN, vel.begin() + (s + 1) * 3 * VN, R(0));
      std::fill(fld.begin() + s * 4 * N, fld.begin() + (s + 1) * 4 * N, R(0));
      std::fill(expn.begin() + s * N, expn.begin() + (s + 1) * N, R(0));
      if (smokeDiv > 1)  // zeroSmokeBricks (smoke.wgsl:188-223): all three smoke pools
        for (auto* pool : {&smk, &smkP, &smkN}) std::fill(pool->begin() + s * SN, pool->begin() + (s + 1) * SN, R(0));
    }
  }

  // ---------------------------------------------------------------- transport
  template <class F>
  void forActiveCells(F fn) {
    long n = (long)active.size();
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < n; i++) {
      uint32_t id = active[i];
      int slot = entryPage(entries[id]);
      I3 b = brickOf(id);
      for (int c = 0; c < N; c++) {
        int x = b[0] * B + (c & (B - 1)), y = b[1] * B + ((c >> shift) & (B - 1)), z = b[2] * B + (c >> (2 * shift));
        fn(id, slot, c, x, y, z);
      }
    }
  }
  // The same over the velocity lattice's cells.
  template <class F>
  void forActiveVCells(F fn) {
    long n = (long)active.size();
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < n; i++) {
      uint32_t id = active[i];
      int slot = entryPage(entries[id]);
      I3 b = brickOf(id);
      for (int c = 0; c < VN; c++) {
        int x = b[0] * VB + (c & (VB - 1)), y = b[1] * VB + ((c >> vshift) & (VB - 1)), z = b[2] * VB + (c >> (2 * vshift));
        fn(id, slot, c, x, y, z);
      }
    }
  }
  R sv(R x) { return store_round(x, prec.vel); }
  R ss(R x) { return store_round(x, prec.scal); }

  // advectVelocityWithBounds (fluid-velocity-transport.wgsl:28-100)
  void advectVelocity() {
    forActiveVCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      // Bounds over the 2x2x2 forward block of the velocity.
      for (int k = 0; k < 3; k++) {
        R lo = R(1e5), hi = R(-1e5);
        for (int dz = 0; dz < 2; dz++)
          for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
              R v = vcell(vel, 3, k, x + dx, y + dy, z + dz);
              lo = std::min(lo, v);
              hi = std::max(hi, v);
            }
        vmin[((size_t)slot * 3 + k) * VN + c] = store_round(lo, prec.bounds);
        vmax[((size_t)slot * 3 + k) * VN + c] = store_round(hi, prec.bounds);
      }
      V3<R> pos = vcenter(x, y, z);
      if (solidAt(pos[0], pos[1], pos[2])) {
        for (int k = 0; k < 3; k++) velP[((size_t)slot * 3 + k) * VN + c] = 0;
        return;
      }
      V3<R> orig = v3<R>(vel[((size_t)slot * 3 + 0) * VN + c], vel[((size_t)slot * 3 + 1) * VN + c],
                         vel[((size_t)slot * 3 + 2) * VN + c]);
      for (int comp = 0; comp < 3; comp++) {
        V3<R> face = pos;
        face[comp] += R(0.5) * vh;
        V3<R> fv = velocityOnFace(x, y, z, comp, orig);
        V3<R> mid, dep;
        for (int a = 0; a < 3; a++) mid[a] = face[a] - R(0.5) * dt * fv[a];
        V3<R> vm = velocityAt(mid);
        for (int a = 0; a < 3; a++) dep[a] = face[a] - dt * vm[a];
        int32_t* d = &vdonor[(((size_t)slot * 3 + comp) * VN + c) * 3];
        V3<R> shifted = dep;
        shifted[comp] -= R(0.5) * vh;
        for (int a = 0; a < 3; a++) d[a] = floori((double)(shifted[a] / vh - R(0.5)));
        velP[((size_t)slot * 3 + comp) * VN + c] = sv(velComp(vel, dep, comp));
      }
    });
  }
  // correctVelocity (fluid-velocity-transport.wgsl:104-179)
  void correctVelocity() {
    forActiveVCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      V3<R> pos = vcenter(x, y, z);
      if (solidAt(pos[0], pos[1], pos[2])) {
        for (int k = 0; k < 3; k++) velC[((size_t)slot * 3 + k) * VN + c] = 0;
        return;
      }
      V3<R> orig;
      for (int k = 0; k < 3; k++) orig[k] = vel[((size_t)slot * 3 + k) * VN + c];
      for (int comp = 0; comp < 3; comp++) {
        R predicted = velP[((size_t)slot * 3 + comp) * VN + c];
        const int32_t* d = &vdonor[(((size_t)slot * 3 + comp) * VN + c) * 3];
        int bs = brickSlot(d[0] >> vshift, d[1] >> vshift, d[2] >> vshift);
        R lo = 0, hi = 0;
        if (bs >= 0) {
          int lc = vlocal(d[0], d[1], d[2]);
          lo = vmin[((size_t)bs * 3 + comp) * VN + lc];
          hi = vmax[((size_t)bs * 3 + comp) * VN + lc];
        }
        R result;
        if (lo == hi && predicted == lo) {
          result = predicted;
        } else {
          V3<R> face = pos;
          face[comp] += R(0.5) * vh;
          V3<R> fv = velocityOnFace(x, y, z, comp, orig);
          V3<R> mid, fwd;
          for (int a = 0; a < 3; a++) mid[a] = face[a] + R(0.5) * dt * fv[a];
          V3<R> vm = velocityAt(mid);
          for (int a = 0; a < 3; a++) fwd[a] = face[a] + dt * vm[a];
          fwd[comp] -= R(0.5) * vh;
          R reversed = vsample(velP, 3, comp, fwd[0] / vh, fwd[1] / vh, fwd[2] / vh);
          R corrected = predicted + R(0.5) * (orig[comp] - reversed);
          result = (corrected < lo || corrected > hi) ? predicted : corrected;
        }
        velC[((size_t)slot * 3 + comp) * VN + c] = sv(result);
      }
    });
  }
  // fluid-advection.wgsl:53-61 traceBack / traceForward from a cell centre.
  V3<R> trace(V3<R> p, V3<R> cv, R sign) {
    V3<R> mid;
    for (int a = 0; a < 3; a++) mid[a] = p[a] + sign * R(0.5) * dt * cv[a];
    V3<R> vm = velocityAt(mid);
    V3<R> out;
    for (int a = 0; a < 3; a++) out[a] = p[a] + sign * dt * vm[a];
    return out;
  }
  // advectScalars (fluid-scalar-transport.wgsl:38-142)
  void advectScalars() {
    forActiveCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      V3<R> pos = center(x, y, z);
      V3<R> cv = velocityAt(pos);
      V3<R> dep = trace(pos, cv, R(-1));
      R out[4];
      if (!maccormack) {
        for (int k = 0; k < 4; k++) out[k] = sampleCells(fld, 4, k, dep[0] / h, dep[1] / h, dep[2] / h);
        out[2] = clampr(out[2], R(0), R(1));
      } else {
        R dc[3] = {R(x) + (dep[0] - pos[0]) / h, R(y) + (dep[1] - pos[1]) / h, R(z) + (dep[2] - pos[2]) / h};
        int base[3];
        R fr[3];
        for (int a = 0; a < 3; a++) {
          base[a] = floori((double)dc[a]);
          fr[a] = dc[a] - std::floor(dc[a]);
        }
        R mn[3] = {R(65504), R(65504), R(65504)}, mx[3] = {R(-65504), R(-65504), R(-65504)};
        R lmin = 1, lmax = 0;
        R value[4] = {0, 0, 0, 0};
        for (int dz = 0; dz < 2; dz++)
          for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
              R s[4];
              for (int k = 0; k < 4; k++) s[k] = cellAt(fld, 4, k, base[0] + dx, base[1] + dy, base[2] + dz);
              R bsx = store_round(s[0], prec.bounds == STORE_EXACT ? prec.scal : STORE_F16);
              R bsy = store_round(s[1], prec.bounds == STORE_EXACT ? prec.scal : STORE_F16);
              R bsz = store_round(s[2], prec.bounds == STORE_EXACT ? prec.scal : STORE_F16);
              R bsw = store_round(s[3], prec.bounds == STORE_EXACT ? prec.scal : STORE_F16);
              mn[0] = std::min(mn[0], bsx); mn[1] = std::min(mn[1], bsy); mn[2] = std::min(mn[2], bsw);
              mx[0] = std::max(mx[0], bsx); mx[1] = std::max(mx[1], bsy); mx[2] = std::max(mx[2], bsw);
              lmin = std::min(lmin, bsz);
              lmax = std::max(lmax, bsz);
              R w = (dx ? fr[0] : R(1) - fr[0]) * (dy ? fr[1] : R(1) - fr[1]) * (dz ? fr[2] : R(1) - fr[2]);
              for (int k = 0; k < 4; k++) value[k] += s[k] * w;
            }
        R* bnd = &sb[(size_t)slot * 8 * N];
        bnd[0 * N + c] = mn[0]; bnd[1 * N + c] = mn[1]; bnd[2 * N + c] = mn[2]; bnd[3 * N + c] = lmin;
        bnd[4 * N + c] = mx[0]; bnd[5 * N + c] = mx[1]; bnd[6 * N + c] = mx[2]; bnd[7 * N + c] = lmax;
        out[0] = value[0];
        out[1] = value[1];
        out[2] = lifetimeZero ? R(0) : value[2];
        out[3] = value[3];
      }
      // With coarse smoke the fine X channel carries no density (fluid-scalar-transport.wgsl:127, :137).
      if (smokeDiv > 1) out[0] = 0;
      for (int k = 0; k < 4; k++) fldP[((size_t)slot * 4 + k) * N + c] = ss(out[k]);
    });
  }
  R rampIntegral(int ch, R lo, R hi) {
    R area = 0;
    for (int i = 1; i < flame.counts[ch]; i++) {
      R ax = flame.knots[ch][i - 1][0], ay = flame.knots[ch][i - 1][1];
      R bx = flame.knots[ch][i][0], by = flame.knots[ch][i][1];
      R left = std::max(lo, ax), right = std::min(hi, bx);
      if (right > left) {
        R y0 = mixr(ay, by, (left - ax) / (bx - ax));
        R y1 = mixr(ay, by, (right - ax) / (bx - ax));
        area += (right - left) * (y0 + y1) * R(0.5);
      }
    }
    return area;
  }
  // evaluateFlame (flame-common.wgsl:30-42)
  void evaluateFlame(R before, R& after, R prod[3]) {
    if (before <= 0) {
      after = 0;
      prod[0] = prod[1] = prod[2] = 0;
      return;
    }
    after = std::max(R(0), before - flame.dt / flame.lifespan);
    prod[0] = flame.smoke * flame.lifespan * rampIntegral(0, after, before);
    prod[1] = flame.heat * flame.lifespan * rampIntegral(1, after, before);
    prod[2] = flame.expansion * (flame.lifespan * rampIntegral(2, after, before) / flame.dt);
  }
  R emitterWeight(const Emitter<R>& e, V3<R> p) {
    R d[3];
    for (int a = 0; a < 3; a++) d[a] = (p[a] - e.pos[a]) / std::max(e.size[a], (R)0.03f);
    R r = e.box ? std::max(std::fabs(d[0]), std::max(std::fabs(d[1]), std::fabs(d[2])))
                : std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (r >= R(1) || !e.enabled) return 0;
    return R(1) - smoothstep(R(0.5), R(1), r);
  }
  void burstVariation(const Emitter<R>& e, V3<R> p, R out[2]) {
    if (e.strength == 0) {
      out[0] = out[1] = 1;
      return;
    }
    V3<R> q;
    const R off[3] = {R(3.17), R(7.53), R(11.29)};
    for (int a = 0; a < 3; a++) q[a] = (p[a] - e.pos[a]) / e.period + off[a];
    V3<R> q2 = v3<R>(q[0] + R(17.3), q[1] + R(2.8), q[2] + R(8.6));
    out[0] = R(1) - e.strength * burst_pattern(q, seedBits);
    out[1] = R(1) - e.strength * burst_pattern(q2, seedBits);
  }
  // evolveFields (fluid-field-evolution.wgsl:9-84) with correctedScalars
  // (fluid-scalar-transport.wgsl:144-199) and recordContent (fluid-content.wgsl:29-64).
  void evolveFields() {
    long n = (long)active.size();
    std::vector<uint32_t> busyOut(n, 0), expandsOut(n, 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < n; i++) {
      uint32_t id = active[i];
      int slot = entryPage(entries[id]);
      I3 b = brickOf(id);
      int tile = (int)(id >> 6);
      uint32_t busy = 0;
      bool expands = false;
      for (int c = 0; c < N; c++) {
        int x = b[0] * B + (c & (B - 1)), y = b[1] * B + ((c >> shift) & (B - 1)), z = b[2] * B + (c >> (2 * shift));
        V3<R> pos = center(x, y, z);
        bool cvSampled = false;
        V3<R> cv;
        auto traceVel = [&]() {
          if (!cvSampled) {
            cv = velocityAt(pos);
            cvSampled = true;
          }
          return cv;
        };
        R value[4] = {0, 0, 0, 0};
        R expansion = 0;
        bool injected = false;
        if (!solidAt(pos[0], pos[1], pos[2])) {
          R tr[4];
          const R* adv = &fldP[(size_t)slot * 4 * N];
          if (!maccormack) {
            for (int k = 0; k < 4; k++) tr[k] = adv[k * N + c];
          } else {
            const R* bnd = &sb[(size_t)slot * 8 * N];
            R mn[3] = {bnd[0 * N + c], bnd[1 * N + c], bnd[2 * N + c]};
            R mx[3] = {bnd[4 * N + c], bnd[5 * N + c], bnd[6 * N + c]};
            R lmin = bnd[3 * N + c], lmax = bnd[7 * N + c];
            if (mn[0] == mx[0] && mn[1] == mx[1] && mn[2] == mx[2] && lmin == lmax) {
              tr[0] = mn[0]; tr[1] = mn[1]; tr[2] = clampr(lmin, R(0), R(1)); tr[3] = mn[2];
            } else {
              R a[4] = {adv[0 * N + c], adv[1 * N + c], adv[2 * N + c], adv[3 * N + c]};
              V3<R> fwd = trace(pos, traceVel(), R(1));
              R o[4];
              for (int k = 0; k < 4; k++) o[k] = fld[((size_t)slot * 4 + k) * N + c];
              R lifetime = a[2];
              R rev[3];
              if (lmin != lmax || a[2] != lmin) {
                R fc[3] = {R(x) + (fwd[0] - pos[0]) / h, R(y) + (fwd[1] - pos[1]) / h, R(z) + (fwd[2] - pos[2]) / h};
                int base[3];
                R fr[3];
                for (int ax = 0; ax < 3; ax++) {
                  base[ax] = floori((double)fc[ax]);
                  fr[ax] = fc[ax] - std::floor(fc[ax]);
                }
                R rs[4] = {0, 0, 0, 0};
                for (int dz = 0; dz < 2; dz++)
                  for (int dy = 0; dy < 2; dy++)
                    for (int dx = 0; dx < 2; dx++) {
                      R w = (dx ? fr[0] : R(1) - fr[0]) * (dy ? fr[1] : R(1) - fr[1]) * (dz ? fr[2] : R(1) - fr[2]);
                      for (int k = 0; k < 4; k++) rs[k] += cellAt(fldP, 4, k, base[0] + dx, base[1] + dy, base[2] + dz) * w;
                    }
                rev[0] = rs[0]; rev[1] = rs[1]; rev[2] = rs[3];
                R cl = a[2] + R(0.5) * (o[2] - rs[2]);
                lifetime = (cl < lmin || cl > lmax) ? a[2] : cl;
              } else {
                rev[0] = sampleCells(fldP, 4, 0, fwd[0] / h, fwd[1] / h, fwd[2] / h);
                rev[1] = sampleCells(fldP, 4, 1, fwd[0] / h, fwd[1] / h, fwd[2] / h);
                rev[2] = sampleCells(fldP, 4, 3, fwd[0] / h, fwd[1] / h, fwd[2] / h);
              }
              R ax3[3] = {a[0], a[1], a[3]}, ox3[3] = {o[0], o[1], o[3]}, bd[3];
              for (int k = 0; k < 3; k++) {
                R corr = ax3[k] + R(0.5) * (ox3[k] - rev[k]);
                bd[k] = (corr < mn[k] || corr > mx[k]) ? ax3[k] : corr;
              }
              tr[0] = bd[0]; tr[1] = bd[1]; tr[2] = clampr(lifetime, R(0), R(1)); tr[3] = bd[2];
            }
          }
          // With coarse smoke the fine X channel stages only this step's source production
          // (fluid-scalar-transport.wgsl:190-199).
          if (smokeDiv > 1) tr[0] = 0;
          // The corrected scalars as the half-float field held them.
          for (int k = 0; k < 4; k++) tr[k] = prec.truncate ? (R)truncate_half((double)tr[k]) : ss(tr[k]);
          R lifetime = tr[2];
          R prodS = 0, prodH = 0, injectedFuel = 0;
          for (int ei : lists[0][tile]) {
            const Emitter<R>& e = emitters[ei];
            R w = emitterWeight(e, pos);
            if (w == 0) continue;
            R var[2];
            burstVariation(e, pos, var);
            lifetime = std::max(lifetime, e.flame * w * var[1]);
            prodS += e.smoke * w * dt;
            prodH += e.heat * var[0] * w * dt;
            injectedFuel += e.fuel * w * dt;
          }
          {  // mesh emission at this cell (fluid-field-evolution.wgsl:33-36)
            const fp_mesh_source& ms = meshSourceAt(x, y, z);
            lifetime = std::max(lifetime, (R)ms.scalar[0]);
            prodS += (R)ms.scalar[2] * dt;
            prodH += (R)ms.scalar[1] * dt;
            injectedFuel += (R)ms.scalar[3] * dt;
          }
          R remaining = 0, burned = 0;
          if (fuelEnabled) {
            remaining = tr[3] + injectedFuel;
            if (tr[1] + prodH >= ignition) {
              lifetime = std::max(lifetime, std::min(remaining, R(1)));
              R unburned = remaining * std::exp(-burnRate * dt);
              burned = remaining - unburned;
              remaining = unburned;
            }
          }
          R after, fp[3];
          evaluateFlame(clampr(lifetime, R(0), R(1)), after, fp);
          expansion = fp[2] + flame.expansion * burned / dt;
          R dS = tr[0] * std::exp(-dissipation * dt) + (prodS + fp[0]) * std::exp(-dissipation * dt * R(0.5));
          R dH = tr[1] * std::exp(-coolingK * dt) + (prodH + fp[1]) * std::exp(-coolingK * dt * R(0.5));
          value[0] = std::max(dS, R(0));
          value[1] = std::max(dH, R(0));
          value[2] = after;
          value[3] = remaining;
          injected = prodS > 0 || prodH > 0 || lifetime > tr[2] || injectedFuel > 0;
        }
        // clearDormant (fluid-common.wgsl:8-13)
        if (!injected && value[2] == 0 && value[0] < R(0.001) && value[1] < R(0.001) && value[3] < R(0.001))
          value[0] = value[1] = value[2] = value[3] = 0;
        for (int k = 0; k < 4; k++) fldN[((size_t)slot * 4 + k) * N + c] = ss(value[k]);
        expn[(size_t)slot * N + c] = store_round(expansion, prec.expn);
        if (expansion != 0) expands = true;
        // holdsContent (fluid-content.wgsl:22-24) tests the value before its store rounds; the
        // fine X channel counts only without coarse smoke.
        if (std::max(std::max(smokeDiv > 1 ? R(0) : value[0], value[2]), value[3]) > (R)cutoff) {
          V3<R> v = traceVel();
          busy |= contentSupport(x, y, z, v);
        }
      }
      busyOut[i] = busy;
      expandsOut[i] = expands;
    }
    for (long i = 0; i < n; i++) {
      uint32_t id = active[i];
      uint32_t flags = 0;
      if (busyOut[i]) {
        flags = CONTENT | (busyOut[i] << 3);
        uint32_t l = id & 63u;
        uint32_t bits = (1u << (l & 3u)) | (16u << ((l >> 2) & 3u)) | (256u << (l >> 4));
        activity[(size_t)capacity * 64 + (id >> 6)] |= bits;
      }
      if (expandsOut[i]) flags |= EXPANDS;
      activity[id] |= flags;
    }
  }
  // contentSupport (fluid-content.wgsl:29-39)
  uint32_t contentSupport(int x, int y, int z, V3<R> v) {
    int id[3] = {x, y, z};
    bool low[3], high[3];
    for (int a = 0; a < 3; a++) {
      R side = R(B);
      R loc = R(id[a] & (B - 1)) + R(0.5);
      R pad = std::min(side, std::max(R(2), R(2) * R(vd)) + std::fabs(v[a]) * dt / h);
      low[a] = loc < pad;
      high[a] = loc + pad >= side;
    }
    uint32_t row = 2u | (low[0] ? 1u : 0u) | (high[0] ? 4u : 0u);
    uint32_t plane = (row << 3u) | (low[1] ? row : 0u) | (high[1] ? (row << 6u) : 0u);
    return (plane << 9u) | (low[2] ? plane : 0u) | (high[2] ? (plane << 18u) : 0u);
  }
  // ---------------------------------------------------------------- coarse smoke
  // Cell `c` of the coarse grid in brick id `b`; its centre in world units.
  I3 coarseCellOf(I3 b, int c) const {
    return I3{b[0] * SB + (c & (SB - 1)), b[1] * SB + ((c >> sshift) & (SB - 1)), b[2] * SB + (c >> (2 * sshift))};
  }
  V3<R> coarseCenter(I3 q) const {
    return v3<R>((R(q[0]) + R(0.5)) * sp, (R(q[1]) + R(0.5)) * sp, (R(q[2]) + R(0.5)) * sp);
  }
  // advectSmoke (smoke.wgsl:101-124): the RK2 back trace of each coarse cell's centre through
  // the start-of-step velocity, the predictor sampled there and (MacCormack) the donors' range,
  // smokeDonorBounds (:63-77): min from 1e30 and max from 0 over the 2x2x2 block.
  void advectSmoke() {
    long n = (long)active.size();
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < n; i++) {
      uint32_t id = active[i];
      size_t slot = (size_t)entryPage(entries[id]);
      I3 b = brickOf(id);
      for (int c = 0; c < SN; c++) {
        I3 q = coarseCellOf(b, c);
        V3<R> pos = coarseCenter(q);
        R density = 0;
        if (!solidAt(pos[0], pos[1], pos[2])) {
          V3<R> dep = trace(pos, velocityAt(pos), R(-1));
          density = coarseSample(smk, dep[0] / sp, dep[1] / sp, dep[2] / sp);
          if (maccormack) {
            int base[3];
            for (int a = 0; a < 3; a++) base[a] = floori((double)(dep[a] / sp - R(0.5)));
            R lo = R(1e30), hi = 0;
            for (int k = 0; k < 8; k++) {
              R v = coarseCell(smk, base[0] + (k & 1), base[1] + ((k >> 1) & 1), base[2] + (k >> 2));
              lo = std::min(lo, v);
              hi = std::max(hi, v);
            }
            smkBnd[(slot * 2 + 0) * SN + c] = store_round(lo, prec.scal);
            smkBnd[(slot * 2 + 1) * SN + c] = store_round(hi, prec.scal);
          }
        }
        smkP[slot * SN + c] = ss(density);
      }
    }
  }
  // contentSupport (fluid-content.wgsl:29-39) on the smoke grid: SB cells a side, the pad in
  // smoke cells (two at least).
  uint32_t smokeSupport(I3 q, V3<R> v) {
    bool low[3], high[3];
    for (int a = 0; a < 3; a++) {
      R side = R(SB);
      R loc = R(q[a] & (SB - 1)) + R(0.5);
      R pad = std::min(side, std::max(R(2), R(2) * (vh / sp)) + std::fabs(v[a]) * dt / sp);
      low[a] = loc < pad;
      high[a] = loc + pad >= side;
    }
    uint32_t row = 2u | (low[0] ? 1u : 0u) | (high[0] ? 4u : 0u);
    uint32_t plane = (row << 3u) | (low[1] ? row : 0u) | (high[1] ? (row << 6u) : 0u);
    return (plane << 9u) | (low[2] ? plane : 0u) | (high[2] ? (plane << 18u) : 0u);
  }
  // evolveSmoke (smoke.wgsl:126-178): bounded MacCormack correction of the predictor, decay,
  // the volume average of the fine cells' source production (smokeProduction :23-38, the mean
  // of each 2x2x2 block of evolved fine fields), dormant clearing, content flags per brick.
  void evolveSmoke() {
    long n = (long)active.size();
    std::vector<uint32_t> busyOut(n, 0);
    const int blocks = smokeDiv / 2;
    const R volume = R(smokeDiv * smokeDiv * smokeDiv / 8);
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < n; i++) {
      uint32_t id = active[i];
      size_t slot = (size_t)entryPage(entries[id]);
      I3 b = brickOf(id);
      uint32_t busy = 0;
      for (int c = 0; c < SN; c++) {
        I3 q = coarseCellOf(b, c);
        V3<R> pos = coarseCenter(q);
        R density = 0;
        if (!solidAt(pos[0], pos[1], pos[2])) {
          V3<R> cv = velocityAt(pos);
          R predictor = smkP[slot * SN + c];
          R bounded = predictor;
          if (maccormack) {
            R lo = smkBnd[(slot * 2 + 0) * SN + c], hi = smkBnd[(slot * 2 + 1) * SN + c];
            if (lo != hi || predictor != lo) {
              R original = smk[slot * SN + c];
              V3<R> fwd = trace(pos, cv, R(1));
              R reversed = coarseSample(smkP, fwd[0] / sp, fwd[1] / sp, fwd[2] / sp);
              R corrected = predictor + R(0.5) * (original - reversed);
              bounded = (corrected < lo || corrected > hi) ? predictor : corrected;
            }
          }
          R transported = prec.truncate ? (R)truncate_half((double)bounded) : bounded;
          R produced[4] = {0, 0, 0, 0};
          for (int bz = 0; bz < blocks; bz++)
            for (int by = 0; by < blocks; by++)
              for (int bx = 0; bx < blocks; bx++) {
                // The shared corner of a 2x2x2 block of fine cells: a trilinear sample there
                // is the block's mean.
                R fx = R(q[0] * smokeDiv + 2 * bx + 1), fy = R(q[1] * smokeDiv + 2 * by + 1),
                  fz = R(q[2] * smokeDiv + 2 * bz + 1);
                for (int k = 0; k < 4; k++) produced[k] += sampleCells(fld, 4, k, fx, fy, fz);
              }
          for (int k = 0; k < 4; k++) produced[k] /= volume;
          density = std::max(R(0), transported * std::exp(-dissipation * dt) + produced[0]);
          if (produced[0] == 0 && produced[2] == 0 && std::max(density, std::max(produced[1], produced[3])) < R(0.001))
            density = 0;
          if (density > (R)cutoff) busy |= smokeSupport(q, cv);
        }
        smkN[slot * SN + c] = ss(density);
      }
      busyOut[i] = busy;
    }
    // recordContent (fluid-content.wgsl:43-64)
    for (long i = 0; i < n; i++) {
      if (!busyOut[i]) continue;
      uint32_t id = active[i];
      uint32_t l = id & 63u;
      uint32_t bits = (1u << (l & 3u)) | (16u << ((l >> 2) & 3u)) | (256u << (l >> 4));
      activity[(size_t)capacity * 64 + (id >> 6)] |= bits;
      activity[id] |= CONTENT | (busyOut[i] << 3);
    }
  }
  void transport() {
    advectVelocity();
    correctVelocity();
    advectScalars();
    evolveFields();
    fld.swap(fldN);
    if (smokeDiv > 1) {
      advectSmoke();
      evolveSmoke();
      smk.swap(smkN);
    }
  }

  // ---------------------------------------------------------------- forces
  void buildNoise() {
    noiseTable.resize(64 * 64 * 64);
    for (int z = 0; z < 64; z++)
      for (int y = 0; y < 64; y++)
        for (int x = 0; x < 64; x++) {
          V3<float> p = v3<float>((x + 0.5f) / 64.0f * 16.0f, (y + 0.5f) / 64.0f * 16.0f, (z + 0.5f) / 64.0f * 16.0f);
          V3<float> dx = noise_gradient(p);
          V3<float> dy = noise_gradient(v3<float>(p[0] + 7.1f, p[1] + 3.7f, p[2] + 11.3f));
          V3<float> dz = noise_gradient(v3<float>(p[0] + 5.2f, p[1] + 7.9f, p[2] + 9.5f));
          V3<float> c = v3<float>(dz[1] - dy[2], dx[2] - dz[0], dy[0] - dx[1]);
          for (int a = 0; a < 3; a++) c[a] = (float)round_f16(c[a]);  // rgba16float texture
          noiseTable[(z * 64 + y) * 64 + x] = c;
        }
  }
  // curlNoise (fluid-forces.wgsl:3-9): a repeat-addressed trilinear fetch of the table.
  V3<R> curlNoise(V3<R> p) {
    static const R rot[3][3] = {{R(.36), R(-.8), R(.48)}, {R(.48), R(.6), R(.64)}, {R(-.8), R(0), R(.6)}};  // columns
    R uvw[3];
    for (int a = 0; a < 3; a++) uvw[a] = (rot[0][a] * p[0] + rot[1][a] * p[1] + rot[2][a] * p[2]) / R(16);
    int i0[3];
    R f[3];
    for (int a = 0; a < 3; a++) {
      R t = uvw[a] * R(64) - R(0.5);
      i0[a] = floori((double)t);
      f[a] = t - std::floor(t);
    }
    R s[3] = {0, 0, 0};
    for (int dz = 0; dz < 2; dz++)
      for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) {
          int xi = (i0[0] + dx) & 63, yi = (i0[1] + dy) & 63, zi = (i0[2] + dz) & 63;
          R w = (dx ? f[0] : R(1) - f[0]) * (dy ? f[1] : R(1) - f[1]) * (dz ? f[2] : R(1) - f[2]);
          const V3<float>& v = noiseTable[(zi * 64 + yi) * 64 + xi];
          for (int a = 0; a < 3; a++) s[a] += (R)v[a] * w;
        }
    V3<R> out;
    for (int a = 0; a < 3; a++) out[a] = rot[a][0] * s[0] + rot[a][1] * s[1] + rot[a][2] * s[2];
    return out;
  }
  // meshCovers (force-fields.wgsl:27-47): a mesh target of force `index` covers velocity cell
  // (x,y,z) while the cell's brick has an id.
  bool meshCovers(int index, int x, int y, int z) {
    if (brickId(x >> vshift, y >> vshift, z >> vshift) < 0) return false;
    return coverage.count({index, x, y, z}) != 0;
  }
  // externalForces + coverage (force-fields.wgsl:49-103) at velocity cell (x,y,z), centre p.
  V3<R> externalForces(int tile, int x, int y, int z, V3<R> p) {
    V3<R> result = v3<R>(0, 0, 0);
    for (int index : lists[1][tile]) {
      const Force<R>& f = forces[index];
      R weight = 1;
      if (f.targeted && !(f.hasMesh && meshCovers(index, x, y, z))) {
        R covered = 0;
        for (int r = 0; r < f.regionCount; r++) {
          const Region<R>& g = regions[f.regionFirst + r];
          R d[3];
          for (int a = 0; a < 3; a++) d[a] = std::fabs((p[a] - g.center[a]) / std::max(g.size[a], (R)0.03f));
          R dist = g.box ? std::max(d[0], std::max(d[1], d[2])) : std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
          covered = std::max(covered, R(1) - smoothstep(R(0.5), R(1), dist));
        }
        weight = covered;
      }
      if (weight == 0) continue;
      V3<R> acc = v3<R>(f.axis[0] * f.strength, f.axis[1] * f.strength, f.axis[2] * f.strength);
      if (f.kind == 1) {
        V3<R> q;
        R off[3] = {seedU, -timeU * R(0.7), seedU * R(0.25)};
        for (int a = 0; a < 3; a++) q[a] = p[a] * f.scale * R(0.65) + off[a];
        V3<R> q2 = v3<R>(q[0] * R(2.03) + R(13.7), q[1] * R(2.03) + R(5.3), q[2] * R(2.03) + R(19.1));
        V3<R> n1 = curlNoise(q), n2 = curlNoise(q2);
        for (int a = 0; a < 3; a++) acc[a] = (n1[a] + R(0.45) * n2[a]) * f.strength;
      } else if (f.kind >= 2) {
        R delta[3], radial[3];
        for (int a = 0; a < 3; a++) radial[a] = delta[a] = p[a] - f.center[a];
        if (f.kind == 2) {
          R dd = delta[0] * f.axis[0] + delta[1] * f.axis[1] + delta[2] * f.axis[2];
          for (int a = 0; a < 3; a++) radial[a] -= f.axis[a] * dd;
        }
        R rr = radial[0] * radial[0] + radial[1] * radial[1] + radial[2] * radial[2];
        R distance = std::sqrt(rr);
        R radius = std::max(f.scale, R(0.01));
        R dir[3];
        for (int a = 0; a < 3; a++) dir[a] = radial[a] / std::max(distance, radius * R(0.25));
        R falloff = R(1) / (R(1) + rr / (radius * radius));
        if (f.kind == 2) {
          R cr[3] = {f.axis[1] * dir[2] - f.axis[2] * dir[1], f.axis[2] * dir[0] - f.axis[0] * dir[2],
                     f.axis[0] * dir[1] - f.axis[1] * dir[0]};
          for (int a = 0; a < 3; a++)
            acc[a] = (cr[a] * f.strength - dir[a] * f.inward + f.axis[a] * f.lift) * falloff;
        } else {
          for (int a = 0; a < 3; a++) acc[a] = dir[a] * f.strength * falloff;
        }
      }
      for (int a = 0; a < 3; a++) result[a] += acc[a] * weight;
    }
    return result;
  }
  // computeCurl (fluid-forces.wgsl:38-75) over the corrected velocity.
  void computeCurl() {
    forActiveVCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      auto cc = [&](int px, int py, int pz, int comp) {
        int q[3] = {px, py, pz};
        q[comp] -= 1;
        return R(0.5) * (vcell(velC, 3, comp, px, py, pz) + vcell(velC, 3, comp, q[0], q[1], q[2]));
      };
      R hh = R(0.5) / vh;
      R dx0 = (cc(x + 1, y, z, 1) - cc(x - 1, y, z, 1)) * hh, dx1 = (cc(x + 1, y, z, 2) - cc(x - 1, y, z, 2)) * hh;
      R dy0 = (cc(x, y + 1, z, 0) - cc(x, y - 1, z, 0)) * hh, dy1 = (cc(x, y + 1, z, 2) - cc(x, y - 1, z, 2)) * hh;
      R dz0 = (cc(x, y, z + 1, 0) - cc(x, y, z - 1, 0)) * hh, dz1 = (cc(x, y, z + 1, 1) - cc(x, y, z - 1, 1)) * hh;
      R cv[3] = {dy1 - dz1, dz0 - dx1, dx0 - dy0};
      R mag = std::sqrt(cv[0] * cv[0] + cv[1] * cv[1] + cv[2] * cv[2]);
      for (int k = 0; k < 3; k++) curl[((size_t)slot * 4 + k) * VN + c] = store_round(cv[k], prec.curl);
      curl[((size_t)slot * 4 + 3) * VN + c] = store_round(mag, prec.curl);
    });
  }
  // centerForce (fluid-forces.wgsl:79-104), cellForce (:113-118)
  V3<R> cellForce(int tile, int x, int y, int z) {
    if (brickSlot(x >> vshift, y >> vshift, z >> vshift) < 0) return v3<R>(0, 0, 0);
    V3<R> w = vcenter(x, y, z);
    V3<R> F = v3<R>(0, 0, 0);
    if (!solidAt(w[0], w[1], w[2])) {
      R heat = fieldAverage(fld, 4, 1, x, y, z), density = fieldAverage(fld, 4, 0, x, y, z);
      // smokeVelocityAverage (smoke.wgsl:4-21): at one velocity cell per smoke spacing or less
      // the coarse density sampled at the cell centre, else the mean of its 2x2x2 blocks.
      if (smokeDiv > 1) {
        int ratio = std::max(1, vd / smokeDiv);
        if (ratio == 1) {
          density = coarseSample(smk, w[0] / sp, w[1] / sp, w[2] / sp);
        } else {
          density = 0;
          for (int k = 0; k < ratio; k += 2)
            for (int j = 0; j < ratio; j += 2)
              for (int i = 0; i < ratio; i += 2)
                density += coarseSample(smk, R(x * ratio + i + 1), R(y * ratio + j + 1), R(z * ratio + k + 1));
          density /= R(ratio * ratio * ratio / 8);
        }
      }
      V3<R> conf = v3<R>(0, 0, 0);
      if (vorticity != 0) {
        R c[3] = {vcell(curl, 4, 0, x, y, z), vcell(curl, 4, 1, x, y, z), vcell(curl, 4, 2, x, y, z)};
        R eta[3] = {vcell(curl, 4, 3, x + 1, y, z) - vcell(curl, 4, 3, x - 1, y, z),
                    vcell(curl, 4, 3, x, y + 1, z) - vcell(curl, 4, 3, x, y - 1, z),
                    vcell(curl, 4, 3, x, y, z + 1) - vcell(curl, 4, 3, x, y, z - 1)};
        R len = std::sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]) + R(0.0001);
        R n[3] = {eta[0] / len, eta[1] / len, eta[2] / len};
        R s = vorticity * vh;
        conf = v3<R>((n[1] * c[2] - n[2] * c[1]) * s, (n[2] * c[0] - n[0] * c[2]) * s, (n[0] * c[1] - n[1] * c[0]) * s);
      }
      V3<R> ext = externalForces(tile, x, y, z, w);
      for (int a = 0; a < 3; a++) F[a] = conf[a] + ext[a];
      F[1] += buoyancy * heat - smokeWeight * density;
    }
    for (int a = 0; a < 3; a++) F[a] = prec.truncate ? (R)truncate_half((double)F[a]) : sv(F[a]);
    return F;
  }
  // sourceVelocity (fluid-forces.wgsl:122-149)
  R sourceVelocity(int tile, R value, V3<R> face, int comp) {
    R result = value;
    for (int ei : lists[0][tile]) {
      const Emitter<R>& e = emitters[ei];
      if (e.response == 0) continue;
      R w = emitterWeight(e, face);
      if (w == 0) continue;
      R radial[3] = {0, 0, 0};
      if (e.outward != 0) {
        R d[3] = {face[0] - e.pos[0], face[1] - e.pos[1], face[2] - e.pos[2]};
        R len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int a = 0; a < 3; a++) radial[a] = d[a] / std::max(len, R(1e-6)) * e.outward;
      }
      result = mixr(result, e.vel[comp] + radial[comp], R(1) - std::exp(-e.response * w * dt));
    }
    // Mesh emission's velocity coupling (fluid-forces.wgsl:143-147) at the face's field cell.
    I3 fc = {floori((double)(face[0] / h + R(0.25))), floori((double)(face[1] / h + R(0.25))),
             floori((double)(face[2] / h + R(0.25)))};
    const fp_mesh_source& ms = meshSourceAt(fc[0], fc[1], fc[2]);
    if (ms.motion[3] > 0)
      result = mixr(result, (R)ms.motion[comp] / (R)ms.motion[3], R(1) - std::exp(-(R)ms.motion[3] * dt));
    return result;
  }
  // applyForces (fluid-forces.wgsl:151-182), then computeDivergence (:184-203).
  void forcesStep() {
    if (vorticity != 0) computeCurl();
    forActiveVCells([&](uint32_t id, int slot, int c, int x, int y, int z) {
      int tile = (int)(id >> 6);
      V3<R> F0 = cellForce(tile, x, y, z);
      V3<R> Fx = cellForce(tile, x + 1, y, z), Fy = cellForce(tile, x, y + 1, z), Fz = cellForce(tile, x, y, z + 1);
      R force[3] = {R(0.5) * (F0[0] + Fx[0]), R(0.5) * (F0[1] + Fy[1]), R(0.5) * (F0[2] + Fz[2])};
      V3<R> pos = vcenter(x, y, z);
      R decay = std::exp(-damping * dt);
      R v[3];
      for (int a = 0; a < 3; a++) v[a] = velC[((size_t)slot * 3 + a) * VN + c] * decay + dt * force[a];
      R out[3];
      for (int a = 0; a < 3; a++) {
        V3<R> face = pos;
        face[a] += R(0.5) * vh;
        out[a] = sourceVelocity(tile, v[a], face, a);
      }
      // enforceFaces (fluid-forces.wgsl:15-31)
      if (solidAt(pos[0], pos[1], pos[2])) {
        out[0] = out[1] = out[2] = 0;
      } else {
        if (solidAt(pos[0] + vh, pos[1], pos[2])) out[0] = 0;
        if (solidAt(pos[0], pos[1] + vh, pos[2])) out[1] = 0;
        if (solidAt(pos[0], pos[1], pos[2] + vh)) out[2] = 0;
      }
      for (int a = 0; a < 3; a++) velF[((size_t)slot * 3 + a) * VN + c] = sv(out[a]);
    });
    forActiveVCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      R d = (velF[((size_t)slot * 3 + 0) * VN + c] - vcell(velF, 3, 0, x - 1, y, z)) / vh +
            (velF[((size_t)slot * 3 + 1) * VN + c] - vcell(velF, 3, 1, x, y - 1, z)) / vh +
            (velF[((size_t)slot * 3 + 2) * VN + c] - vcell(velF, 3, 2, x, y, z - 1)) / vh;
      div[(size_t)slot * VN + c] = store_round(vh * vh * (d - fieldAverage(expn, 1, 0, x, y, z)), prec.p0);
    });
  }

  // ---------------------------------------------------------------- multigrid (pressure.wgsl)
  int storeMode(int level) { return level == 0 ? prec.p0 : prec.pc; }
  // cellAddress (pressure.wgsl:72-92): -1 without storage.
  long cellAddress(int px, int py, int pz, int level) {
    int s = levelShift(level), side = 1 << s;
    int lx = px & (side - 1), ly = py & (side - 1), lz = pz & (side - 1);
    long owner;
    if (level < brickLevels) {
      int slot = brickSlot(px >> s, py >> s, pz >> s);
      if (slot < 0) return -1;
      owner = slot;
    } else {
      int t = tileAt(px >> s, py >> s, pz >> s);
      if (t < 0) return -1;
      owner = t;
    }
    return owner * side * side * side + (lz * side + ly) * side + lx;
  }
  bool brickActive(int bx, int by, int bz) { return brickEntry(bx, by, bz) >= 0; }
  // activeCell (pressure.wgsl:100-136)
  bool activeCell(int px, int py, int pz, int level) {
    if (level >= brickLevels) {
      int n = 1 << (level - brickLevels);
      for (int z = 0; z < n; z++)
        for (int y = 0; y < n; y++)
          for (int x = 0; x < n; x++) {
            int id = brickId(px * n + x, py * n + y, pz * n + z);
            if (id < 0 || entries[id] < 0 || records[(size_t)id * RECORD_WORDS + 27] == 0) return false;
          }
      return true;
    }
    int span = 1 << level;
    int p[3] = {px, py, pz};
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = (p[a] * span - 1) >> brickLevels;
      hi[a] = (p[a] * span + span - 1) >> brickLevels;
    }
    if (ground) lo[1] = std::max(lo[1], 0);
    for (int z = lo[2]; z <= hi[2]; z++)
      for (int y = lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++)
          if (!brickActive(x, y, z)) return false;
    return true;
  }
  bool blockedAt(int px, int py, int pz, int level) {
    R s = vh * R(1 << level);
    return solidAt((R(px) + R(0.5)) * s, (R(py) + R(0.5)) * s, (R(pz) + R(0.5)) * s);
  }
  uint8_t cellTopology(int px, int py, int pz, int level) {
    if (blockedAt(px, py, pz, level)) return STORED_SOLID;
    static const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    uint8_t flags = 0;
    for (int s = 0; s < 6; s++)
      if (!blockedAt(px + off[s][0], py + off[s][1], pz + off[s][2], level)) flags |= (uint8_t)(1u << s);
    return flags;
  }
  std::vector<uint8_t>& topo(int level) { return levels[level].topo; }
  void buildBrickTopology(uint32_t id, int slot, int level) {
    I3 b = brickOf(id);
    int side = levelSide(level), cells = side * side * side;
    for (int o = 0; o < cells; o++) {
      int lx = o % side, ly = (o / side) % side, lz = o / (side * side);
      topo(level)[(size_t)slot * cells + o] = cellTopology(b[0] * side + lx, b[1] * side + ly, b[2] * side + lz, level);
    }
  }
  void buildTopology() {
    if (geometryDirty || topologyEachStep) {
      for (size_t id = 0; id < (size_t)capacity * 64; id++) {
        if (snapshotState[id >> 6] == 0) continue;
        int slot = entryPage(entries[id]);
        if (slot < 0) continue;
        for (int l = 0; l < brickLevels; l++) buildBrickTopology((uint32_t)id, slot, l);
      }
      for (int l = brickLevels; l <= bottom; l++) {
        int side = levelSide(l), cells = side * side * side;
        for (int t = 0; t < capacity; t++) {
          if (snapshotState[t] == 0) continue;
          for (int o = 0; o < cells; o++) {
            int lx = o % side, ly = (o / side) % side, lz = o / (side * side);
            topo(l)[(size_t)t * cells + o] =
                cellTopology(snapshot[t][0] * side + lx, snapshot[t][1] * side + ly, snapshot[t][2] * side + lz, l);
          }
        }
      }
      geometryDirty = false;
    }
  }
  // Fresh slots need their topology every step (PressureSolver.ts:293-302).
  void buildZeroedTopology() {
    for (auto& z : zeroed) {
      int slot = entryPage(entries[z.first]);
      if (slot < 0) continue;
      for (int l = 0; l < brickLevels; l++) buildBrickTopology(z.first, slot, l);
    }
  }
  uint32_t flagsOf(int level, long addr) {
    uint8_t s = topo(level)[addr];
    if (s & STORED_SOLID) return SOLID;
    return s & 63u;
  }
  static R axisDiag(uint32_t flags) {
    return R((flags >> 0) & 1) + R((flags >> 1) & 1) + R((flags >> 2) & 1) + R((flags >> 3) & 1) +
           R((flags >> 4) & 1) + R((flags >> 5) & 1);
  }
  std::vector<R>* inP;
  std::vector<R>* outP;
  std::vector<R>* inRhs;
  R readAt(const std::vector<R>& arr, int px, int py, int pz, int level) {
    long a = cellAddress(px, py, pz, level);
    return a < 0 ? R(0) : arr[a];
  }
  // stencil (pressure.wgsl:360-402): sum of open neighbours and the diagonal; axis weights are
  // 1 on the cubic lattice.
  void stencil(int px, int py, int pz, uint32_t flags, int level, const std::vector<R>& p, R& sum, R& diag) {
    static const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    R v[6];
    for (int s = 0; s < 6; s++)
      v[s] = (flags & (1u << s)) ? readAt(p, px + off[s][0], py + off[s][1], pz + off[s][2], level) : R(0);
    sum = (v[0] + v[1]) + (v[2] + v[3]) + (v[4] + v[5]);
    diag = R((flags >> 0) & 1) + R((flags >> 1) & 1) + (R((flags >> 2) & 1) + R((flags >> 3) & 1)) +
           (R((flags >> 4) & 1) + R((flags >> 5) & 1));
  }
  // Cells a level's dispatch covers: every cell of every listed brick (brick levels), or of
  // every tile (tile levels).
  template <class F>
  void forLevelCells(int level, F fn) {
    int side = levelSide(level), cells = side * side * side;
    if (level < brickLevels) {
      long n = (long)active.size();
#pragma omp parallel for schedule(dynamic, 8)
      for (long i = 0; i < n; i++) {
        I3 b = brickOf(active[i]);
        for (int o = 0; o < cells; o++)
          fn(b[0] * side + o % side, b[1] * side + (o / side) % side, b[2] * side + o / (side * side));
      }
    } else {
#pragma omp parallel for schedule(dynamic, 8)
      for (int t = 0; t < capacity; t++) {
        if (snapshotState[t] == 0) continue;
        for (int o = 0; o < cells; o++)
          fn(snapshot[t][0] * side + o % side, snapshot[t][1] * side + (o / side) % side,
             snapshot[t][2] * side + o / (side * side));
      }
    }
  }
  // relaxCell (pressure.wgsl:468-479); `first` is initializePressure (:485-505).
  void relax(int level, const std::vector<R>& rhs, const std::vector<R>& pin, std::vector<R>& pout, bool first) {
    forLevelCells(level, [&](int px, int py, int pz) {
      long a = cellAddress(px, py, pz, level);
      uint32_t flags = flagsOf(level, a);
      if ((flags & SOLID) || !activeCell(px, py, pz, level)) {
        pout[a] = 0;
        return;
      }
      R sum, diag;
      if (first) {
        diag = R((flags >> 0) & 1) + R((flags >> 1) & 1) + (R((flags >> 2) & 1) + R((flags >> 3) & 1)) +
               (R((flags >> 4) & 1) + R((flags >> 5) & 1));
        pout[a] = store_round(mixr(R(0), (R(0) - rhs[a]) / std::max(diag, R(1e-12)), R(0.8)), storeMode(level));
        return;
      }
      stencil(px, py, pz, flags, level, pin, sum, diag);
      R cand = (sum - rhs[a]) / std::max(diag, R(1e-12));
      pout[a] = store_round(mixr(pin[a], cand, R(0.8)), storeMode(level));
    });
  }
  // restrictCell (pressure.wgsl:601-647): coarse right-hand side and its first iterate.
  void restrictLevel(int fine, const std::vector<R>& rhs, const std::vector<R>& p, std::vector<R>& crhs,
                     std::vector<R>& cfirst) {
    int level = fine + 1;
    forLevelCells(level, [&](int cx, int cy, int cz) {
      R residual = 0;
      bool every = true;
      for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
          for (int x = 0; x < 2; x++) {
            int px = cx * 2 + x, py = cy * 2 + y, pz = cz * 2 + z;
            bool unknown = activeCell(px, py, pz, fine);
            every = every && unknown;
            if (unknown) {
              long a = cellAddress(px, py, pz, fine);
              uint32_t flags = flagsOf(fine, a);
              if (!(flags & SOLID)) {
                R sum, diag;
                stencil(px, py, pz, flags, fine, p, sum, diag);
                residual += rhs[a] - (sum - diag * p[a]);
              }
            }
          }
      R r = residual * R(0.5);
      long out = cellAddress(cx, cy, cz, level);
      R stored = store_round(r, storeMode(level));
      crhs[out] = stored;
      R first = 0;
      if (every) {
        uint32_t flags = flagsOf(level, out);
        if (!(flags & SOLID)) {
          R diag = R((flags >> 0) & 1) + R((flags >> 1) & 1) + (R((flags >> 2) & 1) + R((flags >> 3) & 1)) +
                   (R((flags >> 4) & 1) + R((flags >> 5) & 1));
          first = mixr(R(0), (R(0) - stored) / std::max(diag, R(1e-12)), R(0.8));
        }
      }
      cfirst[out] = store_round(first, storeMode(level));
    });
  }
  bool coarseSolid(int px, int py, int pz, int level) {
    long a = cellAddress(px, py, pz, level);
    if (a < 0) return false;
    return (topo(level)[a] & STORED_SOLID) != 0;
  }
  R coarseValue(const std::vector<R>& coarse, int level, int px, int py, int pz) {
    int groundY = ground ? 0 : -0x7fffffff;
    int c[3] = {px, std::max(py, groundY), pz};
    if (!coarseSolid(c[0], c[1], c[2], level)) return readAt(coarse, c[0], c[1], c[2], level);
    R sum = 0, count = 0;
    for (int axis = 0; axis < 3; axis++)
      for (int side = -1; side <= 1; side += 2) {
        int q[3] = {c[0], c[1], c[2]};
        q[axis] += side;
        q[1] = std::max(q[1], groundY);
        if (!coarseSolid(q[0], q[1], q[2], level)) {
          sum += readAt(coarse, q[0], q[1], q[2], level);
          count += 1;
        }
      }
    return sum / std::max(count, R(1));
  }
  // prolongateCell (pressure.wgsl:726-755)
  void prolongate(int level, const std::vector<R>& pin, const std::vector<R>& coarse, std::vector<R>& pout) {
    int cl = level + 1;
    forLevelCells(level, [&](int px, int py, int pz) {
      long a = cellAddress(px, py, pz, level);
      uint32_t flags = flagsOf(level, a);
      if ((flags & SOLID) || !activeCell(px, py, pz, level)) {
        pout[a] = 0;
        return;
      }
      R q[3] = {(R(px) + R(0.5)) * R(0.5) - R(0.5), (R(py) + R(0.5)) * R(0.5) - R(0.5), (R(pz) + R(0.5)) * R(0.5) - R(0.5)};
      int i[3];
      R f[3];
      for (int k = 0; k < 3; k++) {
        i[k] = floori((double)q[k]);
        f[k] = q[k] - std::floor(q[k]);
      }
      bool fast = colliderCount == 0 && (!ground || i[1] >= 0);
      auto cv = [&](int dx, int dy, int dz) {
        return fast ? readAt(coarse, i[0] + dx, i[1] + dy, i[2] + dz, cl) : coarseValue(coarse, cl, i[0] + dx, i[1] + dy, i[2] + dz);
      };
      R corr = mixr(mixr(mixr(cv(0, 0, 0), cv(1, 0, 0), f[0]), mixr(cv(0, 1, 0), cv(1, 1, 0), f[0]), f[1]),
                    mixr(mixr(cv(0, 0, 1), cv(1, 0, 1), f[0]), mixr(cv(0, 1, 1), cv(1, 1, 1), f[0]), f[1]), f[2]);
      pout[a] = store_round(pin[a] + corr, storeMode(level));
    });
  }
  // The level's pressure pair and right-hand side.
  std::vector<R>& P(int level, int k) { return level == 0 ? pres[k] : levels[level].p[k]; }
  std::vector<R>& RHS(int level) { return level == 0 ? (rhs0 ? *rhs0 : div) : levels[level].rhs; }
  void smooth(int level, int n, bool& initialize) {
    Level& L = levels[level];
    for (int i = 0; i < n; i++) {
      bool first = level == 0 && initialize;
      relax(level, RHS(level), P(level, L.current), P(level, 1 - L.current), first);
      L.current = 1 - L.current;
      if (first) initialize = false;
    }
  }
  // relaxCoarse (pressure.wgsl:549-599): the bottom level, iterations in one group.
  void bottomSolve(int iterations) {
    int level = bottom;
    Level& L = levels[level];
    std::vector<R>& pin = P(level, L.current);
    std::vector<R> value(capacity, 0), source(capacity, 0);
    std::vector<uint32_t> flags(capacity, SOLID);
    std::vector<bool> valid(capacity, false);
    for (int t = 0; t < capacity; t++) {
      valid[t] = snapshotState[t] != 0;
      if (valid[t] && activeCell(snapshot[t][0], snapshot[t][1], snapshot[t][2], level)) {
        long a = cellAddress(snapshot[t][0], snapshot[t][1], snapshot[t][2], level);
        flags[t] = flagsOf(level, a);
        source[t] = RHS(level)[a];
        value[t] = pin[a];
      }
    }
    static const int nb[6] = {neighborIndex(1, 0, 0), neighborIndex(-1, 0, 0), neighborIndex(0, 1, 0),
                              neighborIndex(0, -1, 0), neighborIndex(0, 0, 1), neighborIndex(0, 0, -1)};
    for (int it = 0; it < iterations; it++) {
      std::vector<R> next(capacity, 0);
      for (int t = 0; t < capacity; t++) {
        if (!valid[t] || (flags[t] & SOLID)) continue;
        R v[6];
        for (int s = 0; s < 6; s++) {
          v[s] = 0;
          if (!(flags[t] & (1u << s))) continue;
          int n = tileNeighbors[(size_t)t * 27 + nb[s]];
          if (n >= 0) v[s] = value[n];
        }
        R sum = (v[0] + v[1]) + (v[2] + v[3]) + (v[4] + v[5]);
        uint32_t fl = flags[t];
        R diag = R((fl >> 0) & 1) + R((fl >> 1) & 1) + (R((fl >> 2) & 1) + R((fl >> 3) & 1)) +
                 (R((fl >> 4) & 1) + R((fl >> 5) & 1));
        R cand = (sum - source[t]) / std::max(diag, R(1e-12));
        next[t] = store_round(mixr(value[t], cand, R(0.8)), storeMode(level));
      }
      value.swap(next);
    }
    std::vector<R>& pout = P(level, 1 - L.current);
    for (int t = 0; t < capacity; t++)
      if (valid[t]) {
        long a = cellAddress(snapshot[t][0], snapshot[t][1], snapshot[t][2], level);
        if (a >= 0) pout[a] = value[t];
      }
    L.current = 1 - L.current;
  }
  void cycle(int index, bool& initialize) {
    if (index == bottom) {
      if (capacity <= 256) {
        bottomSolve(19);
      } else {
        smooth(index, 19, initialize);
      }
      return;
    }
    // The finest level's only pre-smoothing is the first iterate from zero; a later V-cycle
    // restricts the residual of the current iterate directly.
    smooth(index, index > 0 ? 2 : (initialize ? 1 : 0), initialize);
    Level& L = levels[index];
    Level& C = levels[index + 1];
    restrictLevel(index, RHS(index), P(index, L.current), RHS(index + 1), P(index + 1, 1));
    C.current = 1;
    cycle(index + 1, initialize);
    prolongate(index, P(index, L.current), P(index + 1, C.current), P(index, 1 - L.current));
    L.current = 1 - L.current;
    smooth(index, 3, initialize);
  }
  // ---- red-black Gauss-Seidel (no reference counterpart; the reference smooths with Jacobi)
  // The coarsest level of the red-black V-cycle.
  int coarsestLevel() const { return mgLevels > 0 ? std::min(mgLevels - 1, bottom) : bottom; }
  // One colour of a level in place: the cells with x + y + z of parity `colour` take
  // (sum of open neighbours - rhs) / diag, the others keep their value. From `zero`, every
  // neighbour reads zero and the other colour's cells become zero.
  void relaxColour(int level, std::vector<R>& p, int colour, bool zero) {
    const std::vector<R>& rhs = RHS(level);
    forLevelCells(level, [&](int px, int py, int pz) {
      long a = cellAddress(px, py, pz, level);
      if (((px + py + pz) & 1) != colour) {
        if (zero) p[a] = 0;
        return;
      }
      uint32_t flags = flagsOf(level, a);
      if ((flags & SOLID) || !activeCell(px, py, pz, level)) {
        p[a] = 0;
        return;
      }
      R sum = 0, diag = axisDiag(flags);
      if (!zero) stencil(px, py, pz, flags, level, p, sum, diag);
      p[a] = store_round((sum - rhs[a]) / std::max(diag, R(1e-12)), storeMode(level));
    });
  }
  // `n` sweeps: red then black, or after a prolongation black then red.
  void sweepsRB(int level, std::vector<R>& p, int n, bool zero, bool post) {
    for (int i = 0; i < n; i++) {
      int first = post ? 1 : 0;
      relaxColour(level, p, first, zero && i == 0);
      relaxColour(level, p, 1 - first, false);
    }
  }
  void cycleRB(int index, bool zero) {
    std::vector<R>& p = P(index, 0);
    if (index == coarsestLevel()) {
      sweepsRB(index, p, bottomSweeps, zero, false);
      return;
    }
    sweepsRB(index, p, preSweeps, zero, false);
    // The restriction's first iterate of the coarse level goes to the level's other buffer,
    // unused: the coarse level starts from zero.
    restrictLevel(index, RHS(index), p, RHS(index + 1), P(index + 1, 1));
    cycleRB(index + 1, true);
    prolongate(index, p, P(index + 1, 0), p);
    sweepsRB(index, p, postSweeps, false, true);
  }
  // One V-cycle of the schedule's smoother on the finest level, from zero (`zero`) or from its
  // current iterate; returns the finest level's buffer that holds the result.
  std::vector<R>& vcycleOnce(bool zero, bool& initialize) {
    if (smoother == FP_SMOOTHER_REDBLACK) {
      cycleRB(0, zero);
      return P(0, 0);
    }
    if (zero) initialize = true;
    cycle(0, initialize);
    return P(0, levels[0].current);
  }

  // ---- flexible conjugate gradients on the finest level (no reference counterpart)
  // Finest-level unknowns, and A v = diag v - (sum of open neighbours) there.
  bool unknown0(int px, int py, int pz, long a) {
    uint32_t flags = flagsOf(0, a);
    return !(flags & SOLID) && activeCell(px, py, pz, 0);
  }
  // Over the finest level's unknown cells: fn(a, flags, px, py, pz) -> a contribution to a sum.
  template <class F>
  double sumUnknowns(F fn) {
    int side = levelSide(0), cells = side * side * side;
    long n = (long)active.size();
    double total = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : total)
    for (long i = 0; i < n; i++) {
      I3 b = brickOf(active[i]);
      for (int o = 0; o < cells; o++) {
        int px = b[0] * side + o % side, py = b[1] * side + (o / side) % side, pz = b[2] * side + o / (side * side);
        long a = cellAddress(px, py, pz, 0);
        if (a < 0 || !unknown0(px, py, pz, a)) continue;
        total += fn(a, flagsOf(0, a), px, py, pz);
      }
    }
    return total;
  }
  R applyAt(const std::vector<R>& v, long a, uint32_t flags, int px, int py, int pz) {
    R sum, diag;
    stencil(px, py, pz, flags, 0, v, sum, diag);
    return diag * v[a] - sum;
  }
  void solveFCG() {
    size_t n = pres[0].size();
    kx.assign(n, 0);
    ks.assign(n, 0);
    kd.assign(n, 0);
    kq.assign(n, 0);
    cgRes2.assign(vcycles, 0.0);
    bool initialize = true;
    rhs0 = nullptr;
    // The start: one V-cycle from zero on the divergence; s = rhs + A x.
    kx = vcycleOnce(true, initialize);
    double rhs2 = 0;
    double r2 = sumUnknowns([&](long a, uint32_t f, int px, int py, int pz) {
      R v = div[a] + applyAt(kx, a, f, px, py, pz);
      ks[a] = v;
      return (double)v * (double)v;
    });
    rhs2 = sumUnknowns([&](long a, uint32_t, int, int, int) { return (double)div[a] * (double)div[a]; });
    cgRes2[0] = r2;
    double dqPrev = 0;
    for (int c = 1; c < vcycles; c++) {
      if (tolerance > 0 && cgRes2[c - 1] <= (double)tolerance * (double)tolerance * rhs2) break;
      // z = V(s): one V-cycle from zero with the residual as its right-hand side.
      rhs0 = &ks;
      std::vector<R> z = vcycleOnce(true, initialize);
      rhs0 = nullptr;
      double beta = 0;
      if (c > 1) {
        double zq = sumUnknowns([&](long a, uint32_t, int, int, int) { return (double)z[a] * (double)kq[a]; });
        beta = dqPrev != 0 ? -zq / dqPrev : 0.0;
      }
      // d = z + beta d; q = A z + beta q (= A d); then d.q and d.s.
      std::vector<R> az(n, 0);
      sumUnknowns([&](long a, uint32_t f, int px, int py, int pz) {
        az[a] = applyAt(z, a, f, px, py, pz);
        return 0.0;
      });
      double dq = sumUnknowns([&](long a, uint32_t, int, int, int) {
        R d = z[a] + (R)beta * kd[a];
        R q = az[a] + (R)beta * kq[a];
        kd[a] = d;
        kq[a] = q;
        return (double)d * (double)q;
      });
      double ds = sumUnknowns([&](long a, uint32_t, int, int, int) { return (double)kd[a] * (double)ks[a]; });
      double alpha = dq != 0 ? -ds / dq : 0.0;
      dqPrev = dq;
      cgRes2[c] = sumUnknowns([&](long a, uint32_t, int, int, int) {
        kx[a] += (R)alpha * kd[a];
        R v = ks[a] + (R)alpha * kq[a];
        ks[a] = v;
        return (double)v * (double)v;
      });
    }
    pres[latest] = kx;
  }
  // PressureSolver.solve (PressureSolver.ts:371-402) with PRESSURE_CYCLES = 1, or the
  // schedule's solve.
  void solvePressure() {
    buildZeroedTopology();
    buildTopology();
    if (krylov == FP_KRYLOV_FCG) {
      levels[0].current = latest;
      solveFCG();
      return;
    }
    cgRes2.assign(vcycles, 0.0);
    // The residual rhs + A p of the finest level's iterate, as a sum of squares.
    auto residual2 = [&](const std::vector<R>& p) {
      return sumUnknowns([&](long a, uint32_t f, int px, int py, int pz) {
        double v = (double)(div[a] + applyAt(p, a, f, px, py, pz));
        return v * v;
      });
    };
    if (smoother == FP_SMOOTHER_REDBLACK) {
      // In place on the finest level's first buffer; later V-cycles correct the current iterate.
      for (int c = 0; c < vcycles; c++) {
        cycleRB(0, c == 0);
        cgRes2[c] = residual2(P(0, 0));
      }
      latest = 0;
      return;
    }
    levels[0].current = latest;
    bool initialize = true;
    for (int c = 0; c < vcycles; c++) {
      cycle(0, initialize);
      if (vcycles > 1) cgRes2[c] = residual2(P(0, levels[0].current));
    }
    latest = levels[0].current;
  }

  // ---------------------------------------------------------------- projection
  bool pressureUnknown(int px, int py, int pz) {
    int p[3] = {px, py, pz}, lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = (p[a] - 1) >> vshift;
      hi[a] = p[a] >> vshift;
    }
    if (ground) lo[1] = std::max(lo[1], 0);
    for (int z = lo[2]; z <= hi[2]; z++)
      for (int y = lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++)
          if (brickEntry(x, y, z) < 0) return false;
    return true;
  }
  R cellPressure(int x, int y, int z) {
    int s = brickSlot(x >> vshift, y >> vshift, z >> vshift);
    if (s < 0) return 0;
    return pres[latest][(size_t)s * VN + vlocal(x, y, z)];
  }
  // project (fluid-forces.wgsl:205-262) into the velocity pool of the next step.
  void projectStep() {
    std::vector<R> out(vel.size(), 0);
    forActiveVCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      V3<R> pos = vcenter(x, y, z);
      R res[3] = {0, 0, 0};
      if (!solidAt(pos[0], pos[1], pos[2])) {
        R cp = pres[latest][(size_t)slot * VN + c];
        bool pu = pressureUnknown(x, y, z);
        for (int a = 0; a < 3; a++) {
          int n[3] = {x, y, z};
          n[a] += 1;
          R v = velF[((size_t)slot * 3 + a) * VN + c];
          V3<R> nc = vcenter(n[0], n[1], n[2]);
          if (solidAt(nc[0], nc[1], nc[2])) {
            res[a] = 0;
          } else if (!pu && !pressureUnknown(n[0], n[1], n[2])) {
            res[a] = 0;
          } else {
            res[a] = v - (cellPressure(n[0], n[1], n[2]) - cp) / vh;
          }
        }
      }
      for (int a = 0; a < 3; a++) out[((size_t)slot * 3 + a) * VN + c] = sv(res[a]);
    });
    vel.swap(out);
  }

  // The projected velocity's divergence less the expansion it keeps, over the interior
  // unknowns (every neighbour solid or an unknown), as the CUDA measurement takes it:
  // out[0] sum of (h div u - h e)^2, out[1] sum of the face velocities' squares, out[2] cells,
  // then the `top` largest cells as (x, y, z, value, solid neighbours, expansion) in out[3..].
  void postDivergence(double* out, int top) {
    std::vector<std::array<double, 6>> cells;
    double d2 = 0, v2 = 0;
    forActiveVCells([&](uint32_t, int slot, int c, int x, int y, int z) {
      (void)slot;
      auto solid = [&](int qx, int qy, int qz) { V3<R> p = vcenter(qx, qy, qz); return solidAt(p[0], p[1], p[2]); };
      if (solid(x, y, z) || !pressureUnknown(x, y, z)) return;
      const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
      int solids = 0;
      for (int k = 0; k < 6; k++) {
        const bool sk = solid(x + off[k][0], y + off[k][1], z + off[k][2]);
        solids += sk ? 1 : 0;
        if (!sk && !pressureUnknown(x + off[k][0], y + off[k][1], z + off[k][2])) return;
      }
      R u0 = vcell(vel, 3, 0, x, y, z), u1 = vcell(vel, 3, 1, x, y, z), u2 = vcell(vel, 3, 2, x, y, z);
      R e = vd == 1 ? expn[(size_t)brickSlot(x >> shift, y >> shift, z >> shift) * N + local(x, y, z)] : R(0);
      double d = (double)((u0 - vcell(vel, 3, 0, x - 1, y, z)) + (u1 - vcell(vel, 3, 1, x, y - 1, z)) +
                          (u2 - vcell(vel, 3, 2, x, y, z - 1)) - vh * e);
#pragma omp critical
      {
        d2 += d * d;
        v2 += (double)u0 * u0 + (double)u1 * u1 + (double)u2 * u2;
        cells.push_back({(double)x, (double)y, (double)z, d, (double)solids, (double)e});
      }
    });
    std::sort(cells.begin(), cells.end(), [](const std::array<double, 6>& a, const std::array<double, 6>& b) {
      return std::fabs(a[3]) > std::fabs(b[3]);
    });
    out[0] = d2;
    out[1] = v2;
    out[2] = (double)cells.size();
    for (int k = 0; k < top && k < (int)cells.size(); k++)
      for (int j = 0; j < 6; j++) out[3 + 6 * k + j] = cells[k][j];
  }

  // ---------------------------------------------------------------- measurement
  // readActivity (FluidSimulation.ts:1701-1746), applied before the next step.
  void readActivity() {
    contentTiles.clear();
    for (int s = 0; s < capacity; s++) {
      uint32_t f = activity[(size_t)capacity * 64 + s];
      if (f && snapshotState[s] != 0) contentTiles.push_back({snapshot[s], f});
    }
    activeBrickCount = (uint32_t)active.size();
    usedSlots = slots - (uint32_t)freeCount;
    uint32_t limit = slotLimit();
    lastFailures = failures;
    poolLimited = failures > 0 && slots >= limit;
    failures = 0;
  }
};

}  // namespace orc

// =========================================================================================
// C API for ctypes (tests and the CPU baseline).
// =========================================================================================
struct or_sim {
  int real;  // 0 double, 1 float
  orc::Sim<double>* d = nullptr;
  orc::Sim<float>* f = nullptr;
  std::string error;
};

template <class S, class Fn>
static auto with(or_sim* s, Fn fn) {
  if (s->d) return fn(*s->d);
  return fn(*s->f);
}

extern "C" {

// mode: 0 storage as the grid's precision says (FP32 -> exact in the real type);
//       2 the reference's half-precision storage with its truncations.
or_sim* or_create(const fp_grid* g, int real, int mode) {
  orc::Prec p;
  if (mode == 2) {
    p.vel = p.scal = p.expn = p.p0 = p.pc = p.curl = p.bounds = orc::STORE_F16;
    p.truncate = true;
  } else if (g->precision == FP_PRECISION_MIXED) {
    p.scal = orc::STORE_F16;
    p.pc = orc::STORE_BF16;
  }
  if (g->brick_size != 8 && g->brick_size != 16 && g->brick_size != 32) return nullptr;
  or_sim* s = new or_sim();
  s->real = real;
  if (real == 0)
    s->d = new orc::Sim<double>(*g, p);
  else
    s->f = new orc::Sim<float>(*g, p);
  return s;
}
// The storage-rounding helpers, exported so the tests can pin them to numpy's.
double or_round_f16(double x) { return orc::round_f16(x); }
double or_round_bf16(double x) { return orc::round_bf16(x); }
double or_truncate_half(double x) { return orc::truncate_half(x); }
double or_noise_hash(int x, int y, int z) { return orc::noise_hash(x, y, z); }

void or_destroy(or_sim* s) {
  if (!s) return;
  delete s->d;
  delete s->f;
  delete s;
}
void or_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}
void or_set_runtime(or_sim* s, float cutoff, double budget, int ground) {
  auto fn = [&](auto& sim) {
    sim.cutoff = cutoff;
    if (budget > 0) sim.voxelBudget = budget;
    sim.ground = ground != 0;
    return 0;
  };
  if (s->d) fn(*s->d); else fn(*s->f);
}
// blackbodyTable (src/engine/blackbody.ts:1-97), restated for the oracle: Planck radiance
// against the multi-lobe CIE observer fit (Wyman, Sloan and Shirley, JCGT 2013), linear sRGB,
// peak-normalised, log2 radiance relative to 1800 K, 512 entries from 500 K to 10000 K.
static void or_blackbody(double kelvin, double rgb[3]) {
  static const double lobes[7][5] = {{0, 0.362, 442, 0.0624, 0.0374},  {0, 1.056, 599.8, 0.0264, 0.0323},
                                     {0, -0.065, 501.1, 0.049, 0.0382}, {1, 0.821, 568.8, 0.0213, 0.0247},
                                     {1, 0.286, 530.9, 0.0613, 0.0322}, {2, 1.217, 437, 0.0845, 0.0278},
                                     {2, 0.681, 459, 0.0385, 0.0725}};
  const double hp = 6.62607015e-34, c = 299792458.0, kb = 1.380649e-23;
  double xyz[3] = {0, 0, 0};
  for (int i = 0; i < 95; i++) {
    double wl = 360.0 + 5.0 * i, w = wl * 1e-9;
    double radiance = 2 * hp * c * c / (std::pow(w, 5) * std::expm1(hp * c / (w * kb * kelvin))) * 5e-9;
    for (const auto& L : lobes) {
      double d = (wl - L[2]) * (wl < L[2] ? L[3] : L[4]);
      xyz[(int)L[0]] += L[1] * std::exp(-0.5 * d * d) * radiance;
    }
  }
  rgb[0] = std::max(0.0, 3.2406 * xyz[0] - 1.5372 * xyz[1] - 0.4986 * xyz[2]);
  rgb[1] = std::max(0.0, -0.9689 * xyz[0] + 1.8758 * xyz[1] + 0.0415 * xyz[2]);
  rgb[2] = std::max(0.0, 0.0557 * xyz[0] - 0.204 * xyz[1] + 1.057 * xyz[2]);
}
void or_blackbody_table(float* out) {
  double ref[3];
  or_blackbody(1800.0, ref);
  double refPeak = std::max(ref[0], std::max(ref[1], ref[2]));
  for (int i = 0; i < 512; i++) {
    double rgb[3];
    or_blackbody(500.0 + 9500.0 * i / 511.0, rgb);
    double peak = std::max(rgb[0], std::max(rgb[1], rgb[2]));
    if (peak <= 0) {
      out[i * 4] = out[i * 4 + 1] = out[i * 4 + 2] = 0.f;
      out[i * 4 + 3] = -32.f;
      continue;
    }
    for (int c = 0; c < 3; c++) out[i * 4 + c] = (float)(rgb[c] / peak);
    out[i * 4 + 3] = (float)std::max(-32.0, std::log2(peak / refPeak));
  }
}
// The render of the current state (the CUDA render's restatement), into `image` (w x h x 4).
int or_render(or_sim* s, const fp_camera* cam, const fp_render_settings* rs, float* image) {
  std::vector<float> lut(512 * 4);
  or_blackbody_table(lut.data());
  if (s->d)
    s->d->render(*cam, *rs, lut.data(), image);
  else
    s->f->render(*cam, *rs, lut.data(), image);
  return 0;
}
// The scene-light sums of the current state (FP64), 8 per anchor.
int or_collect_lights(or_sim* s, const fp_render_settings* rs, const float* anchors, int count, double* sums) {
  std::vector<float> lut(512 * 4);
  or_blackbody_table(lut.data());
  if (s->d)
    s->d->collectLights(*rs, lut.data(), anchors, count, sums);
  else
    s->f->collectLights(*rs, lut.data(), anchors, count, sums);
  return 0;
}
// The number of V-cycles of each later step's pressure solve (the CUDA step's solver setting
// with tolerance 0).
void or_set_solver(or_sim* s, int vcycles) {
  if (s->d)
    s->d->vcycles = vcycles;
  else
    s->f->vcycles = vcycles;
}
// The pressure solve's schedule (fp_solver_schedule) and the CG tolerance, for later steps.
void or_set_schedule(or_sim* s, const fp_solver_schedule* sc, float tolerance) {
  auto fn = [&](auto& sim) {
    sim.smoother = sc->smoother;
    sim.mgLevels = sc->levels;
    sim.preSweeps = sc->pre_sweeps;
    sim.postSweeps = sc->post_sweeps;
    sim.bottomSweeps = sc->bottom_sweeps;
    sim.krylov = sc->krylov;
    sim.topologyEachStep = sc->topology;
    sim.tolerance = tolerance;
  };
  if (s->d)
    fn(*s->d);
  else
    fn(*s->f);
}
// The latest state's post-projection divergence (Sim::postDivergence).
void or_post_divergence(or_sim* s, double* out, int top) {
  if (s->d)
    s->d->postDivergence(out, top);
  else
    s->f->postDivergence(out, top);
}
// The finest level's CG residual sums of squares of the latest solve, one per V-cycle run.
int or_read_cg(or_sim* s, double* out, int capacity) {
  auto fn = [&](auto& sim) -> int {
    int n = std::min(capacity, (int)sim.cgRes2.size());
    for (int i = 0; i < n; i++) out[i] = sim.cgRes2[i];
    return n;
  };
  return s->d ? fn(*s->d) : fn(*s->f);
}
int or_step(or_sim* s, const fp_frame* f, float dt) {
  std::string e = s->d ? s->d->step(*f, dt) : s->f->step(*f, dt);
  s->error = e;
  return e.empty() ? 0 : -1;
}
const char* or_error(or_sim* s) { return s->error.c_str(); }

// Sizes: 0 slots, 1 capacity (tile slots), 2 cells per brick, 3 active bricks, 4 steps,
// 5 used slots, 6 pool limited, 7 failures at the last measurement, 8 tiles.
int64_t or_info(or_sim* s, int what) {
  auto fn = [&](auto& sim) -> int64_t {
    switch (what) {
      case 0: return sim.slots;
      case 1: return sim.capacity;
      case 2: return sim.N;
      case 3: return sim.activeBrickCount;
      case 4: return sim.steps;
      case 5: return sim.usedSlots;
      case 6: return sim.poolLimited;
      case 7: return sim.lastFailures;
      case 8: return sim.dir.count();
      case 9: return sim.SN;  // coarse smoke cells a brick (smokeDivisor > 1)
      case 10: return sim.VN;  // velocity and pressure cells a brick
    }
    return -1;
  };
  return s->d ? fn(*s->d) : fn(*s->f);
}

// Field copy out/in as float, layout [slot][channel][cell] (FP_FIELD_*). `write` copies in.
static int field_io(or_sim* s, int field, float* buf, size_t count, int write) {
  auto fn = [&](auto& sim) -> int {
    using R = typename std::remove_reference<decltype(sim.h)>::type;
    std::vector<R>* v = nullptr;
    switch (field) {
      case FP_FIELD_VELOCITY: v = &sim.vel; break;
      case FP_FIELD_SCALARS: v = &sim.fld; break;
      case FP_FIELD_EXPANSION: v = &sim.expn; break;
      case FP_FIELD_PRESSURE: v = &sim.pres[sim.latest]; break;
      case FP_FIELD_DIVERGENCE: v = &sim.div; break;
      case FP_FIELD_CURL: v = &sim.curl; break;
      case FP_FIELD_SMOKE: v = &sim.smk; break;
      default: return -1;
    }
    if (count != v->size()) return -2;
    if (write)
      for (size_t i = 0; i < count; i++) (*v)[i] = (R)buf[i];
    else
      for (size_t i = 0; i < count; i++) buf[i] = (float)(*v)[i];
    return 0;
  };
  return s->d ? fn(*s->d) : fn(*s->f);
}
int or_read_field(or_sim* s, int field, float* out, size_t count) { return field_io(s, field, out, count, 0); }
int or_write_field(or_sim* s, int field, const float* in, size_t count) {
  return field_io(s, field, const_cast<float*>(in), count, 1);
}
// Double-precision copy out, for the error oracle's comparisons.
int or_read_field64(or_sim* s, int field, double* out, size_t count) {
  if (!s->d) return -1;
  auto& sim = *s->d;
  std::vector<double>* v = nullptr;
  switch (field) {
    case FP_FIELD_VELOCITY: v = &sim.vel; break;
    case FP_FIELD_SCALARS: v = &sim.fld; break;
    case FP_FIELD_EXPANSION: v = &sim.expn; break;
    case FP_FIELD_PRESSURE: v = &sim.pres[sim.latest]; break;
    case FP_FIELD_DIVERGENCE: v = &sim.div; break;
    case FP_FIELD_CURL: v = &sim.curl; break;
    case FP_FIELD_SMOKE: v = &sim.smk; break;
    default: return -1;
  }
  if (count != v->size()) return -2;
  std::memcpy(out, v->data(), count * 8);
  return 0;
}

// Integer tables (FP_TABLE_*); returns the words written or needed.
int64_t or_read_table(or_sim* s, int table, void* out, size_t capacityBytes) {
  auto fn = [&](auto& sim) -> int64_t {
    std::vector<uint32_t> w;
    size_t bricks = (size_t)sim.capacity * 64;
    switch (table) {
      case FP_TABLE_ENTRIES: w.assign(sim.entries.begin(), sim.entries.end()); break;
      case FP_TABLE_PAGES: w.assign(sim.pages.begin(), sim.pages.end()); break;
      case FP_TABLE_STATE: w = sim.state; break;
      case FP_TABLE_ACTIVITY: w = sim.activity; break;
      case FP_TABLE_RECORDS: w.assign(sim.records.begin(), sim.records.end()); break;
      case FP_TABLE_FREE:
        w.push_back((uint32_t)sim.freeCount);
        w.push_back(sim.lastFailures);
        w.insert(w.end(), sim.freeStack.begin(), sim.freeStack.end());
        break;
      case FP_TABLE_ACTIVE:
        w.push_back((uint32_t)sim.active.size());
        w.insert(w.end(), sim.active.begin(), sim.active.end());
        break;
      case FP_TABLE_SOLIDS: w = sim.solids; break;
      case FP_TABLE_TILES:
        for (int t = 0; t < sim.capacity; t++) {
          w.push_back((uint32_t)sim.snapshot[t][0]);
          w.push_back((uint32_t)sim.snapshot[t][1]);
          w.push_back((uint32_t)sim.snapshot[t][2]);
          w.push_back((uint32_t)sim.snapshotState[t]);
        }
        break;
      default: return -1;
    }
    (void)bricks;
    size_t bytes = w.size() * 4;
    if (out && capacityBytes >= bytes) std::memcpy(out, w.data(), bytes);
    return (int64_t)w.size();
  };
  return s->d ? fn(*s->d) : fn(*s->f);
}
// Overwrite the activity flags (teacher forcing of the content measurement).
int or_write_activity(or_sim* s, const uint32_t* in, size_t count) {
  auto fn = [&](auto& sim) -> int {
    if (count != sim.activity.size()) return -2;
    std::memcpy(sim.activity.data(), in, count * 4);
    sim.contentTiles.clear();
    for (int t = 0; t < sim.capacity; t++) {
      uint32_t f = sim.activity[(size_t)sim.capacity * 64 + t];
      if (f && sim.snapshotState[t] != 0) sim.contentTiles.push_back({sim.snapshot[t], f});
    }
    return 0;
  };
  return s->d ? fn(*s->d) : fn(*s->f);
}

}  // extern "C"
