// Host engine: see fp_engine.hpp. Citations are path:line in the reference project.
#include "fp_engine.hpp"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <map>

#include "fp_launch.h"

namespace fp {

static const int TILE_BRICKS = 4;
static const int LINGER_STEPS = 60;  // TileDirectory.ts:8
static const int MIN_TILES = 16;     // FluidSimulation.ts:72
static const int HASH_ROW = 256;     // TileDirectory.ts:17

// ------------------------------------------------------------------------ TileDirectory
void TileDirectory::need(int lx, int ly, int lz, int hx, int hy, int hz, int64_t step) {
  for (int z = lz; z <= hz; z++)
    for (int y = ground ? std::max(0, ly) : ly; y <= hy; y++)
      for (int x = lx; x <= hx; x++) {
        auto it = index_.find(key(x, y, z));
        if (it != index_.end()) {
          Tile& t = slots_[it->second];
          t.needed = step;
          if (t.closing) {
            t.closing = false;
            dirty = true;
          }
          continue;
        }
        int slot = -1;
        for (size_t i = 0; i < slots_.size(); i++)
          if (!slots_[i].alive) {
            slot = (int)i;
            break;
          }
        if (slot < 0) {
          slot = (int)slots_.size();
          slots_.push_back(Tile{});
        }
        slots_[slot] = Tile{x, y, z, step, false, true, nextSeq_++};
        index_[key(x, y, z)] = slot;
        created_.push_back(slot);
        dirty = true;
      }
}
void TileDirectory::retire(int64_t step) {
  for (size_t s = 0; s < slots_.size(); s++) {
    Tile& t = slots_[s];
    if (!t.alive) continue;
    if (t.closing) {
      index_.erase(key(t.x, t.y, t.z));
      t.alive = false;
      dirty = true;
    } else if (step - t.needed > LINGER_STEPS) {
      t.closing = true;
      dirty = true;
    }
  }
  while (!slots_.empty() && !slots_.back().alive) slots_.pop_back();
}
void TileDirectory::clear() {
  slots_.clear();
  index_.clear();
  created_.clear();
  dirty = true;
}
int TileDirectory::slotAt(int x, int y, int z) const {
  auto it = index_.find(key(x, y, z));
  return it == index_.end() ? -1 : it->second;
}
std::vector<int> TileDirectory::takeCreated() {
  std::vector<int> out;
  for (int s : created_)
    if (s < (int)slots_.size() && slots_[s].alive) out.push_back(s);
  created_.clear();
  return out;
}

// ------------------------------------------------------------------------ Engine
int Engine::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FP_OK;
  error_ = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? FP_ENOMEM : FP_EDEVICE;
}

bool Engine::alloc(DeviceBuffer& b, size_t bytes, bool zero) {
  if (b.ptr) cudaFree(b.ptr);
  b.ptr = nullptr;
  b.bytes = 0;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(&b.ptr, bytes) != cudaSuccess) {
    b.ptr = nullptr;
    error_ = "device memory exhausted";
    return false;
  }
  b.bytes = bytes;
  if (zero) cudaMemsetAsync(b.ptr, 0, bytes, stream());
  return true;
}

bool Engine::grow(DeviceBuffer& b, size_t bytes, int fill) {
  if (bytes <= b.bytes && b.ptr) return true;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    error_ = "device memory exhausted";
    return false;
  }
  cudaMemsetAsync(p, fill, bytes, stream());
  if (b.ptr) {
    cudaMemcpyAsync(p, b.ptr, b.bytes, cudaMemcpyDeviceToDevice, stream());
    cudaStreamSynchronize(stream());
    cudaFree(b.ptr);
  }
  b.ptr = p;
  b.bytes = bytes;
  return true;
}

// Host-to-device copies go through a pinned arena, so they are truly asynchronous. The arena
// restarts each step: the previous step's copies ran before its allocation kernels, which
// precede the measurement the step start waits for.
bool Engine::upload(DeviceBuffer& b, const void* src, size_t bytes) {
  if (bytes == 0) return true;
  if (bytes > b.bytes) {
    cudaStreamSynchronize(stream());  // the old buffer may still be read: rare growth
    if (!alloc(b, std::max(bytes + bytes / 2, (size_t)256), false)) return false;
  }
  size_t off = (stageUsed_ + 255) & ~(size_t)255;
  if (off + bytes > stageCap_) {
    cudaStreamSynchronize(stream());  // copies from the old arena must finish before it goes
    if (stageH_) cudaFreeHost(stageH_);
    stageCap_ = std::max(std::max(stageCap_ * 2, off + bytes), (size_t)1 << 20);
    if (cudaMallocHost(&stageH_, stageCap_) != cudaSuccess) {
      stageH_ = nullptr;
      stageCap_ = 0;
      error_ = "pinned host memory exhausted";
      return false;
    }
    off = 0;
  }
  std::memcpy(stageH_ + off, src, bytes);
  stageUsed_ = off + bytes;
  h2d_ += bytes;
  return cudaMemcpyAsync(b.ptr, stageH_ + off, bytes, cudaMemcpyHostToDevice, stream()) == cudaSuccess;
}

uint32_t Engine::slotLimit() const {
  double v = std::floor(budget_ / (double)N_);
  return (uint32_t)std::max(1.0, v);
}

Engine::Engine(const fp_grid& g, Stepper* owner) : owner_(owner) {
  B_ = g.brick_size;
  shift_ = B_ == 8 ? 3 : (B_ == 16 ? 4 : 5);
  N_ = B_ * B_ * B_;
  W_ = N_ / 32;
  vd_ = g.velocity_divisor > 1 ? g.velocity_divisor : 1;
  VB_ = B_ / vd_;
  vshift_ = 0;
  while ((1 << vshift_) < VB_) vshift_++;
  VN_ = VB_ * VB_ * VB_;
  brickLevels_ = vshift_;  // the pressure lives on the velocity lattice
  bottom_ = brickLevels_ + 2;
  h_ = g.voxel_size;
  maccormack_ = g.scalar_maccormack != 0;
  precision_ = g.precision;
  smokeDiv_ = g.smoke_divisor > 1 ? g.smoke_divisor : 1;
  SB_ = B_ / smokeDiv_;
  sshift_ = 0;
  while ((1 << sshift_) < SB_) sshift_++;
  SN_ = SB_ * SB_ * SB_;
  budget_ = g.voxel_budget > 0 ? g.voxel_budget : 8e6;
  measure_ = precision_ == FP_PRECISION_MIXED;  // mixed storage reports its accuracy every step
}

Engine::~Engine() {
  owner_->forget(this);
  cudaStreamSynchronize(stream());
  freeAll();
  DeviceBuffer* render[] = {&renderField_, &renderSmoke_, &sceneDepth_, &slices_, &lighting_, &occupancy_, &lut_, &renderParams_, &image_, &anchors_, &lightSums_, &renderBoxesD_};
  for (DeviceBuffer* b : render)
    if (b->ptr) cudaFree(b->ptr);
  if (renderParamsH_) cudaFreeHost(renderParamsH_);
  if (stageH_) cudaFreeHost(stageH_);
}

cudaStream_t Engine::stream() const { return owner_->stream(); }
int Engine::consume() {
  int rc = owner_->consume();
  if (rc) error_ = owner_->error();
  return rc;
}

void Engine::freeAll() {
  DeviceBuffer* all[] = {&pages_, &entries_, &state_, &activity_, &records_, &blockCounts_, &active_, &zeroList_,
                         &freeStack_, &counters_, &curl_, &expn_, &div_, &sb_, &donors_, &solids_,
                         &tileRecD_, &tileNbrD_, &hashD_, &solver_, &tileMask_, &liveTilesD_, &tileIndexD_,
                         &bounds_};
  for (DeviceBuffer* b : all)
    if (b->ptr) {
      cudaFree(b->ptr);
      b->ptr = nullptr;
      b->bytes = 0;
    }
  for (auto& b : vel_) if (b.ptr) { cudaFree(b.ptr); b = DeviceBuffer{}; }
  for (auto& b : fld_) if (b.ptr) { cudaFree(b.ptr); b = DeviceBuffer{}; }
  for (auto& b : smoke_) if (b.ptr) { cudaFree(b.ptr); b = DeviceBuffer{}; }
  for (DeviceBuffer* b : {&smokeBnd_, &meshTablesD_, &meshSourcesD_, &coverageD_})
    if (b->ptr) { cudaFree(b->ptr); *b = DeviceBuffer{}; }
  meshVersion_ = coverageVersion_ = ~0ull;
  for (auto& b : p0_) if (b.ptr) { cudaFree(b.ptr); b = DeviceBuffer{}; }
  for (auto& b : kry_) if (b.ptr) { cudaFree(b.ptr); b = DeviceBuffer{}; }
  for (int l = 0; l < FP_MAX_LEVELS; l++) {
    if (topo_[l].ptr) { cudaFree(topo_[l].ptr); topo_[l] = DeviceBuffer{}; }
    if (lrhs_[l].ptr) { cudaFree(lrhs_[l].ptr); lrhs_[l] = DeviceBuffer{}; }
    for (auto& b : lp_[l]) if (b.ptr) { cudaFree(b.ptr); b = DeviceBuffer{}; }
  }
}

// FluidSimulation.ts:496-549 allocate(): empty pools of the whole voxel budget, no tiles.
int Engine::initialize() {
  int rc;
  if ((rc = check(cudaSetDevice(owner_->device()), "cudaSetDevice"))) return rc;
  freeAll();
  if (!alloc(counters_, sizeof(FpCounters)) || !alloc(solver_, sizeof(FpSolver)) || !alloc(bounds_, sizeof(FpBounds)))
    return FP_ENOMEM;
  lastSolver_ = FpSolver{};
  slots_ = 0;
  capacity_ = 0;
  if ((rc = allocatePools(slotLimit()))) return rc;
  dir_.clear();
  dir_.ground = ground_;
  contentTiles_.clear();
  if ((rc = setCapacity(MIN_TILES))) return rc;
  if ((rc = applyTiles())) return rc;
  solidsStale_ = true;
  geometryDirty_ = true;
  mayHaveFlame_ = false;
  time_ = 0;
  steps_ = 0;
  latest_ = 0;
  activeBricks_ = usedSlots_ = lastFailures_ = 0;
  bricksStepped_ = 0;
  poolLimited_ = false;
  colliderCount_ = 0;
  prevColliders_.clear();
  prevMasks_.clear();
  for (int k = 0; k < 4; k++) velIdx_[k] = k;
  for (int k = 0; k < 3; k++) fldIdx_[k] = k;
  for (int k = 0; k < 3; k++) smokeIdx_[k] = k;
  return check(cudaStreamSynchronize(stream()), "initialize");
}

// Device bytes of a simulation of `g` once its pools exist: per slot the pools and the brick
// levels, per tile slot (at the minimum capacity) the tables and tile levels.
uint64_t Engine::estimateBytes(const fp_grid& g, uint32_t tiles) {
  int B = g.brick_size, vd = g.velocity_divisor > 1 ? g.velocity_divisor : 1, vshift = 0;
  while ((1 << vshift) < B / vd) vshift++;
  uint64_t N = (uint64_t)B * B * B, VN = N / ((uint64_t)vd * vd * vd);
  double budget = g.voxel_budget > 0 ? g.voxel_budget : 8e6;
  uint64_t slots = (uint64_t)std::max(1.0, std::floor(budget / (double)N));
  // FP32 on the velocity lattice: velocity x4 (3 channels), curl, divergence, pressure x2,
  // donors, topology; on the field lattice: expansion, scalar bounds (8), the scalar
  // predictor (4), solid bits; the two scalar state pools (4 channels) and the coarse levels in
  // the precision's width.
  const uint64_t narrow = g.precision == FP_PRECISION_MIXED ? 2 : 4;
  uint64_t perSlot = VN * 4 * (4 * 3 + 4 + 1 + 2) + VN * 3 * 2 + VN + N * 4 * (1 + 8 + 4) +
                     N * 2 * 4 * narrow + N / 8 + 4;
  for (int l = 1; l < vshift; l++) {
    uint64_t c = (uint64_t)1 << (3 * (vshift - l));
    perSlot += c * (3 * narrow + 1);
  }
  if (g.smoke_divisor > 1) {  // coarse smoke: state pair, FP32 predictor, donor range
    uint64_t d = (uint64_t)g.smoke_divisor;
    perSlot += N / (d * d * d) * (2 * narrow + 4 + 8);
  }
  uint64_t perTile = 64 * (4 * 5 + FP_RECORD_WORDS * 4 + 8) + 16 + 27 * 4 + 16 + 8 + 8 + (64 + 8 + 1) * (3 * narrow + 1);
  return slots * perSlot + (uint64_t)std::max(tiles, (uint32_t)MIN_TILES) * perTile + 64 * 1024;
}

// Tile slots for a budget of `budget` voxels in bricks of `cells`: one per four bricks the
// budget holds, a power of two. Sparse tiles (the margins around sources, the ring around
// content) rarely pass a quarter of the bricks, so a simulation reserved this way does not
// grow its tables while it runs.
uint32_t Engine::tilesForBudget(double budget, int cells) {
  double bricks = std::floor((budget > 0 ? budget : 8e6) / (double)cells);
  uint32_t want = (uint32_t)std::min(1.0e6, std::ceil(bricks / 4.0));
  uint32_t tiles = MIN_TILES;
  while (tiles < want) tiles *= 2;
  return tiles;
}

// Tile capacity of at least `tiles` now, so that the steps do not stop to grow it. The
// capacity only sizes storage: tile slots and brick ids do not depend on it.
int Engine::reserveTiles(uint32_t tiles) {
  int rc = consume();
  if (rc) return rc;
  if ((int)tiles <= capacity_) return FP_OK;
  if (tiles > (1u << 24)) return fail(FP_ELIMIT, "tile reservation too large");
  int cap = capacity_;
  while (cap < (int)tiles) cap *= 2;
  if ((rc = setCapacity(cap))) return rc;
  return applyTiles();
}

// Pools of `slots` slots, all free: the stack pops slot 0 first.
int Engine::allocatePools(uint32_t slots) {
  size_t s = slots, N = N_, VN = VN_;  // field and velocity lattice cells a slot
  bool ok = true;
  for (auto& b : vel_) ok = ok && alloc(b, s * 3 * VN * 4);
  // fld_[1] is the predictor within a step (FP32); fld_[0] and fld_[2] trade the state.
  for (int k = 0; k < 3; k++) ok = ok && alloc(fld_[k], s * 4 * N * (k == 1 ? 4 : scalarBytes()));
  ok = ok && alloc(curl_, s * 4 * VN * 4) && alloc(expn_, s * N * 4) && alloc(div_, s * VN * 4) &&
       alloc(sb_, s * 8 * N * 4) &&
       alloc(donors_, s * 3 * VN * 2) && alloc(solids_, s * W_ * 4) && alloc(p0_[0], s * VN * 4) &&
       alloc(p0_[1], s * VN * 4) && alloc(topo_[0], s * VN) && alloc(freeStack_, s * 4);
  for (int l = 1; l < brickLevels_ && ok; l++) {
    size_t c = s * levelCells(l);
    ok = alloc(lp_[l][0], c * coarseBytes()) && alloc(lp_[l][1], c * coarseBytes()) &&
         alloc(lrhs_[l], c * coarseBytes()) && alloc(topo_[l], c);
  }
  // Coarse smoke: the state pair in the scalars' width, the FP32 predictor and donor range.
  if (ok && smokeDiv_ > 1)
    ok = alloc(smoke_[0], s * SN_ * scalarBytes()) && alloc(smoke_[1], s * SN_ * 4) &&
         alloc(smoke_[2], s * SN_ * scalarBytes()) && alloc(smokeBnd_, s * 2 * SN_ * 4);
  if (!ok) return FP_ENOMEM;
  if (schedule_.krylov) {
    int rc = krylovPools(slots);
    if (rc) return rc;
  }
  std::vector<uint32_t> stack(slots);
  for (uint32_t i = 0; i < slots; i++) stack[i] = slots - 1 - i;
  cudaMemcpy(freeStack_.ptr, stack.data(), s * 4, cudaMemcpyHostToDevice);
  FpCounters c{};
  c.freeCount = (int32_t)slots;
  cudaMemcpy(counters_.ptr, &c, sizeof(c), cudaMemcpyHostToDevice);
  slots_ = slots;
  return FP_OK;
}

// After the budget rose: new slots go under the free stack (fluid-pool-growth.wgsl:12-21),
// live pools keep their contents.
int Engine::growPool(uint32_t target) {
  if (target <= slots_) return FP_OK;
  cudaStreamSynchronize(stream());
  size_t s = target, N = N_, VN = VN_;
  uint32_t added = target - slots_;
  bool ok = true;
  for (auto& b : vel_) ok = ok && grow(b, s * 3 * VN * 4, 0);
  for (int k = 0; k < 3; k++) ok = ok && grow(fld_[k], s * 4 * N * (k == 1 ? 4 : scalarBytes()), 0);
  ok = ok && grow(curl_, s * 4 * VN * 4, 0) && grow(expn_, s * N * 4, 0) && grow(div_, s * VN * 4, 0) &&
       grow(sb_, s * 8 * N * 4, 0) &&
       grow(donors_, s * 3 * VN * 2, 0) && grow(solids_, s * W_ * 4, 0) && grow(p0_[0], s * VN * 4, 0) &&
       grow(p0_[1], s * VN * 4, 0) && grow(topo_[0], s * VN, 0);
  for (int l = 1; l < brickLevels_ && ok; l++) {
    size_t c = s * levelCells(l);
    ok = grow(lp_[l][0], c * coarseBytes(), 0) && grow(lp_[l][1], c * coarseBytes(), 0) &&
         grow(lrhs_[l], c * coarseBytes(), 0) && grow(topo_[l], c, 0);
  }
  if (ok && smokeDiv_ > 1)
    for (int k = 0; k < 3; k++) ok = ok && grow(smoke_[k], s * SN_ * (k == 1 ? 4 : scalarBytes()), 0);
  if (ok && smokeDiv_ > 1) ok = grow(smokeBnd_, s * 2 * SN_ * 4, 0);
  if (!ok) return FP_ENOMEM;
  if (schedule_.krylov) {
    int rc = krylovPools(target);
    if (rc) return rc;
  }
  std::vector<uint32_t> old(slots_);
  cudaMemcpy(old.data(), freeStack_.ptr, (size_t)slots_ * 4, cudaMemcpyDeviceToHost);
  std::vector<uint32_t> next(target);
  for (uint32_t i = 0; i < added; i++) next[i] = slots_ + added - 1 - i;
  for (uint32_t i = 0; i < slots_; i++) next[added + i] = old[i];
  if (!alloc(freeStack_, s * 4, false)) return FP_ENOMEM;
  cudaMemcpy(freeStack_.ptr, next.data(), s * 4, cudaMemcpyHostToDevice);
  FpCounters c;
  cudaMemcpy(&c, counters_.ptr, sizeof(c), cudaMemcpyDeviceToHost);
  c.freeCount += (int32_t)added;
  cudaMemcpy(counters_.ptr, &c, sizeof(c), cudaMemcpyHostToDevice);
  slots_ = target;
  geometryDirty_ = true;
  return FP_OK;
}

// Per-brick and per-tile storage for `capacity` tile slots, keeping every brick's page,
// state, flags, entry and record (FluidSimulation.ts:633-646).
int Engine::setCapacity(int capacity) {
  cudaStreamSynchronize(stream());
  size_t bricks = (size_t)capacity * 64;
  size_t oldBricks = (size_t)capacity_ * 64;
  bool ok = grow(pages_, bricks * 4, 0xff) && grow(entries_, bricks * 4, 0xff) && grow(state_, bricks * 4, 0) &&
            grow(records_, bricks * FP_RECORD_WORDS * 4, 0xff) && alloc(active_, bricks * 4) &&
            alloc(zeroList_, bricks * 8) && alloc(blockCounts_, (bricks / 256 + 1) * 16) &&
            alloc(tileMask_, (size_t)capacity * 8);
  if (!ok) return FP_ENOMEM;
  // activity: bricks, then a word per tile slot.
  {
    DeviceBuffer next;
    if (!alloc(next, (bricks + capacity) * 4)) return FP_ENOMEM;
    if (activity_.ptr) {
      cudaMemcpyAsync(next.ptr, activity_.ptr, oldBricks * 4, cudaMemcpyDeviceToDevice, stream());
      cudaStreamSynchronize(stream());
      cudaFree(activity_.ptr);
    }
    activity_ = next;
  }
  for (int l = brickLevels_; l <= bottom_; l++) {
    size_t c = (size_t)capacity * levelCells(l);
    ok = ok && grow(lp_[l][0], c * coarseBytes(), 0) && grow(lp_[l][1], c * coarseBytes(), 0) &&
         grow(lrhs_[l], c * coarseBytes(), 0) && grow(topo_[l], c, 0);
  }
  if (!ok) return FP_ENOMEM;
  capacity_ = capacity;
  return FP_OK;
}

// applyTiles (FluidSimulation.ts:629-678) with TileDirectory.tables (TileDirectory.ts:151-186).
int Engine::applyTiles() {
  tileVersion_++;
  int needed = std::max(MIN_TILES, dir_.slotsUsed());
  if (needed > capacity_) {
    int cap = capacity_;
    while (cap < needed) cap *= 2;
    int rc = setCapacity(cap);
    if (rc) return rc;
  }
  tileRec_.assign(capacity_, make_int4(0, 0, 0, 0));
  tileNbr_.assign((size_t)capacity_ * 27, -1);
  int size = HASH_ROW;
  while (size < dir_.count() * 2) size *= 2;
  hash_.assign(size, make_int4(-1, -1, -1, -1));
  const auto& slots = dir_.slots();
  for (size_t s = 0; s < slots.size(); s++) {
    const TileDirectory::Tile& t = slots[s];
    if (!t.alive) continue;
    tileRec_[s] = make_int4(t.x, t.y, t.z, t.closing ? 2 : 1);
    uint32_t hsh = (((uint32_t)t.x * 73856093u) ^ ((uint32_t)t.y * 19349663u) ^ ((uint32_t)t.z * 83492791u)) & (size - 1);
    while (hash_[hsh].w >= 0) hsh = (hsh + 1) & (size - 1);
    hash_[hsh] = make_int4(t.x, t.y, t.z, (int)s);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++)
          tileNbr_[s * 27 + (dz + 1) * 9 + (dy + 1) * 3 + dx + 1] = dir_.slotAt(t.x + dx, t.y + dy, t.z + dz);
  }
  // The live slots in ascending order and each slot's position among them: the tile levels of
  // the multigrid walk only these.
  liveTiles_.clear();
  tileIndex_.assign(capacity_, -1);
  for (int s = 0; s < capacity_; s++)
    if (tileRec_[s].w != 0) {
      tileIndex_[s] = (int)liveTiles_.size();
      liveTiles_.push_back(s);
    }
  if (!upload(tileRecD_, tileRec_.data(), tileRec_.size() * sizeof(int4)) ||
      !upload(tileNbrD_, tileNbr_.data(), tileNbr_.size() * 4) || !upload(hashD_, hash_.data(), hash_.size() * sizeof(int4)) ||
      !upload(liveTilesD_, liveTiles_.data(), liveTiles_.size() * 4) ||
      !upload(tileIndexD_, tileIndex_.data(), tileIndex_.size() * 4))
    return FP_ENOMEM;
  // New tiles' bricks start without slots.
  for (int slot : dir_.takeCreated()) {
    size_t off = (size_t)slot * 64 * 4;
    cudaMemsetAsync((char*)pages_.ptr + off, 0xff, 64 * 4, stream());
    cudaMemsetAsync((char*)entries_.ptr + off, 0xff, 64 * 4, stream());
    cudaMemsetAsync((char*)state_.ptr + off, 0, 64 * 4, stream());
    cudaMemsetAsync((char*)activity_.ptr + off, 0, 64 * 4, stream());
  }
  buildClusters();
  dir_.dirty = false;
  geometryDirty_ = true;  // PressureSolver.setBricks -> resetPlans
  return FP_OK;
}

// updateTiles (FluidSimulation.ts:873-912).
void Engine::updateTiles(const fp_frame& f) {
  dir_.retire(steps_);
  // Host arithmetic in double precision, as the reference's JavaScript does it.
  double h = h_, tile = (double)(TILE_BRICKS * B_) * h;
  double margin = (double)(2 * B_) * h + tile;
  double brick = (double)B_ * h;
  sourceBoxes_.clear();
  for (uint32_t i = 0; i < f.source_count; i++) {
    const fp_source& s = f.sources[i];
    if (s.shape == FP_SHAPE_MESH) {
      // A mesh source's samples span [position, size]; a voxel more margin
      // (FluidSimulation.ts:879-893).
      double m = margin + h;
      int lo[3], hi[3];
      for (int a = 0; a < 3; a++) {
        lo[a] = (int)std::floor(((double)s.position[a] - m) / tile);
        hi[a] = (int)std::floor(((double)s.size[a] + m) / tile);
      }
      dir_.need(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], steps_);
      for (int a = 0; a < 3; a++) sourceBoxes_.push_back((int)std::floor((double)s.position[a] / brick));
      for (int a = 0; a < 3; a++) sourceBoxes_.push_back((int)std::floor((double)s.size[a] / brick));
      continue;
    }
    double ext = std::max(std::max(std::max((double)s.size[0], (double)s.size[1]), (double)s.size[2]), 0.03) +
                 (double)s.outward_speed * 0.25;
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = (int)std::floor(((double)s.position[a] - ext - margin) / tile);
      hi[a] = (int)std::floor(((double)s.position[a] + ext + margin) / tile);
    }
    dir_.need(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], steps_);
    // bricksOver (FluidSimulation.ts:862-868): the source's bricks, for the render box.
    for (int a = 0; a < 3; a++) sourceBoxes_.push_back((int)std::floor(((double)s.position[a] - ext) / brick));
    for (int a = 0; a < 3; a++) sourceBoxes_.push_back((int)std::floor(((double)s.position[a] + ext) / brick));
  }
  for (auto& ct : contentTiles_)
    dir_.need(ct.first.x - 1, ct.first.y - 1, ct.first.z - 1, ct.first.x + 1, ct.first.y + 1, ct.first.z + 1, steps_);
}

// packFlameStep (flame.ts:43-87): validate before any state changes.
int Engine::packFlame(const fp_combustion& c, float dt, FpFlame& out) {
  auto finite = [](float v) { return std::isfinite(v); };
  if (!finite(dt)) return fail(FP_EINVAL, "Flame timestep must be finite in f32.");
  if (!finite(c.lifespan)) return fail(FP_EINVAL, "Flame lifespan must be finite in f32.");
  if (dt <= 0 || c.lifespan <= 0) return fail(FP_EINVAL, "Flame timestep and lifespan must be positive in f32.");
  if (!finite(dt / c.lifespan)) return fail(FP_EINVAL, "Lifetime decrement must be finite in f32.");
  if (!finite(c.smoke_rate)) return fail(FP_EINVAL, "Smoke rate must be finite in f32.");
  if (!finite(c.heat_rate)) return fail(FP_EINVAL, "Heat rate must be finite in f32.");
  if (!finite(c.expansion_rate)) return fail(FP_EINVAL, "Expansion rate must be finite in f32.");
  if (c.smoke_rate < 0 || c.heat_rate < 0) return fail(FP_EINVAL, "Smoke and heat rates must be nonnegative.");
  for (float r : {c.smoke_rate, c.heat_rate, c.expansion_rate})
    if (!finite(r * c.lifespan)) return fail(FP_EINVAL, "Integrated flame output must be finite in f32.");
  const char* names[3] = {"smoke", "heat", "expansion"};
  FpFlame F{};
  F.dt = dt;
  F.lifespan = c.lifespan;
  F.smoke = c.smoke_rate;
  F.heat = c.heat_rate;
  F.expansion = c.expansion_rate;
  for (int ch = 0; ch < 3; ch++) {
    const fp_flame_ramp& r = c.ramps[ch];
    if (r.count < 2 || r.count > 8) return fail(FP_EINVAL, std::string(names[ch]) + " ramp needs 2–8 knots.");
    float prev = -1;
    for (uint32_t i = 0; i < r.count; i++) {
      float x = r.knots[i][0], y = r.knots[i][1];
      if (!finite(x)) return fail(FP_EINVAL, std::string(names[ch]) + " lifetime must be finite in f32.");
      if (!finite(y)) return fail(FP_EINVAL, std::string(names[ch]) + " response must be finite in f32.");
      if (x < 0 || x > 1 || y < 0 || y > 1 || x <= prev)
        return fail(FP_EINVAL, std::string(names[ch]) + " knots must increase in f32 with coordinates in [0,1].");
      if ((i == 0 && x != 0) || (i == r.count - 1 && x != 1))
        return fail(FP_EINVAL, std::string(names[ch]) + " ramp must span lifetime 0–1.");
      F.knots[ch][i][0] = x;
      F.knots[ch][i][1] = y;
      prev = x;
    }
    F.counts[ch] = (int)r.count;
  }
  out = F;
  return FP_OK;
}

// Every tile within the world box (FluidSimulation.ts:1163-1188); all tiles without one.
void Engine::bin(int kind, int index, const double* lo, const double* hi, std::vector<std::vector<uint32_t>>& lists) {
  const auto& slots = dir_.slots();
  if (!lo) {
    for (size_t s = 0; s < slots.size(); s++)
      if (slots[s].alive) lists[(size_t)s * 3 + kind].push_back((uint32_t)index);
    return;
  }
  double tile = (double)(TILE_BRICKS * B_) * (double)h_;
  int l[3], u[3];
  for (int a = 0; a < 3; a++) {
    l[a] = (int)std::floor(lo[a] / tile);
    u[a] = (int)std::floor(hi[a] / tile);
  }
  long span = 1;
  for (int a = 0; a < 3; a++) span *= std::max(0, u[a] - l[a] + 1);
  if (span > dir_.count()) {
    for (size_t s = 0; s < slots.size(); s++) {
      const auto& t = slots[s];
      if (t.alive && t.x >= l[0] && t.x <= u[0] && t.y >= l[1] && t.y <= u[1] && t.z >= l[2] && t.z <= u[2])
        lists[s * 3 + kind].push_back((uint32_t)index);
    }
    return;
  }
  for (int z = l[2]; z <= u[2]; z++)
    for (int y = l[1]; y <= u[1]; y++)
      for (int x = l[0]; x <= u[0]; x++) {
        int s = dir_.slotAt(x, y, z);
        if (s >= 0) lists[(size_t)s * 3 + kind].push_back((uint32_t)index);
      }
}

// packScene (FluidSimulation.ts:1150-1366) and ForceFields.prepare (ForceFields.ts:41-114).
// Returns whether the colliders changed.
bool Engine::packScene(const fp_frame& f) {
  std::vector<std::vector<uint32_t>> lists((size_t)capacity_ * 3);
  // Reach boxes in double precision, as the reference's JavaScript computes them.
  double brick = (double)B_ * (double)h_;
  emitters_.clear();
  for (uint32_t i = 0; i < f.source_count; i++) {
    const fp_source& s = f.sources[i];
    if (s.shape == FP_SHAPE_MESH) continue;
    FpEmitter e{};
    for (int a = 0; a < 3; a++) {
      e.pos[a] = s.position[a];
      e.size[a] = s.size[a];
      e.vel[a] = s.velocity[a];
    }
    e.enabled = 1.f;
    e.box = s.shape == FP_SHAPE_BOX ? 1.f : 0.f;
    e.flame = s.flame;
    e.heat = s.heat_rate;
    e.smoke = s.smoke_rate;
    e.response = s.velocity_response;
    e.outward = s.outward_speed;
    e.period = s.has_variation ? s.variation_period : 0.5f;
    e.strength = s.has_variation ? s.variation_strength : 0.f;
    e.fuel = s.fuel_rate;
    int index = (int)emitters_.size();
    emitters_.push_back(e);
    double lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      double ext = std::max((double)s.size[a], 0.03);
      lo[a] = (double)s.position[a] - ext - 2 * brick;
      hi[a] = (double)s.position[a] + ext + 2 * brick;
    }
    bin(0, index, lo, hi, lists);
  }
  colliders_.clear();
  masks_.assign(f.collider_masks, f.collider_masks + f.collider_mask_words);
  for (uint32_t i = 0; i < f.collider_count; i++) {
    const fp_collider& c = f.colliders[i];
    FpCollider k{};
    double lo[3], hi[3];
    if (c.shape == FP_SHAPE_MESH) {
      k.kind = 2.f;
      for (int a = 0; a < 3; a++) {
        k.lo[a] = c.lo[a];
        k.size[a] = c.dims[a];
        lo[a] = (double)c.lo[a] * (double)h_;
        hi[a] = (double)(c.lo[a] + c.dims[a]) * (double)h_;
      }
      k.first = (int)c.mask_offset;
    } else {
      k.kind = c.shape == FP_SHAPE_BOX ? 1.f : 0.f;
      for (int a = 0; a < 3; a++) {
        k.center[a] = c.position[a];
        k.extent[a] = c.size[a];
        for (int b = 0; b < 3; b++) k.axes[a][b] = c.axes[a][b];
      }
      for (int a = 0; a < 3; a++) {
        double ext = c.size[a];
        if (c.shape == FP_SHAPE_BOX)
          ext = std::fabs((double)c.axes[0][a]) * (double)c.size[0] + std::fabs((double)c.axes[1][a]) * (double)c.size[1] +
                std::fabs((double)c.axes[2][a]) * (double)c.size[2];
        lo[a] = (double)c.position[a] - ext;
        hi[a] = (double)c.position[a] + ext;
      }
    }
    colliders_.push_back(k);
    bin(2, (int)i, lo, hi, lists);
  }
  std::vector<uint8_t> packed(colliders_.size() * sizeof(FpCollider));
  if (!packed.empty()) std::memcpy(packed.data(), colliders_.data(), packed.size());
  bool changed = packed != prevColliders_ || masks_ != prevMasks_;
  prevColliders_.swap(packed);
  prevMasks_ = masks_;
  colliderCount_ = (int)colliders_.size();
  forces_.clear();
  regions_.clear();
  for (uint32_t i = 0; i < f.force_count; i++) {
    const fp_force& s = f.forces[i];
    FpForce k{};
    for (int a = 0; a < 3; a++) {
      k.axis[a] = s.vector[a];
      k.center[a] = s.center[a];
    }
    k.strength = s.strength;
    k.kind = (float)s.type;
    k.scale = s.scale;
    k.lift = s.lift;
    k.inward = s.inward;
    k.targeted = s.targeted ? 1.f : 0.f;
    k.regionFirst = (float)regions_.size();
    bool has = false;
    double lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
    int count = 0;
    if (s.targeted) {
      for (uint32_t t = 0; t < s.target_count && s.first_target + t < f.force_target_count; t++) {
        const fp_source& src = f.force_targets[s.first_target + t];
        if (src.shape == FP_SHAPE_MESH) {
          // Mesh targets cover the cells their samples reach (coverage below); the reach
          // grows by their samples' bounds, a velocity cell more (ForceFields.ts:97-107).
          k.hasMesh = 1.f;
          if (!f.target_cell_ranges || f.target_cell_ranges[2 * (s.first_target + t) + 1] == 0) continue;
          for (int a = 0; a < 3; a++) {
            const double vh = (double)h_ * vd_;  // a velocity cell
            double l = (double)src.position[a] - vh, u = (double)src.size[a] + vh;
            lo[a] = has ? std::min(lo[a], l) : l;
            hi[a] = has ? std::max(hi[a], u) : u;
          }
          has = true;
          continue;
        }
        FpRegion r{};
        for (int a = 0; a < 3; a++) {
          r.center[a] = src.position[a];
          r.size[a] = src.size[a];
        }
        r.box = src.shape == FP_SHAPE_BOX ? 3.f : 1.f;
        regions_.push_back(r);
        count++;
        for (int a = 0; a < 3; a++) {
          double ext = std::max((double)src.size[a], 0.03);
          double l = (double)src.position[a] - ext, u = (double)src.position[a] + ext;
          lo[a] = has ? std::min(lo[a], l) : l;
          hi[a] = has ? std::max(hi[a], u) : u;
        }
        has = true;
      }
    }
    k.regionCount = (float)count;
    forces_.push_back(k);
    if (!s.targeted) {
      bin(1, (int)i, nullptr, nullptr, lists);
    } else {
      double l[3], u[3];
      for (int a = 0; a < 3; a++) {
        l[a] = lo[a] - brick;
        u[a] = hi[a] + brick;
      }
      bin(1, (int)i, l, u, lists);
    }
  }
  // Mesh targets' coverage (ForceFields.ts:115-179): per brick id its first entry (or none),
  // then per covered brick a count and, per force covering it, the force's index and a bit
  // per velocity cell; rebuilt when the targets or the tiles change.
  std::vector<int32_t> targets;  // force index, cell count, cells, ... of the mesh targets
  for (uint32_t i = 0; i < f.force_count; i++) {
    const fp_force& s = f.forces[i];
    if (!s.targeted || !f.target_cell_ranges) continue;
    for (uint32_t t = 0; t < s.target_count && s.first_target + t < f.force_target_count; t++) {
      uint32_t ti = s.first_target + t;
      if (f.force_targets[ti].shape != FP_SHAPE_MESH || f.target_cell_ranges[2 * ti + 1] == 0) continue;
      uint32_t first = f.target_cell_ranges[2 * ti], n = f.target_cell_ranges[2 * ti + 1];
      targets.push_back((int32_t)i);
      targets.push_back((int32_t)n);
      targets.insert(targets.end(), f.target_cells + 3 * (size_t)first, f.target_cells + 3 * ((size_t)first + n));
    }
  }
  coverageOn_ = !targets.empty();
  if (coverageOn_ && (targets != coverageTargets_ || coverageVersion_ != tileVersion_)) {
    coverageTargets_ = targets;
    coverageVersion_ = tileVersion_;
    // Velocity cells: the coverage lives on the velocity lattice (force-fields.wgsl:27-47).
    const size_t bricks = (size_t)capacity_ * 64, words = 1 + (size_t)(VN_ + 31) / 32;
    const int mask = VB_ - 1;
    std::map<int, std::map<int, std::vector<uint32_t>>> entries;  // brick id -> force -> bits
    std::vector<int> order;                                        // brick ids, first seen first
    for (size_t p = 0; p < targets.size();) {
      int index = targets[p], n = targets[p + 1];
      const int32_t* cells = &targets[p + 2];
      for (int c = 0; c < n; c++) {
        const int32_t* cell = cells + 3 * c;
        int b[3] = {cell[0] >> vshift_, cell[1] >> vshift_, cell[2] >> vshift_};
        int slot = dir_.slotAt(b[0] >> 2, b[1] >> 2, b[2] >> 2);
        if (slot < 0) continue;
        int id = slot * 64 + (((b[2] & 3) * 4 + (b[1] & 3)) * 4 + (b[0] & 3));
        auto& forcesOf = entries[id];
        if (forcesOf.empty()) order.push_back(id);
        auto& bits = forcesOf[index];
        if (bits.empty()) bits.assign(words - 1, 0u);
        int bit = (((cell[2] & mask) * VB_) + (cell[1] & mask)) * VB_ + (cell[0] & mask);
        bits[bit >> 5] |= 1u << (bit & 31);
      }
      p += 2 + 3 * (size_t)n;
    }
    coverage_.assign(bricks, 0xffffffffu);
    for (int id : order) {
      coverage_[id] = (uint32_t)coverage_.size();
      coverage_.push_back((uint32_t)entries[id].size());
      for (auto& fb : entries[id]) {
        coverage_.push_back((uint32_t)fb.first);
        coverage_.insert(coverage_.end(), fb.second.begin(), fb.second.end());
      }
    }
    if (!upload(coverageD_, coverage_.data(), coverage_.size() * 4)) sceneUploadFailed_ = true;
  }
  // What reaches each tile: an 8-word header per tile slot, then the indices.
  size_t length = (size_t)capacity_ * 8;
  for (auto& l : lists) length += l.size();
  tileLists_.assign(length, 0);
  size_t next = (size_t)capacity_ * 8;
  for (int s = 0; s < capacity_; s++)
    for (int k = 0; k < 3; k++) {
      auto& l = lists[(size_t)s * 3 + k];
      tileLists_[(size_t)s * 8 + 2 * k] = (uint32_t)next;
      tileLists_[(size_t)s * 8 + 2 * k + 1] = (uint32_t)l.size();
      std::copy(l.begin(), l.end(), tileLists_.begin() + next);
      next += l.size();
    }
  // Mesh emission (FluidSimulation.ts:1318-1351): the records, record 0 being none, and each
  // brick's table of them (its cells' record indices), rebuilt when the records or the tiles
  // change.
  meshCount_ = (int)f.mesh_source_count;
  if (meshCount_ > 0) {
    static_assert(sizeof(FpMeshSource) == sizeof(fp_mesh_source), "mesh record layout");
    bool same = meshVersion_ == tileVersion_ && meshRecords_.size() == (size_t)meshCount_ + 1 &&
                std::memcmp(meshRecords_.data() + 1, f.mesh_sources, (size_t)meshCount_ * sizeof(FpMeshSource)) == 0;
    if (!same) {
      meshRecords_.assign(1, FpMeshSource{});
      const FpMeshSource* in = reinterpret_cast<const FpMeshSource*>(f.mesh_sources);
      meshRecords_.insert(meshRecords_.end(), in, in + meshCount_);
      const size_t bricks = (size_t)capacity_ * 64;
      const int mask = B_ - 1;
      std::unordered_map<int, int> tables;
      std::vector<std::pair<size_t, int>> placed;
      for (int r = 1; r <= meshCount_; r++) {
        const int* cell = meshRecords_[r].cell;
        int b[3] = {cell[0] >> shift_, cell[1] >> shift_, cell[2] >> shift_};
        int slot = dir_.slotAt(b[0] >> 2, b[1] >> 2, b[2] >> 2);
        if (slot < 0) continue;
        int id = slot * 64 + (((b[2] & 3) * 4 + (b[1] & 3)) * 4 + (b[0] & 3));
        int table = tables.emplace(id, (int)tables.size()).first->second;
        size_t index = (((((size_t)table << shift_) | (size_t)(cell[2] & mask)) << shift_ | (size_t)(cell[1] & mask))
                        << shift_) | (size_t)(cell[0] & mask);
        placed.push_back({index, r});
      }
      meshTables_.assign(bricks + tables.size() * (size_t)N_, 0);
      std::fill(meshTables_.begin(), meshTables_.begin() + bricks, -1);
      for (auto& t : tables) meshTables_[t.first] = t.second;
      for (auto& p : placed) meshTables_[bricks + p.first] = p.second;
      meshVersion_ = tileVersion_;
      if (!upload(meshTablesD_, meshTables_.data(), meshTables_.size() * 4) ||
          !upload(meshSourcesD_, meshRecords_.data(), meshRecords_.size() * sizeof(FpMeshSource))) {
        sceneUploadFailed_ = true;
        meshVersion_ = ~0ull;
      }
    }
  }
  return changed;
}

// Checks of fp_sim_step before any state changes (FluidSimulation.ts:1367-1369).
int Engine::validate(const fp_frame& f, float dt) {
  if (!std::isfinite(dt) || dt <= 0 || dt > 1.f / 30.f)
    return fail(FP_EINVAL, "Simulation step must be in (0, 1/30]. Use fixed substeps.");
  FpFlame F;
  int rc = packFlame(f.combustion, dt, F);
  if (rc) return rc;
  for (uint32_t i = 0; i < f.collider_count; i++) {
    const fp_collider& c = f.colliders[i];
    if (c.shape == FP_SHAPE_MESH) {
      uint64_t bits = (uint64_t)std::max(0, c.dims[0]) * std::max(0, c.dims[1]) * std::max(0, c.dims[2]);
      if ((uint64_t)c.mask_offset + (bits + 31) / 32 > f.collider_mask_words)
        return fail(FP_EINVAL, "Mesh collider occupancy does not match its size.");
    }
  }
  if (f.target_cell_ranges)
    for (uint32_t t = 0; t < f.force_target_count; t++)
      if (f.force_targets[t].shape == FP_SHAPE_MESH &&
          (uint64_t)f.target_cell_ranges[2 * t] + f.target_cell_ranges[2 * t + 1] > f.target_cell_count)
        return fail(FP_EINVAL, "Mesh force target cells lie outside target_cells.");
  return FP_OK;
}

// The host half of substep (FluidSimulation.ts:1367-1440): grow the pool to the budget,
// update the tiles, pack the scene. The measurement of the previous step was applied.
int Engine::prepare(const fp_frame& f, float dt) {
  int rc = packFlame(f.combustion, dt, flame_);
  if (rc) return rc;
  if (dir_.ground != ground_) {
    dir_.ground = ground_;
    geometryDirty_ = true;
  }
  uint32_t limit = slotLimit();
  if (limit > slots_ && (rc = growPool(limit))) return rc;
  updateTiles(f);
  if (dir_.dirty && (rc = applyTiles())) return rc;
  updateRenderBox();
  sceneUploadFailed_ = false;
  if (packScene(f)) {
    solidsStale_ = true;
    geometryDirty_ = true;
  }
  if (sceneUploadFailed_) {
    coverageVersion_ = ~0ull;  // built again by the next step
    return fail(FP_ENOMEM, "device memory exhausted (mesh emission or force coverage tables)");
  }
  mayHaveFlame_ = mayHaveFlame_ || f.fuel.enabled;
  for (uint32_t i = 0; i < f.source_count; i++) mayHaveFlame_ = mayHaveFlame_ || f.sources[i].flame > 0;
  return FP_OK;
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

size_t Engine::sceneBytes() const {
  return align256(emitters_.size() * sizeof(FpEmitter)) + align256(colliders_.size() * sizeof(FpCollider)) +
         align256(masks_.size() * 4) + align256(forces_.size() * sizeof(FpForce)) +
         align256(regions_.size() * sizeof(FpRegion)) + align256(tileLists_.size() * 4) +
         (vd_ > 1 ? align256(sizeof(SimParams)) : 0);  // the velocity view
}

void Engine::writeStep(SimParams& P, uint8_t* hostBase, uint8_t* devBase, size_t off, const fp_frame& f, float dt,
                       uint32_t* readback, const float4* noise) {
  // The scene blobs, each 256-byte aligned, into the launch's upload.
  auto put = [&](const void* src, size_t bytes) -> const void* {
    if (bytes) std::memcpy(hostBase + off, src, bytes);
    const void* d = devBase + off;
    off += align256(bytes);
    return d;
  };
  std::memset(&P, 0, sizeof(P));
  P.emitters = (const FpEmitter*)put(emitters_.data(), emitters_.size() * sizeof(FpEmitter));
  P.colliders = (const FpCollider*)put(colliders_.data(), colliders_.size() * sizeof(FpCollider));
  P.masks = (const uint32_t*)put(masks_.data(), masks_.size() * 4);
  P.forces = (const FpForce*)put(forces_.data(), forces_.size() * sizeof(FpForce));
  P.regions = (const FpRegion*)put(regions_.data(), regions_.size() * sizeof(FpRegion));
  P.tileLists = (const uint32_t*)put(tileLists_.data(), tileLists_.size() * 4);
  P.buildSolids = buildSolids() ? 1 : 0;
  P.topoAll = topoAll() ? 1 : 0;
  P.curlOn = f.simulation.vorticity != 0.f ? 1 : 0;
  P.readback = readback;
  P.B = B_;
  P.shift = shift_;
  P.N = N_;
  P.W = W_;
  P.brickLevels = brickLevels_;
  P.bottom = bottom_;
  P.h = h_;
  P.invH = 1.f / h_;
  P.dt = dt;
  P.buoyancy = f.simulation.buoyancy;
  P.cooling = f.simulation.cooling;
  P.smokeWeight = f.simulation.smoke_weight;
  P.damping = f.simulation.velocity_damping;
  P.dissipation = f.simulation.dissipation;
  P.vorticity = f.simulation.vorticity;
  P.cutoff = cutoff_;
  P.time = (float)time_;
  P.seedF = (float)f.simulation.seed;
  std::memcpy(&P.seedBits, &P.seedF, 4);
  P.lifetimeZero = mayHaveFlame_ ? 0 : 1;
  P.fuelEnabled = f.fuel.enabled ? 1 : 0;
  P.ignition = f.fuel.ignition_heat;
  P.burnRate = f.fuel.burn_rate;
  P.ground = ground_ ? 1 : 0;
  P.colliderCount = colliderCount_;
  P.maccormack = maccormack_ ? 1 : 0;
  P.solidsAll = solidsStale_ ? 1 : 0;
  P.held = (int)std::max<int64_t>(0, (int64_t)slots_ - (int64_t)slotLimit());
  P.slots = slots_;
  P.capacity = capacity_;
  P.tileRec = (const int4*)tileRecD_.ptr;
  P.tileNbr = (const int*)tileNbrD_.ptr;
  P.tileMask = (uint64_t*)tileMask_.ptr;
  P.liveTiles = (const int*)liveTilesD_.ptr;
  P.tileIndex = (const int*)tileIndexD_.ptr;
  P.liveCount = (int)liveTiles_.size();
  P.hash = (const int4*)hashD_.ptr;
  P.hashMask = (uint32_t)hash_.size() - 1;
  P.pages = (int*)pages_.ptr;
  P.entries = (int*)entries_.ptr;
  P.state = (uint32_t*)state_.ptr;
  P.activity = (uint32_t*)activity_.ptr;
  P.records = (int*)records_.ptr;
  P.blockCounts = (uint32_t*)blockCounts_.ptr;
  P.active = (uint32_t*)active_.ptr;
  P.zeroList = (uint32_t*)zeroList_.ptr;
  P.freeStack = (uint32_t*)freeStack_.ptr;
  P.counters = (FpCounters*)counters_.ptr;
  P.vel = (float*)vel_[velIdx_[0]].ptr;
  P.velP = (float*)vel_[velIdx_[1]].ptr;
  P.velC = (float*)vel_[velIdx_[2]].ptr;
  P.velF = (float*)vel_[velIdx_[3]].ptr;
  P.curl = (float*)curl_.ptr;
  P.fld = (float*)fld_[fldIdx_[0]].ptr;
  P.fldP = (float*)fld_[fldIdx_[1]].ptr;
  P.fldN = (float*)fld_[fldIdx_[2]].ptr;
  P.expn = (float*)expn_.ptr;
  P.div = (float*)div_.ptr;
  P.sb = (float*)sb_.ptr;
  P.smokeDiv = smokeDiv_;
  P.smokeShift = sshift_;
  P.smokeCells = SN_;
  P.smk = (float*)smoke_[smokeIdx_[0]].ptr;
  P.smkP = (float*)smoke_[smokeIdx_[1]].ptr;
  P.smkN = (float*)smoke_[smokeIdx_[2]].ptr;
  P.smkB = (float*)smokeBnd_.ptr;
  P.meshCount = meshCount_;
  P.meshTables = (const int*)meshTablesD_.ptr;
  P.meshSources = (const FpMeshSource*)meshSourcesD_.ptr;
  P.forceCoverage = coverageOn_ ? (const uint32_t*)coverageD_.ptr : nullptr;
  P.donors = (uint16_t*)donors_.ptr;
  P.solids = (uint32_t*)solids_.ptr;
  P.p0[0] = (float*)p0_[0].ptr;
  P.p0[1] = (float*)p0_[1].ptr;
  P.p0[2] = (float*)p0_[2].ptr;
  for (int k = 0; k < 3; k++) P.kry[k] = (float*)kry_[k].ptr;
  P.latest = latest_;
  P.scalarHalf = precision_ == FP_PRECISION_MIXED ? 1 : 0;
  P.coarseBf16 = precision_ == FP_PRECISION_MIXED ? 1 : 0;
  P.vcycles = vcycles_;
  P.tolerance = tolerance_;
  P.solver = (FpSolver*)solver_.ptr;
  P.bounds = (FpBounds*)bounds_.ptr;
  for (int l = 0; l <= bottom_; l++) {
    P.topo[l] = (uint8_t*)topo_[l].ptr;
    if (l > 0) {
      P.lp[l][0] = (float*)lp_[l][0].ptr;
      P.lp[l][1] = (float*)lp_[l][1].ptr;
      P.lrhs[l] = (float*)lrhs_[l].ptr;
    }
  }
  P.flame = flame_;
  P.noise = noise;
  // The lattice views: this SimParams is the field view, and the velocity view too when d = 1;
  // with d > 1 the velocity view follows the scene, alike but for its lattice.
  P.velDiv = vd_;
  P.solidSpan = 1;
  P.fshift = shift_;
  P.fineH = h_;
  const SimParams* self = reinterpret_cast<const SimParams*>(devBase + (reinterpret_cast<uint8_t*>(&P) - hostBase));
  P.fview = self;
  P.vview = self;
  if (vd_ > 1) {
    SimParams* V = reinterpret_cast<SimParams*>(hostBase + off);
    P.vview = reinterpret_cast<const SimParams*>(devBase + off);
    off += align256(sizeof(SimParams));
    *V = P;
    V->B = VB_;
    V->shift = vshift_;
    V->N = VN_;
    V->h = h_ * (float)vd_;
    V->invH = 1.f / V->h;
    V->solidSpan = vd_;
  }
  stepH2d_ = h2d_ + sizeof(SimParams) + sceneBytes();
  stepD2h_ = readbackWords() * 4;
  h2d_ = 0;
}

void Engine::launched(float dt, int latest) {
  solidsStale_ = false;
  geometryDirty_ = false;
  latest_ = latest;
  std::swap(velIdx_[0], velIdx_[1]);
  std::swap(fldIdx_[0], fldIdx_[2]);
  std::swap(smokeIdx_[0], smokeIdx_[2]);
  stageUsed_ = 0;
  time_ += dt;
  steps_++;
}

// readActivity (FluidSimulation.ts:1701-1746), applied before the next step: the
// measurement lags the step by exactly one.
void Engine::applyReadback(const uint32_t* words) {
  const FpCounters* c = (const FpCounters*)words;
  std::memcpy(&lastSolver_, words + sizeof(FpCounters) / 4, sizeof(FpSolver));
  const uint32_t* flags = words + (sizeof(FpCounters) + sizeof(FpSolver)) / 4;
  contentTiles_.clear();
  for (int s = 0; s < capacity_ && s < (int)tileRec_.size(); s++)
    if (flags[s] && tileRec_[s].w != 0) contentTiles_.push_back({tileRec_[s], flags[s]});
  activeBricks_ = c->active;
  bricksStepped_ += c->active;
  usedSlots_ = slots_ - (uint32_t)c->freeCount;
  lastFailures_ = c->failures;
  poolLimited_ = c->failures > 0 && slots_ >= slotLimit();
}

int Engine::reset() {
  int rc = consume();
  if (rc) return rc;
  owner_->forget(this);
  cudaStreamSynchronize(stream());
  return initialize();
}

// The latest step's pressure solve, once the step's work is done.
int Engine::readSolver(fp_solver_stats* out) {
  int rc = consume();
  if (rc) return rc;
  if ((rc = check(cudaStreamSynchronize(stream()), "read solver"))) return rc;
  FpSolver S{};
  if ((rc = check(cudaMemcpy(&S, solver_.ptr, sizeof(FpSolver), cudaMemcpyDeviceToHost), "read solver"))) return rc;
  std::memset(out, 0, sizeof(*out));
  out->vcycles = (uint32_t)S.cycles;
  out->unknowns = S.unknowns;
  out->rhs_rms = S.unknowns > 0 ? std::sqrt(S.rhs2 / S.unknowns) : 0.0;
  for (int c = 0; c < S.cycles && c < FP_MAX_VCYCLES; c++)
    out->residual[c] = S.rhs2 > 0 ? std::sqrt(S.res2[c] / S.rhs2) : 0.0;
  out->divergence = S.measured && S.vel2 > 0 ? std::sqrt(S.div2 / S.vel2) : -1.0;
  out->measured = S.measured;
  return FP_OK;
}

int Engine::readBounds(fp_bounds* out) {
  std::memset(out, 0, sizeof(*out));
#ifdef FP_BOUNDS
  int rc = consume();
  if (rc) return rc;
  if ((rc = check(cudaStreamSynchronize(stream()), "read bounds"))) return rc;
  FpBounds b{};
  if ((rc = check(cudaMemcpy(&b, bounds_.ptr, sizeof(b), cudaMemcpyDeviceToHost), "read bounds"))) return rc;
  out->checked = 1;
  out->count = b.count;
  out->site = b.site;
  out->index = b.index;
  out->limit = b.limit;
#endif
  return FP_OK;
}

int Engine::setSolver(int vcycles, float tolerance) {
  if (vcycles < 1 || vcycles > FP_MAX_VCYCLES)
    return fail(FP_EINVAL, "vcycles must be from 1 to " + std::to_string(FP_MAX_VCYCLES) + ".");
  if (!std::isfinite(tolerance) || tolerance < 0.f) return fail(FP_EINVAL, "tolerance must be finite and nonnegative.");
  vcycles_ = vcycles;
  tolerance_ = tolerance;
  return FP_OK;
}

int Engine::krylovPools(uint32_t slots) {
  size_t bytes = (size_t)slots * VN_ * 4;
  bool ok = grow(p0_[2], bytes, 0);
  for (auto& b : kry_) ok = ok && grow(b, bytes, 0);
  return ok ? FP_OK : fail(FP_ENOMEM, "out of device memory for the CG buffers");
}

int Engine::setSchedule(const fp_solver_schedule& sc) {
  if (sc.smoother != FP_SMOOTHER_JACOBI && sc.smoother != FP_SMOOTHER_REDBLACK)
    return fail(FP_EINVAL, "smoother must be FP_SMOOTHER_JACOBI or FP_SMOOTHER_REDBLACK.");
  if (sc.krylov != FP_KRYLOV_NONE && sc.krylov != FP_KRYLOV_FCG)
    return fail(FP_EINVAL, "krylov must be FP_KRYLOV_NONE or FP_KRYLOV_FCG.");
  if (sc.topology != 0 && sc.topology != 1) return fail(FP_EINVAL, "topology must be 0 or 1.");
  fp_solver_schedule next = sc;
  if (sc.smoother == FP_SMOOTHER_REDBLACK) {
    if (sc.levels != 0 && (sc.levels < 2 || sc.levels > bottom_ + 1))
      return fail(FP_EINVAL, "levels must be 0 or from 2 to " + std::to_string(bottom_ + 1) + ".");
    if (sc.pre_sweeps < 1 || sc.pre_sweeps > 8) return fail(FP_EINVAL, "pre_sweeps must be from 1 to 8.");
    if (sc.post_sweeps < 0 || sc.post_sweeps > 8) return fail(FP_EINVAL, "post_sweeps must be from 0 to 8.");
    if (sc.bottom_sweeps < 1 || sc.bottom_sweeps > 64) return fail(FP_EINVAL, "bottom_sweeps must be from 1 to 64.");
  } else {
    next.levels = next.pre_sweeps = next.post_sweeps = next.bottom_sweeps = 0;  // the reference's plan
  }
  int rc = consume();
  if (rc) return rc;
  if (next.krylov && (rc = krylovPools(slots_))) return rc;
  schedule_ = next;
  return FP_OK;
}

int Engine::setRuntime(float cutoff, double budget, int ground) {
  if (!std::isfinite(cutoff)) return fail(FP_EINVAL, "grid.cutoff must be a finite number from 0 to 1.");
  cutoff_ = cutoff;
  if (budget > 0) budget_ = budget;
  ground_ = ground != 0;
  return FP_OK;
}

uint64_t Engine::memoryBytes() const {
  uint64_t bytes = 0;
  const DeviceBuffer* all[] = {&pages_, &entries_, &state_, &activity_, &records_, &blockCounts_, &active_,
                               &zeroList_, &freeStack_, &counters_, &curl_, &expn_, &div_, &sb_,
                               &donors_, &solids_, &tileRecD_, &tileNbrD_, &hashD_, &solver_, &tileMask_,
                               &liveTilesD_, &tileIndexD_, &bounds_};
  for (const DeviceBuffer* b : all) bytes += b->bytes;
  for (auto& b : vel_) bytes += b.bytes;
  for (auto& b : fld_) bytes += b.bytes;
  for (auto& b : smoke_) bytes += b.bytes;
  bytes += smokeBnd_.bytes + meshTablesD_.bytes + meshSourcesD_.bytes + coverageD_.bytes;
  for (auto& b : p0_) bytes += b.bytes;
  for (auto& b : kry_) bytes += b.bytes;
  for (int l = 0; l < FP_MAX_LEVELS; l++) bytes += topo_[l].bytes + lrhs_[l].bytes + lp_[l][0].bytes + lp_[l][1].bytes;
  return bytes;
}

int Engine::stats(fp_stats* out) {
  int rc = consume();
  if (rc) return rc;
  std::memset(out, 0, sizeof(*out));
  out->time = time_;
  out->steps = (uint64_t)steps_;
  out->active_bricks = activeBricks_;
  out->bricks_stepped = bricksStepped_;
  out->brick_cells = (uint32_t)N_;
  out->pool_limited = poolLimited_;
  out->pool_slots = slots_;
  out->used_slots = usedSlots_;
  out->tiles = (uint32_t)dir_.count();
  out->tile_capacity = (uint32_t)capacity_;
  out->failures = lastFailures_;
  out->memory_bytes = memoryBytes();
  // The pressure solve's measurements travel with the next step's measurement: these are the
  // step before the latest one's (readSolver gives the latest step's).
  const FpSolver& S = lastSolver_;
  out->last_vcycles = S.cycles > 0 ? (uint32_t)S.cycles : (steps_ > 1 ? 1u : 0u);
  out->last_residual = S.cycles > 0 && S.rhs2 > 0 ? std::sqrt(S.res2[S.cycles - 1] / S.rhs2) : -1.0;
  out->last_divergence = S.measured && S.vel2 > 0 ? std::sqrt(S.div2 / S.vel2) : -1.0;
  out->kernel_launches = owner_->launches();
  out->h2d_bytes = stepH2d_;
  out->d2h_bytes = stepD2h_;
  out->host_prepare_ms = owner_->hostPrepareMs();
  out->host_wait_ms = owner_->hostWaitMs();
  return FP_OK;
}

int Engine::readField(int field, float* host, size_t bytes) {
  const DeviceBuffer* b = nullptr;
  size_t ch = 0;
  switch (field) {
    case FP_FIELD_VELOCITY: b = &vel_[velIdx_[0]]; ch = 3; break;
    case FP_FIELD_SCALARS: b = &fld_[fldIdx_[0]]; ch = 4; break;
    case FP_FIELD_EXPANSION: b = &expn_; ch = 1; break;
    case FP_FIELD_PRESSURE: b = &p0_[latest_]; ch = 1; break;
    case FP_FIELD_DIVERGENCE: b = &div_; ch = 1; break;
    case FP_FIELD_CURL: b = &curl_; ch = 4; break;
    case FP_FIELD_SMOKE:
      if (smokeDiv_ == 1) return fail(FP_EINVAL, "the smoke field exists with smokeDivisor 2 or 4 only");
      b = &smoke_[smokeIdx_[0]];
      ch = 1;
      break;
    default: return fail(FP_EINVAL, "unknown field");
  }
  const bool velocityLattice =
      field == FP_FIELD_VELOCITY || field == FP_FIELD_PRESSURE || field == FP_FIELD_DIVERGENCE || field == FP_FIELD_CURL;
  const size_t cells = field == FP_FIELD_SMOKE ? (size_t)SN_ : (velocityLattice ? (size_t)VN_ : (size_t)N_);
  size_t need = (size_t)slots_ * ch * cells * 4;
  if (bytes != need) return fail(FP_EINVAL, "field buffer size mismatch: need " + std::to_string(need) + " bytes");
  int rc = consume();
  if (rc) return rc;
  if ((rc = check(cudaStreamSynchronize(stream()), "read field"))) return rc;
  if ((field == FP_FIELD_SCALARS || field == FP_FIELD_SMOKE) && scalarBytes() == 2) {
    // FP16 storage: widened to FP32 for the caller.
    std::vector<__half> raw(need / 4);
    if ((rc = check(cudaMemcpy(raw.data(), b->ptr, raw.size() * 2, cudaMemcpyDeviceToHost), "read field"))) return rc;
    for (size_t i = 0; i < raw.size(); i++) host[i] = __half2float(raw[i]);
    return FP_OK;
  }
  return check(cudaMemcpy(host, b->ptr, need, cudaMemcpyDeviceToHost), "read field");
}

int Engine::readTable(int table, void* host, size_t* bytes) {
  int rc = consume();
  if (rc) return rc;
  if ((rc = check(cudaStreamSynchronize(stream()), "read table"))) return rc;
  size_t bricks = (size_t)capacity_ * 64;
  std::vector<uint32_t> w;
  auto fetch = [&](const DeviceBuffer& b, size_t words, size_t offsetWords = 0) {
    size_t old = w.size();
    w.resize(old + words);
    cudaMemcpy(w.data() + old, (const uint32_t*)b.ptr + offsetWords, words * 4, cudaMemcpyDeviceToHost);
  };
  switch (table) {
    case FP_TABLE_ENTRIES: fetch(entries_, bricks); break;
    case FP_TABLE_PAGES: fetch(pages_, bricks); break;
    case FP_TABLE_STATE: fetch(state_, bricks); break;
    case FP_TABLE_ACTIVITY: fetch(activity_, bricks + capacity_); break;
    case FP_TABLE_RECORDS: fetch(records_, bricks * FP_RECORD_WORDS); break;
    case FP_TABLE_FREE: {
      FpCounters c;
      cudaMemcpy(&c, counters_.ptr, sizeof(c), cudaMemcpyDeviceToHost);
      w.push_back((uint32_t)c.freeCount);
      w.push_back(lastFailures_);
      fetch(freeStack_, slots_);
      break;
    }
    case FP_TABLE_ACTIVE: {
      FpCounters c;
      cudaMemcpy(&c, counters_.ptr, sizeof(c), cudaMemcpyDeviceToHost);
      w.push_back(c.active);
      fetch(active_, c.active);
      break;
    }
    case FP_TABLE_SOLIDS: fetch(solids_, (size_t)slots_ * W_); break;
    case FP_TABLE_TILES:
      for (int t = 0; t < capacity_; t++) {
        int4 r = t < (int)tileRec_.size() ? tileRec_[t] : make_int4(0, 0, 0, 0);
        w.push_back((uint32_t)r.x);
        w.push_back((uint32_t)r.y);
        w.push_back((uint32_t)r.z);
        w.push_back((uint32_t)r.w);
      }
      break;
    default: return fail(FP_EINVAL, "unknown table");
  }
  size_t need = w.size() * 4;
  if (!host || *bytes < need) {
    *bytes = need;
    return fail(FP_ELIMIT, "table buffer too small");
  }
  std::memcpy(host, w.data(), need);
  *bytes = need;
  return FP_OK;
}

// readBricks (FluidSimulation.ts:1749-1779): world boxes of the bricks holding a slot.
int Engine::readBricks(float* boxes, uint32_t* count) {
  int rc = consume();
  if (rc) return rc;
  if ((rc = check(cudaStreamSynchronize(stream()), "read bricks"))) return rc;
  size_t bricks = (size_t)capacity_ * 64;
  std::vector<int> pages(bricks);
  cudaMemcpy(pages.data(), pages_.ptr, bricks * 4, cudaMemcpyDeviceToHost);
  float size = (float)B_ * h_;
  uint32_t n = 0;
  for (size_t id = 0; id < bricks; id++) {
    const int4& t = tileRec_[id / 64];
    if (t.w == 0 || pages[id] < 0) continue;
    if (boxes && n < *count) {
      int l = (int)(id % 64);
      float mn[3] = {(float)(t.x * 4 + (l & 3)) * size, (float)(t.y * 4 + ((l >> 2) & 3)) * size,
                     (float)(t.z * 4 + (l >> 4)) * size};
      for (int a = 0; a < 3; a++) {
        boxes[n * 6 + a] = mn[a];
        boxes[n * 6 + 3 + a] = mn[a] + size;
      }
    }
    n++;
  }
  bool fits = boxes && n <= *count;
  *count = n;
  return fits ? FP_OK : fail(FP_ELIMIT, "brick buffer too small");
}

}  // namespace fp
