// Session snapshot and restore: a simulation's whole state between two steps as one blob.
//
// No reference counterpart: the reference's document (editor/document.ts:60-61) saves a scene's
// settings, not a simulation's state. Here a snapshot holds everything a later step reads, so a
// server can evict a session to host memory and bring it back, or move it to another GPU, and
// the restored simulation steps on bit for bit as the original would have:
//   - the grid it was made for (a restore into another grid fails);
//   - the host state: tile directory, tables, counters, time, the scene's last colliders and
//     mesh tables, the solver settings, the rotating buffer indices;
//   - every device buffer of the simulation (pools, tables, multigrid levels, measurement), at
//     its size. The render pools are rebuilt at the next render and are not saved.
// The blob is little-endian native layout, for this library build only.
#include <cstring>

#include "fp_engine.hpp"

namespace fp {

namespace {

constexpr uint32_t MAGIC = 0x4e535046u;  // "FPSN"
constexpr uint32_t VERSION = 4;

struct Writer {
  std::vector<uint8_t>& out;
  void raw(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    out.insert(out.end(), b, b + n);
  }
  template <class T>
  void pod(const T& v) {
    raw(&v, sizeof(T));
  }
  template <class T>
  void vec(const std::vector<T>& v) {
    uint64_t n = v.size();
    pod(n);
    if (n) raw(v.data(), n * sizeof(T));
  }
};

struct Reader {
  const uint8_t* p;
  const uint8_t* end;
  bool ok = true;
  void raw(void* dst, size_t n) {
    if (!ok || (size_t)(end - p) < n) {
      ok = false;
      return;
    }
    std::memcpy(dst, p, n);
    p += n;
  }
  template <class T>
  void pod(T& v) {
    raw(&v, sizeof(T));
  }
  template <class T>
  void vec(std::vector<T>& v) {
    uint64_t n = 0;
    pod(n);
    if (!ok || n > (uint64_t)(end - p) / sizeof(T)) {
      ok = false;
      return;
    }
    v.resize(n);
    if (n) raw(v.data(), n * sizeof(T));
  }
};

}  // namespace

// The buffers a snapshot carries, in a fixed order.
#define FP_SNAPSHOT_BUFFERS(X)                                                                            \
  X(pages_) X(entries_) X(state_) X(activity_) X(records_) X(blockCounts_) X(active_) X(zeroList_)        \
  X(freeStack_) X(counters_) X(vel_[0]) X(vel_[1]) X(vel_[2]) X(vel_[3]) X(curl_) X(fld_[0]) X(fld_[1])   \
  X(fld_[2]) X(expn_) X(div_) X(sb_) X(donors_) X(solids_) X(p0_[0]) X(p0_[1])           \
  X(p0_[2]) X(kry_[0]) X(kry_[1]) X(kry_[2]) X(tileRecD_) X(tileNbrD_) X(hashD_) X(solver_) X(tileMask_) \
  X(liveTilesD_) X(tileIndexD_) X(smoke_[0]) X(smoke_[1]) X(smoke_[2]) X(smokeBnd_) X(meshTablesD_)      \
  X(meshSourcesD_) X(coverageD_) \
  FP_SNAPSHOT_LEVEL(X, 0) FP_SNAPSHOT_LEVEL(X, 1) FP_SNAPSHOT_LEVEL(X, 2) FP_SNAPSHOT_LEVEL(X, 3)     \
  FP_SNAPSHOT_LEVEL(X, 4) FP_SNAPSHOT_LEVEL(X, 5) FP_SNAPSHOT_LEVEL(X, 6) FP_SNAPSHOT_LEVEL(X, 7)
// The multigrid levels: topology, pressure pair, right-hand side (index 43 + 4 level on).
#define FP_SNAPSHOT_LEVEL(X, l) X(topo_[l]) X(lp_[l][0]) X(lp_[l][1]) X(lrhs_[l])
static_assert(FP_MAX_LEVELS == 8, "the snapshot lists eight multigrid levels");

int Engine::snapshot(std::vector<uint8_t>& out) {
  int rc = consume();
  if (rc) return rc;
  if ((rc = check(cudaStreamSynchronize(stream()), "snapshot"))) return rc;
  out.clear();
  {
    // Room for every buffer at once: the pools of a large budget take gigabytes.
    size_t bytes = 1 << 20;
#define FP_SIZE(b) bytes += (b.ptr ? b.bytes : 0) + 8;
    FP_SNAPSHOT_BUFFERS(FP_SIZE)
#undef FP_SIZE
    bytes += (tileRec_.size() + hash_.size()) * sizeof(int4) + tileNbr_.size() * 4 + coverage_.size() * 4 +
             meshTables_.size() * 4 + meshRecords_.size() * sizeof(FpMeshSource);
    out.reserve(bytes);
  }
  Writer w{out};
  w.pod(MAGIC);
  w.pod(VERSION);
  const int grid[6] = {B_, vd_, smokeDiv_, precision_, maccormack_ ? 1 : 0, 0};
  w.raw(grid, sizeof(grid));
  w.pod(h_);
  // host state
  w.pod(budget_);
  w.pod(cutoff_);
  w.pod(ground_);
  w.vec(dir_.slots_);
  std::vector<std::pair<uint64_t, int>> index(dir_.index_.begin(), dir_.index_.end());
  w.vec(index);
  w.vec(dir_.created_);
  w.pod(dir_.ground);
  w.pod(dir_.dirty);
  w.pod(capacity_);
  w.vec(tileRec_);
  w.vec(tileNbr_);
  w.vec(hash_);
  w.pod(time_);
  w.pod(steps_);
  w.pod(mayHaveFlame_);
  w.pod(solidsStale_);
  w.pod(geometryDirty_);
  w.pod(colliderCount_);
  w.vec(prevColliders_);
  w.vec(prevMasks_);
  w.vec(contentTiles_);
  w.pod(activeBricks_);
  w.pod(usedSlots_);
  w.pod(lastFailures_);
  w.pod(bricksStepped_);
  w.pod(poolLimited_);
  w.pod(latest_);
  w.pod(vcycles_);
  w.pod(tolerance_);
  w.pod(schedule_);
  w.pod(measure_);
  w.pod(lastSolver_);
  w.pod(slots_);
  w.raw(velIdx_, sizeof(velIdx_));
  w.raw(fldIdx_, sizeof(fldIdx_));
  w.raw(smokeIdx_, sizeof(smokeIdx_));
  w.vec(meshRecords_);
  w.vec(meshTables_);
  w.pod(meshCount_);
  w.pod(tileVersion_);
  w.pod(meshVersion_);
  w.vec(coverage_);
  w.vec(coverageTargets_);
  w.pod(coverageOn_);
  w.pod(coverageVersion_);
  w.vec(liveTiles_);
  w.vec(tileIndex_);
  w.vec(renderBoxes_);
  w.vec(clusterOf_);
  w.vec(clusterBoxes_);
  w.pod(dir_.nextSeq_);
  w.vec(sourceBoxes_);
  // device buffers: size, then contents
  std::vector<uint8_t> host;
#define FP_SAVE(b)                                                                                   \
  {                                                                                                  \
    uint64_t n = b.ptr ? (uint64_t)b.bytes : 0;                                                      \
    w.pod(n);                                                                                        \
    if (n) {                                                                                         \
      size_t at = out.size();                                                                        \
      out.resize(at + n);                                                                            \
      if ((rc = check(cudaMemcpy(out.data() + at, b.ptr, n, cudaMemcpyDeviceToHost), "snapshot"))) \
        return rc;                                                                                   \
    }                                                                                                \
  }
  FP_SNAPSHOT_BUFFERS(FP_SAVE)
#undef FP_SAVE
  return FP_OK;
}

int Engine::restore(const uint8_t* data, size_t bytes) {
  Reader r{data, data + bytes};
  uint32_t magic = 0, version = 0;
  r.pod(magic);
  r.pod(version);
  if (!r.ok || magic != MAGIC || version != VERSION) return fail(FP_EINVAL, "not a snapshot of this library");
  int grid[6];
  float h = 0.f;
  r.raw(grid, sizeof(grid));
  r.pod(h);
  const int mine[6] = {B_, vd_, smokeDiv_, precision_, maccormack_ ? 1 : 0, 0};
  if (!r.ok || std::memcmp(grid, mine, sizeof(grid)) != 0 || h != h_)
    return fail(FP_EINVAL, "the snapshot was taken of another grid");
  int rc = consume();
  if (rc) return rc;
  owner_->forget(this);
  if ((rc = check(cudaStreamSynchronize(stream()), "restore"))) return rc;
  // Host state into temporaries first: a truncated blob changes nothing.
  Engine& e = *this;
  double budget;
  float cutoff;
  bool ground;
  TileDirectory dir;
  std::vector<std::pair<uint64_t, int>> index;
  r.pod(budget);
  r.pod(cutoff);
  r.pod(ground);
  r.vec(dir.slots_);
  r.vec(index);
  r.vec(dir.created_);
  r.pod(dir.ground);
  r.pod(dir.dirty);
  for (auto& kv : index) dir.index_[kv.first] = kv.second;
  int capacity;
  std::vector<int4> tileRec, hash;
  std::vector<int> tileNbr;
  r.pod(capacity);
  r.vec(tileRec);
  r.vec(tileNbr);
  r.vec(hash);
  double time;
  int64_t steps;
  bool mayHaveFlame, solidsStale, geometryDirty;
  int colliderCount;
  std::vector<uint8_t> prevColliders;
  std::vector<uint32_t> prevMasks;
  std::vector<std::pair<int4, uint32_t>> contentTiles;
  r.pod(time);
  r.pod(steps);
  r.pod(mayHaveFlame);
  r.pod(solidsStale);
  r.pod(geometryDirty);
  r.pod(colliderCount);
  r.vec(prevColliders);
  r.vec(prevMasks);
  r.vec(contentTiles);
  uint32_t activeBricks, usedSlots, lastFailures, slots;
  uint64_t bricksStepped, tileVersion, meshVersion, coverageVersion;
  bool poolLimited, measure, coverageOn;
  int latest, vcycles, meshCount;
  float tolerance;
  fp_solver_schedule schedule;
  FpSolver lastSolver;
  int velIdx[4], fldIdx[3], smokeIdx[3];
  std::vector<FpMeshSource> meshRecords;
  std::vector<int> meshTables, liveTiles, tileIndex, sourceBoxes;
  std::vector<uint32_t> coverage;
  std::vector<int32_t> coverageTargets;
  r.pod(activeBricks);
  r.pod(usedSlots);
  r.pod(lastFailures);
  r.pod(bricksStepped);
  r.pod(poolLimited);
  r.pod(latest);
  r.pod(vcycles);
  r.pod(tolerance);
  r.pod(schedule);
  r.pod(measure);
  r.pod(lastSolver);
  r.pod(slots);
  r.raw(velIdx, sizeof(velIdx));
  r.raw(fldIdx, sizeof(fldIdx));
  r.raw(smokeIdx, sizeof(smokeIdx));
  r.vec(meshRecords);
  r.vec(meshTables);
  r.pod(meshCount);
  r.pod(tileVersion);
  r.pod(meshVersion);
  r.vec(coverage);
  r.vec(coverageTargets);
  r.pod(coverageOn);
  r.pod(coverageVersion);
  r.vec(liveTiles);
  r.vec(tileIndex);
  std::vector<int> renderBoxes, clusterOf, clusterBoxes;
  uint64_t nextSeq = 0;
  r.vec(renderBoxes);
  r.vec(clusterOf);
  r.vec(clusterBoxes);
  r.pod(nextSeq);
  r.vec(sourceBoxes);
  if (!r.ok) return fail(FP_EINVAL, "the snapshot is truncated");
  // Device buffers: each resized to its saved size and filled. First every size is read and
  // the tables' and pools' sizes checked against the saved capacity and slots, so that no
  // kernel can later index past a buffer.
  {
    Reader probe = r;
    std::vector<uint64_t> sizes;
#define FP_PROBE(b)                                                        \
  {                                                                        \
    uint64_t n = 0;                                                        \
    probe.pod(n);                                                          \
    if (probe.ok && n > (uint64_t)(probe.end - probe.p)) probe.ok = false; \
    if (probe.ok) probe.p += n;                                            \
    sizes.push_back(n);                                                    \
  }
    FP_SNAPSHOT_BUFFERS(FP_PROBE)
#undef FP_PROBE
    if (!probe.ok) return fail(FP_EINVAL, "the snapshot is truncated");
    const uint64_t ids = (uint64_t)capacity * 64, vpool = (uint64_t)slots * 3 * VN_ * 4;
    bool sane = capacity > 0 && sizes[0] >= ids * 4 && sizes[1] >= ids * 4 && sizes[2] >= ids * 4 &&
                sizes[3] >= (ids + capacity) * 4 && sizes[4] >= ids * FP_RECORD_WORDS * 4 && sizes[8] >= (uint64_t)slots * 4;
    for (int k = 10; k < 14; k++) sane = sane && sizes[k] >= vpool;  // vel_
    sane = sane && sizes[23] >= (uint64_t)slots * VN_ * 4 && sizes[24] >= (uint64_t)slots * VN_ * 4;  // p0_[0..1]
    sane = sane && tileRec.size() == (size_t)capacity && tileNbr.size() == (size_t)capacity * 27;
    // Every level's topology and values: per slot on the brick levels, per tile slot on the
    // tile levels.
    for (int l = 0; l <= bottom_ && sane; l++) {
      const uint64_t cells = (uint64_t)levelCells(l) * (l < brickLevels_ ? slots : (uint64_t)capacity);
      sane = sizes[43 + 4 * l] >= cells;
      if (l > 0) sane = sane && sizes[44 + 4 * l] >= cells * coarseBytes() && sizes[45 + 4 * l] >= cells * coarseBytes() &&
                        sizes[46 + 4 * l] >= cells * coarseBytes();
    }
    if (!sane) return fail(FP_EINVAL, "the snapshot's tables do not match its sizes");
    // The buffer selectors index the pools (a step only swaps two: permutations), and the live
    // tiles are tile slots in ascending order, each at its own position in the slot ->
    // position table (both lists are built together).
    auto permutation = [](const int* v, int n) {
      unsigned seen = 0;
      for (int k = 0; k < n; k++) {
        if (v[k] < 0 || v[k] >= n || ((seen >> v[k]) & 1u)) return false;
        seen |= 1u << v[k];
      }
      return true;
    };
    bool consistent = permutation(velIdx, 4) && permutation(fldIdx, 3) && permutation(smokeIdx, 3);
    for (size_t j = 0; consistent && j < liveTiles.size(); j++)
      consistent = liveTiles[j] >= 0 && (size_t)liveTiles[j] < tileIndex.size() && tileIndex[liveTiles[j]] == (int)j &&
                   (j == 0 || liveTiles[j] > liveTiles[j - 1]);
    if (!consistent) return fail(FP_EINVAL, "the snapshot's buffer selectors or live tiles are inconsistent");
  }
#define FP_LOAD(b)                                                                                      \
  {                                                                                                     \
    uint64_t n = 0;                                                                                     \
    r.pod(n);                                                                                           \
    if (n == 0) {                                                                                       \
      if (e.b.ptr) cudaFree(e.b.ptr);                                                                   \
      e.b = DeviceBuffer{};                                                                             \
    } else {                                                                                            \
      if (e.b.bytes != n && !alloc(e.b, n, false)) return fail(FP_ENOMEM, "out of device memory for the restore"); \
      if ((rc = check(cudaMemcpy(e.b.ptr, r.p, n, cudaMemcpyHostToDevice), "restore"))) return rc;     \
      r.p += n;                                                                                         \
    }                                                                                                   \
  }
  FP_SNAPSHOT_BUFFERS(FP_LOAD)
#undef FP_LOAD
  budget_ = budget;
  cutoff_ = cutoff;
  ground_ = ground;
  dir_ = dir;
  capacity_ = capacity;
  tileRec_ = tileRec;
  tileNbr_ = tileNbr;
  hash_ = hash;
  time_ = time;
  steps_ = steps;
  mayHaveFlame_ = mayHaveFlame;
  solidsStale_ = solidsStale;
  geometryDirty_ = geometryDirty;
  colliderCount_ = colliderCount;
  prevColliders_ = prevColliders;
  prevMasks_ = prevMasks;
  contentTiles_ = contentTiles;
  activeBricks_ = activeBricks;
  usedSlots_ = usedSlots;
  lastFailures_ = lastFailures;
  bricksStepped_ = bricksStepped;
  poolLimited_ = poolLimited;
  latest_ = latest;
  vcycles_ = vcycles;
  tolerance_ = tolerance;
  schedule_ = schedule;
  measure_ = measure;
  lastSolver_ = lastSolver;
  slots_ = slots;
  std::memcpy(velIdx_, velIdx, sizeof(velIdx));
  std::memcpy(fldIdx_, fldIdx, sizeof(fldIdx));
  std::memcpy(smokeIdx_, smokeIdx, sizeof(smokeIdx));
  meshRecords_ = meshRecords;
  meshTables_ = meshTables;
  meshCount_ = meshCount;
  tileVersion_ = tileVersion;
  meshVersion_ = meshVersion;
  coverage_ = coverage;
  coverageTargets_ = coverageTargets;
  coverageOn_ = coverageOn;
  coverageVersion_ = coverageVersion;
  liveTiles_ = liveTiles;
  tileIndex_ = tileIndex;
  renderBoxes_ = renderBoxes;
  clusterOf_ = clusterOf;
  clusterBoxes_ = clusterBoxes;
  dir_.nextSeq_ = nextSeq;
  sourceBoxes_ = sourceBoxes;
  return FP_OK;
}

}  // namespace fp
