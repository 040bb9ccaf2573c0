// Sparse geometric multigrid for the pressure (src/engine/shaders/pressure.wgsl and
// src/engine/PressureSolver.ts). Level 0 is the velocity grid; each brick holds levels down
// to 2^3 cells; three tile levels (4^3, 2^3 and one cell per tile) follow. Weighted Jacobi
// (omega 0.8) smoothing, residual restriction that also writes the coarse level's first
// iterate, trilinear prolongation with Neumann ghosts at solid coarse cells, and a bottom
// solve in one CTA. Brick levels run a CTA per computing brick; tile levels a CTA per tile.
#include "fp_device.cuh"
#include "fp_launch.h"

namespace {

constexpr uint32_t SOLIDF = 1024u;

FP_DEV int levelShift(const SimParams& P, int level) {
  return level < P.brickLevels ? P.brickLevels - level : P.brickLevels + 2 - level;
}

// cellAddress (pressure.wgsl:72-92): -1 without storage.
FP_DEV long cellAddress(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  int s = levelShift(P, level), side = 1 << s, m = side - 1;
  long owner;
  if (level < P.brickLevels) {
    int slot = brickSlot(P, H, px >> s, py >> s, pz >> s);
    if (slot < 0) return -1;
    owner = slot;
  } else {
    int t = tileAt(P, H, px >> s, py >> s, pz >> s);
    if (t < 0) return -1;
    owner = t;
  }
  return owner * side * side * side + ((pz & m) * side + (py & m)) * side + (px & m);
}

// activeCell (pressure.wgsl:100-136): whether a level's cell is a pressure unknown.
FP_DEV bool activeCell(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  int bl = P.brickLevels;
  if (level >= bl) {
    int n = 1 << (level - bl);
    for (int z = 0; z < n; z++)
      for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
          int id = brickIdAt(P, H, px * n + x, py * n + y, pz * n + z);
          if (id < 0 || P.entries[id] < 0 || P.records[(size_t)id * FP_RECORD_WORDS + 27] == 0) return false;
        }
    return true;
  }
  int span = 1 << level;
  int lx = (px * span - 1) >> bl, ly = (py * span - 1) >> bl, lz = (pz * span - 1) >> bl;
  int hx = (px * span + span - 1) >> bl, hy = (py * span + span - 1) >> bl, hz = (pz * span + span - 1) >> bl;
  if (P.ground) ly = max(ly, 0);
  for (int z = lz; z <= hz; z++)
    for (int y = ly; y <= hy; y++)
      for (int x = lx; x <= hx; x++)
        if (brickSlot(P, H, x, y, z) < 0) return false;
  return true;
}

FP_DEV uint32_t expandFlags(uint8_t t) { return (t & FP_STORED_SOLID) ? SOLIDF : (uint32_t)(t & 63u); }
FP_DEV float diagOf(uint32_t f) {
  return (float)((f >> 0) & 1u) + (float)((f >> 1) & 1u) + ((float)((f >> 2) & 1u) + (float)((f >> 3) & 1u)) +
         ((float)((f >> 4) & 1u) + (float)((f >> 5) & 1u));
}
FP_DEV float readAt(const SimParams& P, const Home& H, const float* arr, int px, int py, int pz, int level) {
  long a = cellAddress(P, H, px, py, pz, level);
  return a < 0 ? 0.f : arr[a];
}
// stencil (pressure.wgsl:360-402): open neighbours' sum; cubic cells weigh 1 on every axis.
FP_DEV float stencilSum(const SimParams& P, const Home& H, const float* p, int px, int py, int pz, uint32_t f,
                        int level) {
  float v0 = (f & 1u) ? readAt(P, H, p, px + 1, py, pz, level) : 0.f;
  float v1 = (f & 2u) ? readAt(P, H, p, px - 1, py, pz, level) : 0.f;
  float v2 = (f & 4u) ? readAt(P, H, p, px, py + 1, pz, level) : 0.f;
  float v3 = (f & 8u) ? readAt(P, H, p, px, py - 1, pz, level) : 0.f;
  float v4 = (f & 16u) ? readAt(P, H, p, px, py, pz + 1, level) : 0.f;
  float v5 = (f & 32u) ? readAt(P, H, p, px, py, pz - 1, level) : 0.f;
  return (v0 + v1) + (v2 + v3) + (v4 + v5);
}

FP_DEV bool coarseSolid(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  long a = cellAddress(P, H, px, py, pz, level);
  if (a < 0) return false;
  return (P.topo[level][a] & FP_STORED_SOLID) != 0;
}
// coarseValue (pressure.wgsl:670-696): Neumann ghosts at solid coarse cells, the ground mirrored.
FP_DEV float coarseValue(const SimParams& P, const Home& H, const float* coarse, int level, int px, int py, int pz) {
  int groundY = P.ground ? 0 : -0x7fffffff;
  int c[3] = {px, max(py, groundY), pz};
  if (!coarseSolid(P, H, c[0], c[1], c[2], level)) return readAt(P, H, coarse, c[0], c[1], c[2], level);
  float sum = 0.f, count = 0.f;
  for (int axis = 0; axis < 3; axis++)
    for (int side = -1; side <= 1; side += 2) {
      int q[3] = {c[0], c[1], c[2]};
      q[axis] += side;
      q[1] = max(q[1], groundY);
      if (!coarseSolid(P, H, q[0], q[1], q[2], level)) {
        sum += readAt(P, H, coarse, q[0], q[1], q[2], level);
        count += 1.f;
      }
    }
  return sum / fmaxf(count, 1.f);
}

// Operation on one cell of a level (relaxCell, prolongateCell, restrictCell).
enum Op { RELAX = 0, PROLONG = 1, RESTRICT = 2 };

struct Args {
  int level;  // output level
  const float* rhs;
  const float* pin;
  const float* coarse;
  float* pout;
  float* cfirst;
};

FP_DEV void relaxCell(const SimParams& P, const Home& H, const Args& A, long a, int px, int py, int pz) {
  uint32_t f = expandFlags(P.topo[A.level][a]);
  if ((f & SOLIDF) || !activeCell(P, H, px, py, pz, A.level)) {
    A.pout[a] = 0.f;
    return;
  }
  float sum = stencilSum(P, H, A.pin, px, py, pz, f, A.level);
  float cand = (sum - A.rhs[a]) / fmaxf(diagOf(f), 1e-12f);
  A.pout[a] = mixf(A.pin[a], cand, 0.8f);
}

FP_DEV void prolongCell(const SimParams& P, const Home& H, const Args& A, long a, int px, int py, int pz) {
  uint32_t f = expandFlags(P.topo[A.level][a]);
  if ((f & SOLIDF) || !activeCell(P, H, px, py, pz, A.level)) {
    A.pout[a] = 0.f;
    return;
  }
  int cl = A.level + 1;
  float qx = ((float)px + 0.5f) * 0.5f - 0.5f, qy = ((float)py + 0.5f) * 0.5f - 0.5f, qz = ((float)pz + 0.5f) * 0.5f - 0.5f;
  int ix = (int)floorf(qx), iy = (int)floorf(qy), iz = (int)floorf(qz);
  float fx = qx - floorf(qx), fy = qy - floorf(qy), fz = qz - floorf(qz);
  bool fast = P.colliderCount == 0 && (!P.ground || iy >= 0);
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
    v[k] = fast ? readAt(P, H, A.coarse, ix + dx, iy + dy, iz + dz, cl)
                : coarseValue(P, H, A.coarse, cl, ix + dx, iy + dy, iz + dz);
  }
  float corr = mixf(mixf(mixf(v[0], v[1], fx), mixf(v[2], v[3], fx), fy), mixf(mixf(v[4], v[5], fx), mixf(v[6], v[7], fx), fy),
                    fz);
  A.pout[a] = A.pin[a] + corr;
}

// restrictCell (pressure.wgsl:601-647): (cx,cy,cz) is a cell of the coarse (output) level.
FP_DEV void restrictCell(const SimParams& P, const Home& H, const Args& A, long out, int cx, int cy, int cz) {
  int fine = A.level - 1;
  float residual = 0.f;
  bool every = true;
  for (int k = 0; k < 8; k++) {
    int px = cx * 2 + (k & 1), py = cy * 2 + ((k >> 1) & 1), pz = cz * 2 + (k >> 2);
    bool unknown = activeCell(P, H, px, py, pz, fine);
    every = every && unknown;
    if (unknown) {
      long a = cellAddress(P, H, px, py, pz, fine);
      uint32_t f = expandFlags(P.topo[fine][a]);
      if (!(f & SOLIDF)) {
        float sum = stencilSum(P, H, A.pin, px, py, pz, f, fine);
        residual += A.rhs[a] - (sum - diagOf(f) * A.pin[a]);
      }
    }
  }
  float r = residual * 0.5f;
  A.pout[out] = r;  // the coarse right-hand side
  float first = 0.f;
  if (every) {
    uint32_t f = expandFlags(P.topo[A.level][out]);
    if (!(f & SOLIDF)) first = mixf(0.f, (0.f - r) / fmaxf(diagOf(f), 1e-12f), 0.8f);
  }
  A.cfirst[out] = first;
}

template <int OP>
FP_DEV void levelCell(const SimParams& P, const Home& H, const Args& A, long a, int px, int py, int pz) {
  if (OP == RELAX) relaxCell(P, H, A, a, px, py, pz);
  if (OP == PROLONG) prolongCell(P, H, A, a, px, py, pz);
  if (OP == RESTRICT) restrictCell(P, H, A, a, px, py, pz);
}

// Every cell of `A.level` in every computing brick.
template <int OP>
__global__ void __launch_bounds__(256) k_level_bricks(const SimParams* __restrict__ Pp, Args A) {
  const SimParams& P = *Pp;
  __shared__ int nslot[27];
  uint32_t total = P.counters->active;
  int s = levelShift(P, A.level), side = 1 << s, cells = side * side * side;
  for (uint32_t i = blockIdx.x; i < total; i += gridDim.x) {
    Home H = enterBrick(P, P.active[i], nslot);
    long base = (long)nslot[13] * cells;
    for (int o = threadIdx.x; o < cells; o += blockDim.x) {
      int lx = o & (side - 1), ly = (o >> s) & (side - 1), lz = o >> (2 * s);
      levelCell<OP>(P, H, A, base + o, H.bx * side + lx, H.by * side + ly, H.bz * side + lz);
    }
    __syncthreads();
  }
}

FP_DEV Home enterTile(const SimParams& P, int t, int4 rec) {
  Home H;
  H.tile = t;
  H.tx = rec.x;
  H.ty = rec.y;
  H.tz = rec.z;
  H.bx = H.by = H.bz = -(1 << 29);  // no home brick: lookups go through the tiles
  H.nslot = nullptr;
  return H;
}

// Every cell of `A.level` (a tile level) in every tile.
template <int OP>
__global__ void __launch_bounds__(64) k_level_tiles(const SimParams* __restrict__ Pp, Args A) {
  const SimParams& P = *Pp;
  int s = levelShift(P, A.level), side = 1 << s, cells = side * side * side;
  for (int t = blockIdx.x; t < P.capacity; t += gridDim.x) {
    int4 rec = __ldg(&P.tileRec[t]);
    if (rec.w == 0) continue;
    Home H = enterTile(P, t, rec);
    for (int o = threadIdx.x; o < cells; o += blockDim.x) {
      int lx = o & (side - 1), ly = (o >> s) & (side - 1), lz = o >> (2 * s);
      levelCell<OP>(P, H, A, (long)t * cells + o, rec.x * side + lx, rec.y * side + ly, rec.z * side + lz);
    }
  }
}

// relaxCoarse (pressure.wgsl:549-599): the bottom level, one cell per tile slot, every
// iteration in one CTA. Tile slots stride over the threads; each slot's flags (SOLIDF where
// it is no unknown) and a ping-pong pair of values live in shared memory, so any number of
// tiles that fits 12 bytes a slot needs one launch.
__global__ void __launch_bounds__(1024) k_bottom(const SimParams* __restrict__ Pp, int level, int iterations,
                                                  const float* __restrict__ rhs, const float* __restrict__ pin,
                                                  float* __restrict__ pout) {
  const SimParams& P = *Pp;
  extern __shared__ float bottomSmem[];
  int cap = P.capacity;
  float* cur = bottomSmem;
  float* nxt = bottomSmem + cap;
  uint32_t* flags = reinterpret_cast<uint32_t*>(bottomSmem + 2 * cap);
  for (int t = threadIdx.x; t < cap; t += blockDim.x) {
    int4 rec = __ldg(&P.tileRec[t]);
    uint32_t f = SOLIDF | (rec.w != 0 ? 0x80000000u : 0u);  // top bit: a live tile slot
    float v = 0.f;
    if (rec.w != 0) {
      Home H = enterTile(P, t, rec);
      if (activeCell(P, H, rec.x, rec.y, rec.z, level)) {
        f = expandFlags(P.topo[level][t]) | 0x80000000u;
        v = pin[t];
      }
    }
    flags[t] = f;
    cur[t] = v;
  }
  __syncthreads();
  const int nbIndex[6] = {nbrIndex(1, 0, 0), nbrIndex(-1, 0, 0), nbrIndex(0, 1, 0),
                          nbrIndex(0, -1, 0), nbrIndex(0, 0, 1), nbrIndex(0, 0, -1)};
  for (int it = 0; it < iterations; it++) {
    for (int t = threadIdx.x; t < cap; t += blockDim.x) {
      uint32_t f = flags[t];
      float next = 0.f;
      if ((f & 0x80000000u) && !(f & SOLIDF)) {
        float w[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
          int n = ((f >> k) & 1u) ? __ldg(&P.tileNbr[t * 27 + nbIndex[k]]) : -1;
          w[k] = n >= 0 ? cur[n] : 0.f;
        }
        float sum = (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
        float cand = (sum - rhs[t]) / fmaxf(diagOf(f & 63u), 1e-12f);
        next = mixf(cur[t], cand, 0.8f);
      }
      nxt[t] = next;
    }
    __syncthreads();
    float* tmp = cur;
    cur = nxt;
    nxt = tmp;
  }
  for (int t = threadIdx.x; t < cap; t += blockDim.x)
    if (flags[t] & 0x80000000u) pout[t] = cur[t];
}

// cellTopology (pressure.wgsl:208-222): solid, or the sides whose neighbours are not solid.
FP_DEV uint8_t cellTopology(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  float s = P.h * (float)(1 << level);
  auto blocked = [&](int x, int y, int z) {
    return solidAt(P, H, ((float)x + 0.5f) * s, ((float)y + 0.5f) * s, ((float)z + 0.5f) * s);
  };
  if (blocked(px, py, pz)) return FP_STORED_SOLID;
  uint8_t flags = 0;
  if (!blocked(px + 1, py, pz)) flags |= 1;
  if (!blocked(px - 1, py, pz)) flags |= 2;
  if (!blocked(px, py + 1, pz)) flags |= 4;
  if (!blocked(px, py - 1, pz)) flags |= 8;
  if (!blocked(px, py, pz + 1)) flags |= 16;
  if (!blocked(px, py, pz - 1)) flags |= 32;
  return flags;
}

// buildBrickTopology (pressure.wgsl:259-278): the brick levels of every slotted brick, or of
// the slots granted this step.
__global__ void __launch_bounds__(128) k_topo_bricks(const SimParams* __restrict__ Pp, int all) {
  const SimParams& P = *Pp;
  uint32_t total = all ? (uint32_t)P.capacity * 64u : P.counters->fresh;
  for (uint32_t i = blockIdx.x; i < total; i += gridDim.x) {
    uint32_t id;
    int slot;
    if (all) {
      id = i;
      if (__ldg(&P.tileRec[id >> 6]).w == 0) continue;
      slot = entryPage(P.entries[id]);
    } else {
      id = P.zeroList[2 * i];
      slot = (int)P.zeroList[2 * i + 1];
    }
    if (slot < 0) continue;
    int tile = (int)(id >> 6);
    int4 rec = __ldg(&P.tileRec[tile]);
    Home H = enterTile(P, tile, rec);
    int l = id & 63;
    int bx = rec.x * 4 + (l & 3), by = rec.y * 4 + ((l >> 2) & 3), bz = rec.z * 4 + (l >> 4);
    for (int level = 0; level < P.brickLevels; level++) {
      int s = levelShift(P, level), side = 1 << s, cells = side * side * side;
      for (int o = threadIdx.x; o < cells; o += blockDim.x) {
        int lx = o & (side - 1), ly = (o >> s) & (side - 1), lz = o >> (2 * s);
        P.topo[level][(size_t)slot * cells + o] = cellTopology(P, H, bx * side + lx, by * side + ly, bz * side + lz, level);
      }
    }
  }
}

// buildTileTopology (pressure.wgsl:281-305): every tile's cells at the tile levels.
__global__ void __launch_bounds__(64) k_topo_tiles(const SimParams* __restrict__ Pp) {
  const SimParams& P = *Pp;
  for (int t = blockIdx.x; t < P.capacity; t += gridDim.x) {
    int4 rec = __ldg(&P.tileRec[t]);
    if (rec.w == 0) continue;
    Home H = enterTile(P, t, rec);
    for (int level = P.brickLevels; level <= P.bottom; level++) {
      int s = levelShift(P, level), side = 1 << s, cells = side * side * side;
      for (int o = threadIdx.x; o < cells; o += blockDim.x) {
        int lx = o & (side - 1), ly = (o >> s) & (side - 1), lz = o >> (2 * s);
        P.topo[level][(size_t)t * cells + o] =
            cellTopology(P, H, rec.x * side + lx, rec.y * side + ly, rec.z * side + lz, level);
      }
    }
  }
}

}  // namespace

void fp_launch_topology(const SimParams* dP, int brickLevels, int bottom, bool all, int capacity, int sms,
                        cudaStream_t st) {
  (void)brickLevels;
  (void)bottom;
  k_topo_bricks<<<sms * 4, 128, 0, st>>>(dP, all ? 1 : 0);
  if (all) k_topo_tiles<<<capacity < sms * 8 ? capacity : sms * 8, 64, 0, st>>>(dP);
}

static int tileGrid(int capacity, int sms) { return capacity < sms * 8 ? capacity : sms * 8; }

void fp_launch_relax(const SimParams* dP, int level, bool tiles, const float* rhs, const float* pin, float* pout,
                     int capacity, int sms, cudaStream_t st) {
  Args A{level, rhs, pin, nullptr, pout, nullptr};
  if (tiles)
    k_level_tiles<RELAX><<<tileGrid(capacity, sms), 64, 0, st>>>(dP, A);
  else
    k_level_bricks<RELAX><<<sms * 4, 256, 0, st>>>(dP, A);
}

void fp_launch_restrict(const SimParams* dP, int fine, bool tiles, const float* rhs, const float* p, float* crhs,
                        float* cfirst, int capacity, int sms, cudaStream_t st) {
  Args A{fine + 1, rhs, p, nullptr, crhs, cfirst};
  if (tiles)
    k_level_tiles<RESTRICT><<<tileGrid(capacity, sms), 64, 0, st>>>(dP, A);
  else
    k_level_bricks<RESTRICT><<<sms * 4, 256, 0, st>>>(dP, A);
}

void fp_launch_prolong(const SimParams* dP, int level, bool tiles, const float* pin, const float* coarse, float* pout,
                       int capacity, int sms, cudaStream_t st) {
  Args A{level, nullptr, pin, coarse, pout, nullptr};
  if (tiles)
    k_level_tiles<PROLONG><<<tileGrid(capacity, sms), 64, 0, st>>>(dP, A);
  else
    k_level_bricks<PROLONG><<<sms * 4, 256, 0, st>>>(dP, A);
}

int fp_bottom_capacity() { return (200 * 1024) / 12; }

void fp_launch_bottom(const SimParams* dP, int level, int iterations, const float* rhs, const float* pin, float* pout,
                      int capacity, cudaStream_t st) {
  size_t smem = (size_t)capacity * 12;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    configured = true;
  }
  k_bottom<<<1, 1024, smem, st>>>(dP, level, iterations, rhs, pin, pout);
}
