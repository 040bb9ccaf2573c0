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
    // Multigrid homes are live tiles, and a live tile is its own centre neighbour.
    int tx = px >> s, ty = py >> s, tz = pz >> s;
    int t = (tx == H.tx && ty == H.ty && tz == H.tz && H.tile >= 0) ? H.tile : tileAt(P, H, tx, ty, tz);
    if (t < 0) return -1;
    owner = t;
  }
  return owner * side * side * side + ((pz & m) * side + (py & m)) * side + (px & m);
}

// Whether cell (px,py,pz) of tile level `level` is a pressure unknown: every brick it covers
// computes, from the tile's mask of computing bricks (k_tile_masks, this step).
FP_DEV bool tileCellActive(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  int s = levelShift(P, level), side = 1 << s;
  int tx = px >> s, ty = py >> s, tz = pz >> s;
  int t = (tx == H.tx && ty == H.ty && tz == H.tz && H.tile >= 0) ? H.tile : tileAt(P, H, tx, ty, tz);
  if (t < 0) return false;
  uint64_t m = P.tileMask[t];
  int lx = px & (side - 1), ly = py & (side - 1), lz = pz & (side - 1);
  if (side == 4) return (m >> ((lz * 4 + ly) * 4 + lx)) & 1ull;  // a cell per brick
  if (side == 2) {                                                   // 2^3 bricks a cell
    uint64_t c = 0x0000000000330033ull << (2 * lx + 8 * ly + 32 * lz);
    return (m & c) == c;
  }
  return m == ~0ull;  // the whole tile
}

// activeCell (pressure.wgsl:100-136): whether a level's cell is a pressure unknown.
FP_DEV bool activeCell(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  int bl = P.brickLevels;
  if (level >= bl) return tileCellActive(P, H, px, py, pz, level);  // every covered brick computes
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
// Levels above the finest hold BF16 values in FP_PRECISION_MIXED.
FP_DEV bool narrowLevel(const SimParams& P, int level) { return level > 0 && P.coarseBf16 != 0; }
FP_DEV float readAt(const SimParams& P, const Home& H, const float* arr, int px, int py, int pz, int level) {
  if (!arr) return 0.f;  // a relaxation from zero
  long a = cellAddress(P, H, px, py, pz, level);
  return a < 0 ? 0.f : ldBf(arr, a, narrowLevel(P, level));
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
  bool rhsN, pinN, coarseN, poutN, cfirstN;  // the buffer holds BF16
  bool skip;                                 // a later V-cycle of a converged solve: no work
  int colour;                                // MgSel::colour
};

// A launch names its buffers by selector, level * 4 + which (0 and 1 the level's pressure
// pair, 2 its right-hand side; -1 none), and each simulation of the batch resolves them.
FP_DEV float* mgBuffer(const SimParams& P, int sel) {
  if (sel < 0) return nullptr;
  int level = sel >> 2, which = sel & 3;
  if (which == 2) return level == 0 ? P.div : P.lrhs[level];
  if (which == 3) return level == 0 ? P.kry[0] : nullptr;
  return level == 0 ? P.p0[which] : P.lp[level][which];
}
FP_DEV Args resolve(const SimParams& P, const MgSel& S) {
  Args A;
  A.level = S.level;
  A.rhs = mgBuffer(P, S.rhs);
  A.pin = mgBuffer(P, S.pin);
  A.coarse = mgBuffer(P, S.coarse);
  A.pout = mgBuffer(P, S.pout);
  A.cfirst = mgBuffer(P, S.cfirst);
  A.rhsN = S.rhs >= 0 && narrowLevel(P, S.rhs >> 2);
  A.pinN = S.pin >= 0 && narrowLevel(P, S.pin >> 2);
  A.coarseN = S.coarse >= 0 && narrowLevel(P, S.coarse >> 2);
  A.poutN = S.pout >= 0 && narrowLevel(P, S.pout >> 2);
  A.cfirstN = S.cfirst >= 0 && narrowLevel(P, S.cfirst >> 2);
  A.skip = S.cycle > 0 && P.solver->converged != 0;
  A.colour = S.colour;
  return A;
}

// Red-black: the cell's colour, 0 for x + y + z even.
FP_DEV int parityOf(int px, int py, int pz) { return (px + py + pz) & 1; }

FP_DEV void relaxCell(const SimParams& P, const Home& H, const Args& A, long a, int px, int py, int pz) {
  if (A.colour != 0 && parityOf(px, py, pz) != A.colour - 1) {
    // Red-black, the other colour: kept, or zero when the level starts from zero.
    if (!A.pin) stBf(A.pout, a, 0.f, A.poutN);
    return;
  }
  uint32_t f = expandFlags(P.topo[A.level][a]);
  if ((f & SOLIDF) || !activeCell(P, H, px, py, pz, A.level)) {
    stBf(A.pout, a, 0.f, A.poutN);
    return;
  }
  float sum = A.pin ? stencilSum(P, H, A.pin, px, py, pz, f, A.level) : 0.f;
  float cand = (sum - ldBf(A.rhs, a, A.rhsN)) / fmaxf(diagOf(f), 1e-12f);
  if (A.colour != 0)
    stBf(A.pout, a, cand, A.poutN);  // Gauss-Seidel in place
  else
    stBf(A.pout, a, mixf(A.pin ? ldBf(A.pin, a, A.pinN) : 0.f, cand, 0.8f), A.poutN);
}

FP_DEV void prolongCell(const SimParams& P, const Home& H, const Args& A, long a, int px, int py, int pz) {
  uint32_t f = expandFlags(P.topo[A.level][a]);
  if ((f & SOLIDF) || !activeCell(P, H, px, py, pz, A.level)) {
    stBf(A.pout, a, 0.f, A.poutN);
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
  stBf(A.pout, a, ldBf(A.pin, a, A.pinN) + corr, A.poutN);
}

// restrictCell (pressure.wgsl:601-647): (cx,cy,cz) is a cell of the coarse (output) level.
FP_DEV void restrictCell(const SimParams& P, const Home& H, const Args& A, long out, int cx, int cy, int cz) {
  int fine = A.level - 1;
  float residual = 0.f;
  bool every = true;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int px = cx * 2 + (k & 1), py = cy * 2 + ((k >> 1) & 1), pz = cz * 2 + (k >> 2);
    bool unknown = activeCell(P, H, px, py, pz, fine);
    every = every && unknown;
    if (unknown) {
      long a = cellAddress(P, H, px, py, pz, fine);
      uint32_t f = expandFlags(P.topo[fine][a]);
      if (!(f & SOLIDF)) {
        float sum = stencilSum(P, H, A.pin, px, py, pz, f, fine);
        residual += ldBf(A.rhs, a, A.rhsN) - (sum - diagOf(f) * ldBf(A.pin, a, A.pinN));
      }
    }
  }
  float r = residual * 0.5f;
  stBf(A.pout, out, r, A.poutN);  // the coarse right-hand side
  float first = 0.f;
  if (every) {
    uint32_t f = expandFlags(P.topo[A.level][out]);
    if (!(f & SOLIDF)) first = mixf(0.f, (0.f - r) / fmaxf(diagOf(f), 1e-12f), 0.8f);
  }
  stBf(A.cfirst, out, first, A.cfirstN);
}

template <int OP>
FP_DEV void levelCell(const SimParams& P, const Home& H, const Args& A, long a, int px, int py, int pz) {
  if (OP == RELAX) relaxCell(P, H, A, a, px, py, pz);
  if (OP == PROLONG) prolongCell(P, H, A, a, px, py, pz);
  if (OP == RESTRICT) restrictCell(P, H, A, a, px, py, pz);
}

// Staged brick levels. A CTA copies, for its bricks, the values of the level it reads plus a
// rim into shared memory, and once per brick whether each negative-octant neighbour brick
// computes; the cell operations then read no directory. Same arithmetic, same order as
// relaxCell / restrictCell / prolongCell above.
//   RELAX     stage A.pin at A.level;           write A.pout at A.level
//   RESTRICT  stage A.pin at A.level - 1 (fine); write A.pout, A.cfirst at A.level (coarse)
//   PROLONG   stage A.coarse at A.level + 1;    write A.pout at A.level
// SB, the staged level's cells per brick side, fixes every shape at compile time; SB = 1 is
// the first tile level (one cell per brick), which prolongation stages through the tiles.
template <int OP, int SB>
struct Staged {
  static constexpr int R = OP == PROLONG ? 2 : 1;  // rim: prolongation's Neumann ghosts reach two
  static constexpr int S = SB + 2 * R, S2 = S * S, S3 = S2 * S;
  static constexpr int FS = OP == PROLONG ? 2 * SB : SB;  // the fine level's side
  static constexpr int OS = OP == RESTRICT ? SB / 2 : FS;  // the output level's side
  static constexpr int OUT = OS * OS * OS;
  static constexpr int GROUP = OUT >= 256 ? 256 : (OUT >= 64 ? 64 : 32);  // threads per brick
  static constexpr int NG = 256 / GROUP;                                  // bricks per CTA
  static constexpr int WORDS = S3 + (OP == PROLONG ? (S3 + 3) / 4 : 0);   // values + solid bytes
  static constexpr size_t SMEM = (size_t)NG * WORDS * sizeof(float);
};
constexpr int log2c(int v) { return v <= 1 ? 0 : 1 + log2c(v / 2); }

template <int OP, int SB>
__global__ void __launch_bounds__(256) k_level_bricks_staged(FpBatch bt, MgSel Sl) {
  using K = Staged<OP, SB>;
  constexpr int S = K::S, S2 = K::S2, S3 = K::S3, R = K::R, GROUP = K::GROUP, NG = K::NG;
  constexpr int FS = K::FS, fs = log2c(FS), FCELLS = FS * FS * FS;
  __shared__ int nslotAll[NG][27];
  __shared__ int needAll[NG][8];  // bit k of the index: -1 on axis k
  extern __shared__ float stAll[];
  const int g = threadIdx.x / GROUP, t = threadIdx.x % GROUP;
  int* nslot = nslotAll[g];
  int* need = needAll[g];
  float* st = stAll + g * K::WORDS;
  uint8_t* solidSt = reinterpret_cast<uint8_t*>(st + S3);
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t base = blockIdx.x * NG; base < total; base += gridDim.x * NG) {
    uint32_t item = base + g;
    uint32_t i;
    const SimParams& P = *workSim(bt, FP_WORK_ACTIVE, item < total ? item : base, i).vview;
    const Args A = resolve(P, Sl);
    const bool has = item < total && !A.skip && homeOk(P, P.active[i]);  // homeOk: the bounds-checked build
    const int fineLevel = OP == RESTRICT ? A.level - 1 : A.level;
    const int stageLevel = OP == PROLONG ? A.level + 1 : fineLevel;
    const float* src = OP == PROLONG ? A.coarse : A.pin;
    const bool srcN = OP == PROLONG ? A.coarseN : A.pinN;
    const uint32_t id = has ? P.active[i] : 0u;
    Home H = homeOf(P, id, nslot);
    if (has && t < 27) nslot[t] = checkSlot(P, FP_SITE_RECORD, entryPage(P.records[(size_t)id * FP_RECORD_WORDS + t]));
    __syncthreads();
    const int ox = H.bx * SB - R, oy = H.by * SB - R, oz = H.bz * SB - R;
    // Relaxation and prolongation: this thread's own cells' flags and right-hand side or
    // current value, loaded before the stage so that both sets of loads are in flight together.
    constexpr int K = OP == RESTRICT ? 1 : (FCELLS + GROUP - 1) / GROUP;
    uint8_t ownTopo[K];
    float ownValue[K];
    if (OP != RESTRICT && has) {
      const long slot0 = nslot[13];
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int o = t + k * GROUP;
        if (o < FCELLS) {
          const long a = slot0 * FCELLS + o;
          ownTopo[k] = P.topo[fineLevel][a];
          ownValue[k] = OP == RELAX ? ldBf(A.rhs, a, A.rhsN) : ldBf(A.pin, a, A.pinN);
        }
      }
    }
    bool solidStaged = false;  // prolongation: a solid coarse cell in this thread's stage cells
    if (has) {
      if (t < 8) {
        int dx = -(t & 1), dy = -((t >> 1) & 1), dz = -(t >> 2);
        bool below = P.ground && H.by + dy < 0;
        need[t] = below || nslot[nbrIndex(dx, dy, dz)] >= 0;
      }
      for (int q = t; q < S3; q += GROUP) {
        const int lx = q % S, ly = (q / S) % S, lz = q / S2;
        long a;
        if (SB > 1) {
          // Brick levels: the neighbour brick from the record, the cell within it.
          const int dx = lx < R ? -1 : (lx >= R + SB ? 1 : 0), dy = ly < R ? -1 : (ly >= R + SB ? 1 : 0),
                    dz = lz < R ? -1 : (lz >= R + SB ? 1 : 0);
          const int s = nslot[nbrIndex(dx, dy, dz)];
          const int cx = (lx - R) & (SB - 1), cy = (ly - R) & (SB - 1), cz = (lz - R) & (SB - 1);
          a = s < 0 ? -1 : (long)s * (SB * SB * SB) + (cz * SB + cy) * SB + cx;
        } else {
          a = cellAddress(P, H, ox + lx, oy + ly, oz + lz, stageLevel);
        }
        // A relaxation from zero stages nothing; a red-black half-sweep stages only the other
        // colour (a cell of the colour it writes reads none of its own colour).
        const bool skipLoad = OP == RELAX && (!src || (A.colour != 0 && ((ox + oy + oz + lx + ly + lz) & 1) == A.colour - 1));
        st[q] = (a < 0 || skipLoad) ? 0.f : ldBf(src, a, srcN);
        if (OP == PROLONG) {
          const bool solid = a >= 0 && (P.topo[stageLevel][a] & FP_STORED_SOLID);
          solidSt[q] = solid ? 1 : 0;
          solidStaged = solidStaged || solid;
        }
      }
    }
    // Without a solid coarse cell anywhere in the CTA's stages a Neumann ghost is the staged
    // value itself (coarseValue's first test), so prolongation may read the stage directly.
    bool anySolid = false;
    if (OP == PROLONG)
      anySolid = __syncthreads_or(solidStaged) != 0;
    else
      __syncthreads();
    if (has) {
      // The negative-octant neighbours that compute, as bits; a fine cell on the brick's low
      // faces is an unknown when every neighbour its faces touch computes (activeCell).
      uint32_t needBits = 0;
#pragma unroll
      for (int k = 0; k < 8; k++) needBits |= need[k] ? 1u << k : 0u;
      auto unknown = [&](int lx, int ly, int lz) {
        uint32_t sub = 1u;  // the octants k whose set axes are all on a low face here
        if (lx == 0) sub |= sub << 1;
        if (ly == 0) sub |= sub << 2;
        if (lz == 0) sub |= sub << 4;
        return (~needBits & sub) == 0u;
      };
      // coarseValue (pressure.wgsl:670-696) from the stage.
      auto ghost = [&](int cx, int cy, int cz) {
        int groundY = P.ground ? 0 : -0x7fffffff;
        int c[3] = {cx, max(cy, groundY), cz};
        auto at = [&](int x, int y, int z) { return ((z - oz) * S + (y - oy)) * S + (x - ox); };
        int ci = at(c[0], c[1], c[2]);
        if (!solidSt[ci]) return st[ci];
        float sum = 0.f, count = 0.f;
        for (int axis = 0; axis < 3; axis++)
          for (int side = -1; side <= 1; side += 2) {
            int q[3] = {c[0], c[1], c[2]};
            q[axis] += side;
            q[1] = max(q[1], groundY);
            int qi = at(q[0], q[1], q[2]);
            if (!solidSt[qi]) {
              sum += st[qi];
              count += 1.f;
            }
          }
        return sum / fmaxf(count, 1.f);
      };
      const long slot = nslot[13];
      // Stencil sum of the open sides of a fine cell, from the stage (RELAX, RESTRICT).
      auto sumAt = [&](int lx, int ly, int lz, uint32_t f) {
        int c = ((lz + 1) * S + (ly + 1)) * S + (lx + 1);
        float v0 = (f & 1u) ? st[c + 1] : 0.f, v1 = (f & 2u) ? st[c - 1] : 0.f;
        float v2 = (f & 4u) ? st[c + S] : 0.f, v3 = (f & 8u) ? st[c - S] : 0.f;
        float v4 = (f & 16u) ? st[c + S2] : 0.f, v5 = (f & 32u) ? st[c - S2] : 0.f;
        return (v0 + v1) + (v2 + v3) + (v4 + v5);
      };
      if (OP == RELAX || OP == PROLONG) {
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int o = t + k * GROUP;
          if (o >= FCELLS) break;
          const int lx = o & (FS - 1), ly = (o >> fs) & (FS - 1), lz = o >> (2 * fs);
          const long a = slot * FCELLS + o;
          if (OP == RELAX && A.colour != 0 &&
              ((H.bx * FS + lx + H.by * FS + ly + H.bz * FS + lz) & 1) != A.colour - 1) {
            // Red-black, the other colour: kept, or zero when the level starts from zero.
            if (!src) stBf(A.pout, a, 0.f, A.poutN);
            continue;
          }
          uint32_t f = expandFlags(ownTopo[k]);
          if ((f & SOLIDF) || !unknown(lx, ly, lz)) {
            stBf(A.pout, a, 0.f, A.poutN);
            continue;
          }
          if (OP == RELAX) {
            float cand = (sumAt(lx, ly, lz, f) - ownValue[k]) / fmaxf(diagOf(f), 1e-12f);
            if (A.colour != 0) {
              stBf(A.pout, a, cand, A.poutN);  // Gauss-Seidel in place
            } else {
              float center = st[((lz + 1) * S + (ly + 1)) * S + (lx + 1)];
              stBf(A.pout, a, mixf(center, cand, 0.8f), A.poutN);
            }
          } else {
            int px = H.bx * FS + lx, py = H.by * FS + ly, pz = H.bz * FS + lz;
            float qx = ((float)px + 0.5f) * 0.5f - 0.5f, qy = ((float)py + 0.5f) * 0.5f - 0.5f,
                  qz = ((float)pz + 0.5f) * 0.5f - 0.5f;
            int ix = (int)floorf(qx), iy = (int)floorf(qy), iz = (int)floorf(qz);
            float fx = qx - floorf(qx), fy = qy - floorf(qy), fz = qz - floorf(qz);
            bool fast = (P.colliderCount == 0 || !anySolid) && (!P.ground || iy >= 0);
            // Below the ground the mirrored ghosts read the row above it, which a brick under
            // y = 0 does not stage: those read through the directory.
            bool staged = !(P.ground && H.by < 0);
            float v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
              int dx = q & 1, dy = (q >> 1) & 1, dz = q >> 2;
              v[q] = fast     ? st[((iz + dz - oz) * S + (iy + dy - oy)) * S + (ix + dx - ox)]
                     : staged ? ghost(ix + dx, iy + dy, iz + dz)
                              : coarseValue(P, H, A.coarse, A.level + 1, ix + dx, iy + dy, iz + dz);
            }
            float corr = mixf(mixf(mixf(v[0], v[1], fx), mixf(v[2], v[3], fx), fy),
                              mixf(mixf(v[4], v[5], fx), mixf(v[6], v[7], fx), fy), fz);
            stBf(A.pout, a, ownValue[k] + corr, A.poutN);
          }
        }
      } else {  // RESTRICT: coarse cells of this brick at A.level
        constexpr int cside = FS / 2, cs = fs - 1, ccells = cside * cside * cside;
        for (int o = t; o < ccells; o += GROUP) {
          const int cx = o & (cside - 1), cy = (o >> cs) & (cside - 1), cz = o >> (2 * cs);
          float residual = 0.f;
          bool every = true;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            int lx = cx * 2 + (k & 1), ly = cy * 2 + ((k >> 1) & 1), lz = cz * 2 + (k >> 2);
            bool u = unknown(lx, ly, lz);
            every = every && u;
            if (u) {
              long a = slot * FCELLS + (((lz << fs) | ly) << fs | lx);
              uint32_t f = expandFlags(P.topo[fineLevel][a]);
              if (!(f & SOLIDF)) {
                float center = st[((lz + 1) * S + (ly + 1)) * S + (lx + 1)];
                residual += ldBf(A.rhs, a, A.rhsN) - (sumAt(lx, ly, lz, f) - diagOf(f) * center);
              }
            }
          }
          float r = residual * 0.5f;
          // From the last brick level (2^3 a brick) the coarse level is the first tile level,
          // one cell a brick at the brick's own id (tile slot x 64 + its place in the tile).
          const long out = SB == 2 ? (long)id : slot * ccells + o;
          stBf(A.pout, out, r, A.poutN);
          float first = 0.f;
          if (every) {
            uint32_t f = expandFlags(P.topo[A.level][out]);
            if (!(f & SOLIDF)) first = mixf(0.f, (0.f - r) / fmaxf(diagOf(f), 1e-12f), 0.8f);
          }
          stBf(A.cfirst, out, first, A.cfirstN);
        }
      }
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

// Every cell of `A.level` (a tile level of CELLS cells a tile) in every tile: a thread per
// cell, 64 / CELLS tiles per CTA; no barriers, so threads of dead tiles just move on.
template <int OP, int CELLS>
__global__ void __launch_bounds__(64) k_level_tiles(FpBatch bt, MgSel Sl) {
  constexpr int NT = 64 / CELLS, s = CELLS == 64 ? 2 : (CELLS == 8 ? 1 : 0), side = 1 << s;
  const int g = threadIdx.x / CELLS, o = threadIdx.x % CELLS;
  uint32_t total = workTotal(bt, FP_WORK_TILES);
  for (uint32_t item = blockIdx.x * NT + g; item < total; item += gridDim.x * NT) {
    uint32_t local;
    const SimParams& P = *workSim(bt, FP_WORK_TILES, item, local).vview;
    const int t = P.liveTiles[local];
    const Args A = resolve(P, Sl);
    if (A.skip) continue;
    int4 rec = __ldg(&P.tileRec[t]);
    if (rec.w == 0) continue;
    Home H = enterTile(P, t, rec);
    int lx = o & (side - 1), ly = (o >> s) & (side - 1), lz = o >> (2 * s);
    levelCell<OP>(P, H, A, (long)t * CELLS + o, rec.x * side + lx, rec.y * side + ly, rec.z * side + lz);
  }
}

// Staged tile levels: k_level_bricks_staged with a live tile in place of a brick. A group of 64
// threads copies, for its tile, the values of the level it reads over the tile and a rim from
// the tile's 27 neighbour tiles (tileNbr) into shared memory; a cell is an unknown when its
// brick computes (the tile's mask, tileCellActive). Same arithmetic, same order as relaxCell /
// restrictCell / prolongCell.
//   RELAX     stage A.pin at A.level (TS = 4: the first tile level, a cell a brick)
//   RESTRICT  stage A.pin at A.level - 1 (TS = 4); write A.pout, A.cfirst at A.level (2^3 a tile)
//   PROLONG   stage A.coarse at A.level + 1 (TS = 2); write A.pout at A.level (4^3 a tile)
template <int OP, int TS>
struct TileStaged {
  static constexpr int R = OP == PROLONG ? 2 : 1;  // prolongation's Neumann ghosts reach two
  static constexpr int S = TS + 2 * R, S2 = S * S, S3 = S2 * S;
  static constexpr int FS = OP == PROLONG ? 2 * TS : TS;  // the fine level's side (4: a cell a brick)
  static constexpr int FCELLS = FS * FS * FS;
  static constexpr int GROUP = 64, NG = 4;  // threads per tile, tiles per CTA
  static constexpr int WORDS = S3 + (OP == PROLONG ? (S3 + 3) / 4 : 0);  // values + solid bytes
  static constexpr size_t SMEM = (size_t)NG * WORDS * sizeof(float);
  static_assert(FS == 4 && FCELLS == GROUP, "the fine level is the first tile level, a thread a cell");
};

template <int OP, int TS>
__global__ void __launch_bounds__(256) k_level_tiles_staged(FpBatch bt, MgSel Sl) {
  using K = TileStaged<OP, TS>;
  constexpr int S = K::S, S2 = K::S2, S3 = K::S3, R = K::R, GROUP = K::GROUP, NG = K::NG, FCELLS = K::FCELLS;
  constexpr int TS3 = TS * TS * TS;
  __shared__ int nbrAll[NG][27];
  extern __shared__ float stAll[];
  const int g = threadIdx.x / GROUP, t = threadIdx.x % GROUP;
  int* nbr = nbrAll[g];
  float* st = stAll + g * K::WORDS;
  uint8_t* solidSt = reinterpret_cast<uint8_t*>(st + S3);
  const uint32_t total = workTotal(bt, FP_WORK_TILES);
  for (uint32_t base = blockIdx.x * NG; base < total; base += gridDim.x * NG) {
    const uint32_t item = base + g;
    uint32_t local;
    const SimParams& P = *workSim(bt, FP_WORK_TILES, item < total ? item : base, local).vview;
    const Args A = resolve(P, Sl);
    const int tile = item < total ? P.liveTiles[local] : 0;
    const int4 rec = item < total ? __ldg(&P.tileRec[tile]) : make_int4(0, 0, 0, 0);
    const bool has = item < total && !A.skip && rec.w != 0;
    const int fineLevel = OP == RESTRICT ? A.level - 1 : A.level;
    const int stageLevel = OP == PROLONG ? A.level + 1 : fineLevel;
    const float* src = OP == PROLONG ? A.coarse : A.pin;
    const bool srcN = OP == PROLONG ? A.coarseN : A.pinN;
    if (has && t < 27) nbr[t] = checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[(size_t)tile * 27 + t]));
    __syncthreads();
    // The stage's first cell, in cells of the staged level.
    const int ox = rec.x * TS - R, oy = rec.y * TS - R, oz = rec.z * TS - R;
    // This thread's fine cell (RELAX, PROLONG): its flags and right-hand side or value, loaded
    // before the stage so that both sets of loads are in flight together.
    const long own = (long)tile * FCELLS + t;
    uint8_t ownTopo = 0;
    float ownValue = 0.f;
    if (OP != RESTRICT && has) {
      ownTopo = P.topo[fineLevel][own];
      ownValue = OP == RELAX ? ldBf(A.rhs, own, A.rhsN) : ldBf(A.pin, own, A.pinN);
    }
    bool solidStaged = false;
    if (has) {
      for (int q = t; q < S3; q += GROUP) {
        const int lx = q % S, ly = (q / S) % S, lz = q / S2;
        const int dx = lx < R ? -1 : (lx >= R + TS ? 1 : 0), dy = ly < R ? -1 : (ly >= R + TS ? 1 : 0),
                  dz = lz < R ? -1 : (lz >= R + TS ? 1 : 0);
        const int n = nbr[nbrIndex(dx, dy, dz)];
        const int cx = (lx - R) & (TS - 1), cy = (ly - R) & (TS - 1), cz = (lz - R) & (TS - 1);
        const long a = n < 0 ? -1 : (long)n * TS3 + (cz * TS + cy) * TS + cx;
        const bool skipLoad = OP == RELAX && (!src || (A.colour != 0 && ((ox + oy + oz + lx + ly + lz) & 1) == A.colour - 1));
        st[q] = (a < 0 || skipLoad) ? 0.f : ldBf(src, a, srcN);
        if (OP == PROLONG) {
          const bool solid = a >= 0 && (P.topo[stageLevel][a] & FP_STORED_SOLID);
          solidSt[q] = solid ? 1 : 0;
          solidStaged = solidStaged || solid;
        }
      }
    }
    bool anySolid = false;
    if (OP == PROLONG)
      anySolid = __syncthreads_or(solidStaged) != 0;
    else
      __syncthreads();
    if (has) {
      const uint64_t mask = P.tileMask[tile];
      auto unknown = [&](int lx, int ly, int lz) { return ((mask >> ((lz * 4 + ly) * 4 + lx)) & 1ull) != 0ull; };
      auto sumAt = [&](int lx, int ly, int lz, uint32_t f) {
        int c = ((lz + 1) * S + (ly + 1)) * S + (lx + 1);
        float v0 = (f & 1u) ? st[c + 1] : 0.f, v1 = (f & 2u) ? st[c - 1] : 0.f;
        float v2 = (f & 4u) ? st[c + S] : 0.f, v3 = (f & 8u) ? st[c - S] : 0.f;
        float v4 = (f & 16u) ? st[c + S2] : 0.f, v5 = (f & 32u) ? st[c - S2] : 0.f;
        return (v0 + v1) + (v2 + v3) + (v4 + v5);
      };
      const int lx = t & 3, ly = (t >> 2) & 3, lz = t >> 4;
      const int px = rec.x * 4 + lx, py = rec.y * 4 + ly, pz = rec.z * 4 + lz;
      if (OP == RELAX) {
        if (A.colour != 0 && parityOf(px, py, pz) != A.colour - 1) {
          if (!src) stBf(A.pout, own, 0.f, A.poutN);  // the other colour: kept, or zero from zero
        } else {
          const uint32_t f = expandFlags(ownTopo);
          if ((f & SOLIDF) || !unknown(lx, ly, lz)) {
            stBf(A.pout, own, 0.f, A.poutN);
          } else {
            float cand = (sumAt(lx, ly, lz, f) - ownValue) / fmaxf(diagOf(f), 1e-12f);
            if (A.colour != 0) {
              stBf(A.pout, own, cand, A.poutN);  // Gauss-Seidel in place
            } else {
              float center = st[((lz + 1) * S + (ly + 1)) * S + (lx + 1)];
              stBf(A.pout, own, mixf(center, cand, 0.8f), A.poutN);
            }
          }
        }
      } else if (OP == PROLONG) {
        const uint32_t f = expandFlags(ownTopo);
        if ((f & SOLIDF) || !unknown(lx, ly, lz)) {
          stBf(A.pout, own, 0.f, A.poutN);
        } else {
          float qx = ((float)px + 0.5f) * 0.5f - 0.5f, qy = ((float)py + 0.5f) * 0.5f - 0.5f,
                qz = ((float)pz + 0.5f) * 0.5f - 0.5f;
          int ix = (int)floorf(qx), iy = (int)floorf(qy), iz = (int)floorf(qz);
          float fx = qx - floorf(qx), fy = qy - floorf(qy), fz = qz - floorf(qz);
          bool fast = (P.colliderCount == 0 || !anySolid) && (!P.ground || iy >= 0);
          // Below the ground the mirrored ghosts read the row above it, which a tile under y = 0
          // does not stage: those read through the directory.
          const bool staged = !(P.ground && rec.y < 0);
          auto at = [&](int x, int y, int z) { return ((z - oz) * S + (y - oy)) * S + (x - ox); };
          auto ghost = [&](int cx, int cy, int cz) {
            int groundY = P.ground ? 0 : -0x7fffffff;
            int c[3] = {cx, max(cy, groundY), cz};
            int ci = at(c[0], c[1], c[2]);
            if (!solidSt[ci]) return st[ci];
            float sum = 0.f, count = 0.f;
            for (int axis = 0; axis < 3; axis++)
              for (int side = -1; side <= 1; side += 2) {
                int q[3] = {c[0], c[1], c[2]};
                q[axis] += side;
                q[1] = max(q[1], groundY);
                int qi = at(q[0], q[1], q[2]);
                if (!solidSt[qi]) {
                  sum += st[qi];
                  count += 1.f;
                }
              }
            return sum / fmaxf(count, 1.f);
          };
          float v[8];
#pragma unroll
          for (int q = 0; q < 8; q++) {
            int dx = q & 1, dy = (q >> 1) & 1, dz = q >> 2;
            if (fast) {
              v[q] = st[at(ix + dx, iy + dy, iz + dz)];
            } else if (staged) {
              v[q] = ghost(ix + dx, iy + dy, iz + dz);
            } else {
              Home H = enterTile(P, tile, rec);
              v[q] = coarseValue(P, H, A.coarse, A.level + 1, ix + dx, iy + dy, iz + dz);
            }
          }
          float corr = mixf(mixf(mixf(v[0], v[1], fx), mixf(v[2], v[3], fx), fy),
                            mixf(mixf(v[4], v[5], fx), mixf(v[6], v[7], fx), fy), fz);
          stBf(A.pout, own, ownValue + corr, A.poutN);
        }
      } else if (t < 8) {  // RESTRICT: the tile's 2^3 coarse cells at A.level
        const int cx = t & 1, cy = (t >> 1) & 1, cz = t >> 2;
        float residual = 0.f;
        bool every = true;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          int fx = cx * 2 + (k & 1), fy = cy * 2 + ((k >> 1) & 1), fz = cz * 2 + (k >> 2);
          bool u = unknown(fx, fy, fz);
          every = every && u;
          if (u) {
            long a = (long)tile * FCELLS + ((fz * 4 + fy) * 4 + fx);
            uint32_t f = expandFlags(P.topo[fineLevel][a]);
            if (!(f & SOLIDF)) {
              float center = st[((fz + 1) * S + (fy + 1)) * S + (fx + 1)];
              residual += ldBf(A.rhs, a, A.rhsN) - (sumAt(fx, fy, fz, f) - diagOf(f) * center);
            }
          }
        }
        float r = residual * 0.5f;
        const long out = (long)tile * 8 + t;
        stBf(A.pout, out, r, A.poutN);
        float first = 0.f;
        if (every) {
          uint32_t f = expandFlags(P.topo[A.level][out]);
          if (!(f & SOLIDF)) first = mixf(0.f, (0.f - r) / fmaxf(diagOf(f), 1e-12f), 0.8f);
        }
        stBf(A.cfirst, out, first, A.cfirstN);
      }
    }
    __syncthreads();
  }
}

// relaxCoarse (pressure.wgsl:549-599): the bottom level, one cell per tile slot, every
// iteration in one CTA; a CTA per simulation. The live tiles stride over the threads. When 28
// bytes a live tile fit `smemBytes`, each one's flags (SOLIDF where it is no unknown),
// right-hand side, face neighbours (as live positions) and a ping-pong pair of values live in
// shared memory; else the values ping-pong between the level's two pressure buffers in global
// memory by slot (same arithmetic, same order).
__global__ void __launch_bounds__(1024) k_bottom(FpBatch bt, MgSel Sl, int iterations, int smemBytes) {
  extern __shared__ float bottomSmem[];
  const int nbIndex[6] = {nbrIndex(1, 0, 0), nbrIndex(-1, 0, 0), nbrIndex(0, 1, 0),
                          nbrIndex(0, -1, 0), nbrIndex(0, 0, 1), nbrIndex(0, 0, -1)};
  int sims = batchCount(bt);
  for (int sim = blockIdx.x; sim < sims; sim += gridDim.x) {
    const SimParams& P = *bt.sims[sim].vview;
    const Args A = resolve(P, Sl);
    if (A.skip) continue;  // the same for the whole CTA
    const int level = A.level, L = P.liveCount;
    auto flagOf = [&](int t) -> uint32_t {  // t is live
      int4 rec = __ldg(&P.tileRec[t]);
      Home H = enterTile(P, t, rec);
      return (activeCell(P, H, rec.x, rec.y, rec.z, level) ? expandFlags(P.topo[level][t]) : SOLIDF) | 0x80000000u;
    };
    if ((long)L * 28 <= (long)smemBytes) {
      float* cur = bottomSmem;
      float* nxt = cur + L;
      float* rhs = nxt + L;
      uint32_t* flags = reinterpret_cast<uint32_t*>(rhs + L);
      int16_t* nb = reinterpret_cast<int16_t*>(flags + L);  // 6 a tile
      for (int j = threadIdx.x; j < L; j += blockDim.x) {
        const int t = P.liveTiles[j];
        const uint32_t f = flagOf(t);
        flags[j] = f;
        rhs[j] = ldBf(A.rhs, t, A.rhsN);
        for (int k = 0; k < 6; k++) {
          int n = ((f >> k) & 1u) ? checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[t * 27 + nbIndex[k]])) : -1;
          nb[j * 6 + k] = (int16_t)(n >= 0 ? P.tileIndex[n] : -1);
        }
        // Cells that are no unknown are never read and become zero in the first iteration.
        cur[j] = !(f & SOLIDF) ? ldBf(A.pin, t, A.pinN) : 0.f;
      }
      __syncthreads();
      for (int it = 0; it < iterations; it++) {
        for (int j = threadIdx.x; j < L; j += blockDim.x) {
          const uint32_t f = flags[j];
          float next = 0.f;
          if (!(f & SOLIDF)) {
            float w[6];
#pragma unroll
            for (int k = 0; k < 6; k++) {
              const int n = nb[j * 6 + k];
              w[k] = n >= 0 ? cur[n] : 0.f;
            }
            float sum = (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
            float cand = (sum - rhs[j]) / fmaxf(diagOf(f & 63u), 1e-12f);
            next = mixf(cur[j], cand, 0.8f);
          }
          nxt[j] = next;
        }
        __syncthreads();
        float* tmp = cur;
        cur = nxt;
        nxt = tmp;
      }
      for (int j = threadIdx.x; j < L; j += blockDim.x) stBf(A.pout, P.liveTiles[j], cur[j], A.poutN);
      __syncthreads();
      continue;
    }
    // In global memory: cur starts in pout (a copy of pin), nxt is pin's buffer; both hold the
    // level's storage type.
    float* cur = A.pout;
    float* nxt = const_cast<float*>(A.pin);
    const bool gN = A.poutN;
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
      const int t = P.liveTiles[j];
      const uint32_t f = flagOf(t);
      // pin and pout are the level's two buffers: the copy into pout reads no value it wrote.
      stBf(cur, t, !(f & SOLIDF) ? ldBf(A.pin, t, A.pinN) : 0.f, gN);
    }
    __syncthreads();
    for (int it = 0; it < iterations; it++) {
      for (int j = threadIdx.x; j < L; j += blockDim.x) {
        const int t = P.liveTiles[j];
        const uint32_t f = flagOf(t);
        float next = 0.f;
        if (!(f & SOLIDF)) {
          float w[6];
#pragma unroll
          for (int k = 0; k < 6; k++) {
            int n = ((f >> k) & 1u) ? checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[t * 27 + nbIndex[k]])) : -1;
            w[k] = n >= 0 ? ldBf(cur, n, gN) : 0.f;
          }
          float sum = (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
          float cand = (sum - ldBf(A.rhs, t, A.rhsN)) / fmaxf(diagOf(f & 63u), 1e-12f);
          next = mixf(ldBf(cur, t, gN), cand, 0.8f);
        }
        stBf(nxt, t, next, gN);
      }
      __syncthreads();
      float* tmp = cur;
      cur = nxt;
      nxt = tmp;
    }
    if (cur != A.pout)
      for (int j = threadIdx.x; j < L; j += blockDim.x) {
        const int t = P.liveTiles[j];
        stBf(A.pout, t, ldBf(cur, t, gN), A.poutN);
      }
    __syncthreads();
  }
}

// A value as the storage of a level rounds it.
FP_DEV float bfRound(float v, bool narrow) { return narrow ? __bfloat162float(__float2bfloat16_rn(v)) : v; }

// The second tile level (2^3 cells a tile) and the bottom (one cell a tile) in one CTA per
// simulation: the V-cycle from level bl + 1 down (two relaxations, restriction to the bottom,
// the bottom's iterations, prolongation, three relaxations), with both levels' iterates,
// right-hand sides and flags in shared memory by live tile, __syncthreads between sweeps.
// The arithmetic and its order are those of k_level_tiles (relaxCell, restrictCell,
// prolongCell) and k_bottom; every value a level stores is rounded as its storage rounds it.
//   A.level: level bl + 1; A.rhs its right-hand side; A.pin its first iterate; A.pout where
//   its result goes; A.cfirst: the bottom's result (read back by the prolongation).
constexpr int COARSE_SLOT_BYTES = 8 * 3 * 4 + 8 + 3 * 4 + 4 + 6 * 2 + 27 * 2;  // per live tile
constexpr int COARSE_SMEM = 224 * 1024;
constexpr uint32_t LIVE = 0x80000000u;
constexpr uint8_t UNKNOWN = 0x80;  // level bl + 1 flag byte: activeCell; bit 6 solid; 0-5 open

// The level bl + 1 cell next to cell o of tile t on side k (+x, -x, +y, -y, +z, -z), as an
// index of the level's tile-slot arrays; -1 without a tile there.
// `faces` holds each live tile's six face neighbours as live positions (-1 without one).
FP_DEV int coarseNbr(const int16_t* faces, int j, int o, int k) {
  int l[3] = {o & 1, (o >> 1) & 1, o >> 2};
  const int ax = k >> 1, step = (k & 1) ? -1 : 1;
  int v = l[ax] + step;
  l[ax] = v & 1;
  const int nj = (v < 0 || v > 1) ? faces[j * 6 + k] : j;
  return nj < 0 ? -1 : nj * 8 + ((l[2] * 2 + l[1]) * 2 + l[0]);
}

__global__ void __launch_bounds__(1024) k_coarse(FpBatch bt, MgSel Sl, int iterations) {
  extern __shared__ float coarseSmem[];
  const int nbIndex[6] = {nbrIndex(1, 0, 0), nbrIndex(-1, 0, 0), nbrIndex(0, 1, 0),
                          nbrIndex(0, -1, 0), nbrIndex(0, 0, 1), nbrIndex(0, 0, -1)};
  const int sims = batchCount(bt);
  for (int sim = blockIdx.x; sim < sims; sim += gridDim.x) {
    const SimParams& P = *bt.sims[sim].vview;
    const Args A = resolve(P, Sl);
    if (A.skip) continue;  // the same for the whole CTA
    // Shared arrays by live position j (tile slot P.liveTiles[j]); level L cells at j * 8 + o.
    const int L = A.level, BL = L + 1, nt = P.liveCount, n4 = nt * 8;
    if ((long)nt * COARSE_SLOT_BYTES > COARSE_SMEM) continue;  // the host sizes batches to fit
    const bool nL = narrowLevel(P, L), nB = narrowLevel(P, BL);
    float* pa = coarseSmem;  // level L: iterates, right-hand side
    float* pb = pa + n4;
    float* rh = pb + n4;
    float* ca = rh + n4;  // bottom: iterates, right-hand side
    float* cb = ca + nt;
    float* cr = cb + nt;
    uint32_t* fb = reinterpret_cast<uint32_t*>(cr + nt);
    uint8_t* fl = reinterpret_cast<uint8_t*>(fb + nt);
    int16_t* faces = reinterpret_cast<int16_t*>(fl + n4);  // six a live tile
    // All 27 neighbour tiles of each live tile: the live position, -2 for a tile that is not
    // live (its stored values are read from global memory), -1 for none.
    int16_t* nb27 = faces + nt * 6;
    bool solidNear = false;  // a bottom cell of a neighbour tile is solid
    for (int q = threadIdx.x; q < nt * 27; q += blockDim.x) {
      const int j = q / 27, k = q % 27;
      const int n = checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[P.liveTiles[j] * 27 + k]));
      const int pos = n >= 0 ? P.tileIndex[n] : -1;
      nb27[q] = (int16_t)(n < 0 ? -1 : (pos >= 0 ? pos : -2));
      solidNear = solidNear || (n >= 0 && (P.topo[BL][n] & FP_STORED_SOLID));
      const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
      if ((dx != 0) + (dy != 0) + (dz != 0) == 1) {  // a face: +x, -x, +y, -y, +z, -z
        const int f = dx != 0 ? (dx > 0 ? 0 : 1) : (dy != 0 ? (dy > 0 ? 2 : 3) : (dz > 0 ? 4 : 5));
        faces[j * 6 + f] = (int16_t)pos;
      }
    }
    for (int c = threadIdx.x; c < n4; c += blockDim.x) {
      const int t = P.liveTiles[c >> 3], o = c & 7;
      const long a = (long)t * 8 + o;  // the cell's storage
      int4 rec = __ldg(&P.tileRec[t]);
      Home H = enterTile(P, t, rec);
      int px = rec.x * 2 + (o & 1), py = rec.y * 2 + ((o >> 1) & 1), pz = rec.z * 2 + (o >> 2);
      fl[c] = (uint8_t)(P.topo[L][a] | (activeCell(P, H, px, py, pz, L) ? UNKNOWN : 0));
      pa[c] = ldBf(A.pin, a, nL);
      rh[c] = ldBf(A.rhs, a, nL);
    }
    // Without a solid bottom cell next to any live tile every Neumann ghost of the prolongation
    // is the bottom value itself (coarseValue's first test), read from shared memory.
    const bool anySolid = __syncthreads_or(solidNear) != 0;
    // stencil (pressure.wgsl:360-402) of level L from `src`, cell o of live position j.
    auto sumL = [&](const float* src, int j, int o, uint32_t f) {
      float w[6];
#pragma unroll
      for (int k = 0; k < 6; k++) {
        int n = ((f >> k) & 1u) ? coarseNbr(faces, j, o, k) : -1;
        w[k] = n >= 0 ? src[n] : 0.f;
      }
      return (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
    };
    // relaxCell at level L, src -> dst.
    auto relax = [&](const float* src, float* dst) {
      for (int c = threadIdx.x; c < n4; c += blockDim.x) {
        const uint8_t f = fl[c];
        float v = 0.f;
        if ((f & UNKNOWN) && !(f & FP_STORED_SOLID)) {
          float cand = (sumL(src, c >> 3, c & 7, f & 63u) - rh[c]) / fmaxf(diagOf(f & 63u), 1e-12f);
          v = bfRound(mixf(src[c], cand, 0.8f), nL);
        }
        dst[c] = v;
      }
      __syncthreads();
    };
    relax(pa, pb);
    relax(pb, pa);
    // restrictCell into the bottom (one cell a tile), its first iterate and k_bottom's flags.
    for (int j = threadIdx.x; j < nt; j += blockDim.x) {
      const int t = P.liveTiles[j];
      float r = 0.f, first = 0.f;
      uint32_t f = SOLIDF;
      {
        float residual = 0.f;
        bool every = true;
        for (int k = 0; k < 8; k++) {
          const int c = j * 8 + k;
          const uint8_t fk = fl[c];
          every = every && (fk & UNKNOWN);
          if ((fk & UNKNOWN) && !(fk & FP_STORED_SOLID))
            residual += rh[c] - (sumL(pa, j, k, fk & 63u) - diagOf(fk & 63u) * pa[c]);
        }
        r = residual * 0.5f;
        const uint8_t tb = P.topo[BL][t];
        if (every && !(tb & FP_STORED_SOLID)) first = mixf(0.f, (0.f - r) / fmaxf(diagOf(tb & 63u), 1e-12f), 0.8f);
        // activeCell at the bottom covers the tile's 64 bricks: every cell above is an unknown.
        f = (every ? expandFlags(tb) : SOLIDF) | LIVE;
      }
      cr[j] = bfRound(r, nB);
      ca[j] = !(f & SOLIDF) ? bfRound(first, nB) : 0.f;
      fb[j] = f;
    }
    __syncthreads();
    // relaxCoarse (pressure.wgsl:549-599): FP32 iterates in shared memory.
    float* cur = ca;
    float* nxt = cb;
    for (int it = 0; it < iterations; it++) {
      for (int j = threadIdx.x; j < nt; j += blockDim.x) {
        const uint32_t f = fb[j];
        float next = 0.f;
        if (!(f & SOLIDF)) {
          float w[6];
#pragma unroll
          for (int k = 0; k < 6; k++) {
            const int n = ((f >> k) & 1u) ? faces[j * 6 + k] : -1;
            w[k] = n >= 0 ? cur[n] : 0.f;
          }
          float sum = (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
          float cand = (sum - cr[j]) / fmaxf(diagOf(f & 63u), 1e-12f);
          next = mixf(cur[j], cand, 0.8f);
        }
        nxt[j] = next;
      }
      __syncthreads();
      float* tmp = cur;
      cur = nxt;
      nxt = tmp;
    }
    for (int j = threadIdx.x; j < nt; j += blockDim.x) stBf(A.cfirst, P.liveTiles[j], cur[j], nB);
    __syncthreads();
    // The bottom's stored result at the bottom cell (tile) (dx,dy,dz) from live tile j (slot t):
    // from shared memory as its storage rounds it, from global memory for a tile not live.
    auto bottomNear = [&](int j, int t, int dx, int dy, int dz) {
      const int k = nbrIndex(dx, dy, dz), pos = nb27[j * 27 + k];
      if (pos >= 0) return bfRound(cur[pos], nB);
      if (pos == -1) return 0.f;
      return ldBf(A.cfirst, __ldg(&P.tileNbr[t * 27 + k]), nB);
    };
    // prolongCell at level L from the bottom's stored result, pa -> pb.
    for (int c = threadIdx.x; c < n4; c += blockDim.x) {
      const int t = P.liveTiles[c >> 3], o = c & 7;
      const uint8_t f = fl[c];
      float out = 0.f;
      if ((f & UNKNOWN) && !(f & FP_STORED_SOLID)) {
        int4 rec = __ldg(&P.tileRec[t]);
        Home H = enterTile(P, t, rec);
        int px = rec.x * 2 + (o & 1), py = rec.y * 2 + ((o >> 1) & 1), pz = rec.z * 2 + (o >> 2);
        float qx = ((float)px + 0.5f) * 0.5f - 0.5f, qy = ((float)py + 0.5f) * 0.5f - 0.5f,
              qz = ((float)pz + 0.5f) * 0.5f - 0.5f;
        int ix = (int)floorf(qx), iy = (int)floorf(qy), iz = (int)floorf(qz);
        float fx = qx - floorf(qx), fy = qy - floorf(qy), fz = qz - floorf(qz);
        bool fast = P.colliderCount == 0 && (!P.ground || iy >= 0);
        const int groundY = P.ground ? 0 : -0x7fffffff;
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
          int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
          // The ghost's cell (coarseValue mirrors the ground), next to this tile: no solid cell
          // there, so the ghost and the plain sample are both its value.
          const int ox = ix + dx - rec.x, oy = max(iy + dy, groundY) - rec.y, oz = iz + dz - rec.z;
          const bool near = ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1 && oz >= -1 && oz <= 1;
          v[k] = (!anySolid && near) ? bottomNear(c >> 3, t, ox, oy, oz)
                 : fast              ? readAt(P, H, A.cfirst, ix + dx, iy + dy, iz + dz, BL)
                                     : coarseValue(P, H, A.cfirst, BL, ix + dx, iy + dy, iz + dz);
        }
        float corr = mixf(mixf(mixf(v[0], v[1], fx), mixf(v[2], v[3], fx), fy),
                          mixf(mixf(v[4], v[5], fx), mixf(v[6], v[7], fx), fy), fz);
        out = bfRound(pa[c] + corr, nL);
      }
      pb[c] = out;
    }
    __syncthreads();
    relax(pb, pa);
    relax(pa, pb);
    relax(pb, pa);
    for (int c = threadIdx.x; c < n4; c += blockDim.x) stBf(A.pout, (long)P.liveTiles[c >> 3] * 8 + (c & 7), pa[c], nL);
    __syncthreads();
  }
}

// The finest level's residual rhs - (sum - diag p) over its unknowns, as restrictCell forms
// it, squared and summed in FP64 per simulation.
__global__ void __launch_bounds__(256) k_residual(FpBatch bt, int pSel, int cycle) {
  __shared__ int nslot[27];
  __shared__ double scratch[32];
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = *workSim(bt, FP_WORK_ACTIVE, item, i).vview;
    if (cycle > 0 && P.solver->converged) continue;  // the same for the whole CTA
    if (!homeOk(P, P.active[i])) continue;  // the bounds-checked build only
    Home H = enterBrick(P, P.active[i], nslot);
    const float* p = P.p0[pSel];
    const long slot = nslot[13];
    const int m = P.B - 1;
    double r2 = 0.0, b2 = 0.0, n = 0.0;
    for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
      int x = H.bx * P.B + (c & m), y = H.by * P.B + ((c >> P.shift) & m), z = H.bz * P.B + (c >> (2 * P.shift));
      long a = slot * P.N + c;
      uint32_t f = expandFlags(P.topo[0][a]);
      if ((f & SOLIDF) || !activeCell(P, H, x, y, z, 0)) continue;
      float rhs = P.div[a];
      float r = rhs - (stencilSum(P, H, p, x, y, z, f, 0) - diagOf(f) * p[a]);
      r2 += (double)r * (double)r;
      b2 += (double)rhs * (double)rhs;
      n += 1.0;
    }
    r2 = blockSum(r2, scratch);
    b2 = blockSum(b2, scratch);
    n = blockSum(n, scratch);
    if (threadIdx.x == 0) {
      atomicAdd(&P.solver->res2[cycle], r2);
      if (cycle == 0) {
        atomicAdd(&P.solver->rhs2, b2);
        atomicAdd(&P.solver->unknowns, n);
      }
    }
  }
}

// The red-black bottom (no reference counterpart): `sweeps` red-black Gauss-Seidel sweeps of
// the bottom level (one cell a tile) in place, every sweep the even tiles (x + y + z) then the
// odd ones, in one CTA per simulation. Same cell arithmetic as relaxCell's red-black branch;
// each value is rounded as the level's storage rounds it. With S.pin -1 the level starts from
// zero. Shared memory by live tile when 24 bytes a tile fit, else in place in global memory.
__global__ void __launch_bounds__(1024) k_bottom_rb(FpBatch bt, MgSel Sl, int sweeps, int smemBytes) {
  extern __shared__ float bottomSmem[];
  const int nbIndex[6] = {nbrIndex(1, 0, 0), nbrIndex(-1, 0, 0), nbrIndex(0, 1, 0),
                          nbrIndex(0, -1, 0), nbrIndex(0, 0, 1), nbrIndex(0, 0, -1)};
  constexpr uint32_t ODD = 0x40000000u;
  int sims = batchCount(bt);
  for (int sim = blockIdx.x; sim < sims; sim += gridDim.x) {
    const SimParams& P = *bt.sims[sim].vview;
    const Args A = resolve(P, Sl);
    if (A.skip) continue;  // the same for the whole CTA
    const int level = A.level, L = P.liveCount;
    const bool nB = A.poutN;
    auto flagOf = [&](int t) -> uint32_t {  // t is live
      int4 rec = __ldg(&P.tileRec[t]);
      Home H = enterTile(P, t, rec);
      uint32_t f = activeCell(P, H, rec.x, rec.y, rec.z, level) ? expandFlags(P.topo[level][t]) : SOLIDF;
      return f | (((rec.x + rec.y + rec.z) & 1) ? ODD : 0u);
    };
    if ((long)L * 24 <= (long)smemBytes) {
      float* cur = bottomSmem;
      float* rhs = cur + L;
      uint32_t* flags = reinterpret_cast<uint32_t*>(rhs + L);
      int16_t* nb = reinterpret_cast<int16_t*>(flags + L);  // 6 a tile
      for (int j = threadIdx.x; j < L; j += blockDim.x) {
        const int t = P.liveTiles[j];
        const uint32_t f = flagOf(t);
        flags[j] = f;
        rhs[j] = ldBf(A.rhs, t, A.rhsN);
        for (int k = 0; k < 6; k++) {
          int n = ((f >> k) & 1u) ? checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[t * 27 + nbIndex[k]])) : -1;
          nb[j * 6 + k] = (int16_t)(n >= 0 ? P.tileIndex[n] : -1);
        }
        cur[j] = (A.pin && !(f & SOLIDF)) ? ldBf(A.pin, t, A.pinN) : 0.f;
      }
      __syncthreads();
      for (int it = 0; it < sweeps; it++)
        for (int colour = 0; colour < 2; colour++) {
          for (int j = threadIdx.x; j < L; j += blockDim.x) {
            const uint32_t f = flags[j];
            if ((int)((f & ODD) != 0) != colour) continue;
            float next = 0.f;
            if (!(f & SOLIDF)) {
              float w[6];
#pragma unroll
              for (int k = 0; k < 6; k++) {
                const int n = nb[j * 6 + k];
                w[k] = n >= 0 ? cur[n] : 0.f;
              }
              float sum = (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
              next = bfRound((sum - rhs[j]) / fmaxf(diagOf(f & 63u), 1e-12f), nB);
            }
            cur[j] = next;
          }
          __syncthreads();
        }
      for (int j = threadIdx.x; j < L; j += blockDim.x) stBf(A.pout, P.liveTiles[j], cur[j], nB);
      __syncthreads();
      continue;
    }
    // In place in global memory (A.pout, the level's storage type).
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
      const int t = P.liveTiles[j];
      const uint32_t f = flagOf(t);
      if (!A.pin || (f & SOLIDF)) stBf(A.pout, t, 0.f, nB);
    }
    __syncthreads();
    for (int it = 0; it < sweeps; it++)
      for (int colour = 0; colour < 2; colour++) {
        for (int j = threadIdx.x; j < L; j += blockDim.x) {
          const int t = P.liveTiles[j];
          const uint32_t f = flagOf(t);
          if ((int)((f & ODD) != 0) != colour || (f & SOLIDF)) continue;
          float w[6];
#pragma unroll
          for (int k = 0; k < 6; k++) {
            int n = ((f >> k) & 1u) ? checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[t * 27 + nbIndex[k]])) : -1;
            w[k] = n >= 0 ? ldBf(A.pout, n, nB) : 0.f;
          }
          float sum = (w[0] + w[1]) + (w[2] + w[3]) + (w[4] + w[5]);
          stBf(A.pout, t, (sum - ldBf(A.rhs, t, A.rhsN)) / fmaxf(diagOf(f & 63u), 1e-12f), nB);
        }
        __syncthreads();
      }
  }
}

// ---- Flexible conjugate gradients on the finest level (FP_KRYLOV_FCG; no reference
// counterpart). A v = diag v - (sum of the open neighbours), the operator the relaxation
// inverts; the residual s = rhs + A x has the sign restrictCell's residual has. A CTA per
// computing brick, a thread per cell; FP64 sums per CTA, one double atomic each.
//   begin:     x = p, s = rhs + A p; |s|^2 -> res2[0], |rhs|^2 -> rhs2, unknowns
//   dot:       z.q (the new preconditioned residual against the old A d) -> zq[c]
//   direction: beta = -zq[c] / dq[c-1] (0 at c = 1); d = z + beta d, q = A z + beta q (= A d);
//              d.q -> dq[c], d.s -> ds[c]
//   update:    alpha = -ds[c] / dq[c]; x += alpha d, s += alpha q; |s|^2 -> res2[c]
enum FcgOp { FCG_BEGIN = 0, FCG_DOT = 1, FCG_DIRECTION = 2, FCG_UPDATE = 3 };

template <int OP>
__global__ void __launch_bounds__(256) k_fcg(FpBatch bt, int vSel, int cycle) {
  __shared__ int nslot[27];
  __shared__ double scratch[32];
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = *workSim(bt, FP_WORK_ACTIVE, item, i).vview;
    FpSolver* S = P.solver;
    if (cycle > 0 && S->converged) continue;  // the same for the whole CTA
    if (!homeOk(P, P.active[i])) continue;  // the bounds-checked build only
    Home H = enterBrick(P, P.active[i], nslot);
    const long slot = nslot[13];
    const int m = P.B - 1;
    const float* v = vSel >= 0 ? P.p0[vSel] : nullptr;  // BEGIN: p; DOT, DIRECTION: z
    float* x = P.p0[2];
    float* sres = P.kry[0];
    float* d = P.kry[1];
    float* q = P.kry[2];
    const bool first = cycle <= 1;
    const float beta = (OP == FCG_DIRECTION && !first && S->dq[cycle - 1] != 0.0) ? (float)(-S->zq[cycle] / S->dq[cycle - 1]) : 0.f;
    const float alpha = (OP == FCG_UPDATE && S->dq[cycle] != 0.0) ? (float)(-S->ds[cycle] / S->dq[cycle]) : 0.f;
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
      int px = H.bx * P.B + (c & m), py = H.by * P.B + ((c >> P.shift) & m), pz = H.bz * P.B + (c >> (2 * P.shift));
      long a = slot * P.N + c;
      uint32_t f = expandFlags(P.topo[0][a]);
      bool unknown = !(f & SOLIDF) && activeCell(P, H, px, py, pz, 0);
      if (OP == FCG_BEGIN) {
        float p = v[a];
        x[a] = p;
        float r = 0.f;
        if (unknown) {
          float rhs = P.div[a];
          r = rhs - (stencilSum(P, H, v, px, py, pz, f, 0) - diagOf(f) * p);
          s1 += (double)r * (double)r;
          s2 += (double)rhs * (double)rhs;
          s3 += 1.0;
        }
        sres[a] = r;
      } else if (OP == FCG_DOT) {
        if (unknown) s1 += (double)v[a] * (double)q[a];
      } else if (OP == FCG_DIRECTION) {
        float dn = 0.f, qn = 0.f;
        if (unknown) {
          float z = v[a];
          float az = diagOf(f) * z - stencilSum(P, H, v, px, py, pz, f, 0);
          dn = first ? z : z + beta * d[a];
          qn = first ? az : az + beta * q[a];
          s1 += (double)dn * (double)qn;
          s2 += (double)dn * (double)sres[a];
        }
        d[a] = dn;
        q[a] = qn;
      } else {
        if (unknown) {
          x[a] = x[a] + alpha * d[a];
          float r = sres[a] + alpha * q[a];
          sres[a] = r;
          s1 += (double)r * (double)r;
        }
      }
    }
    s1 = blockSum(s1, scratch);
    if (OP == FCG_BEGIN || OP == FCG_DIRECTION) s2 = blockSum(s2, scratch);
    if (OP == FCG_BEGIN) s3 = blockSum(s3, scratch);
    if (threadIdx.x == 0) {
      if (OP == FCG_BEGIN) {
        atomicAdd(&S->res2[0], s1);
        atomicAdd(&S->rhs2, s2);
        atomicAdd(&S->unknowns, s3);
      } else if (OP == FCG_DOT) {
        atomicAdd(&S->zq[cycle], s1);
      } else if (OP == FCG_DIRECTION) {
        atomicAdd(&S->dq[cycle], s1);
        atomicAdd(&S->ds[cycle], s2);
      } else {
        atomicAdd(&S->res2[cycle], s1);
      }
    }
  }
}

// Each simulation's decision after V-cycle `cycle`: converged once the residual's RMS is at
// most the tolerance times the right-hand side's. One CTA.
__global__ void k_converge(FpBatch bt, int cycle) {
  int sims = batchCount(bt);
  for (int sim = threadIdx.x; sim < sims; sim += blockDim.x) {
    const SimParams& P = *bt.sims[sim].vview;
    FpSolver* S = P.solver;
    if (cycle > 0 && S->converged) continue;
    S->cycles = cycle + 1;
    double tol = (double)P.tolerance;
    // Done: the residual met the tolerance, or this simulation's own cycle limit is reached
    // (the launch runs as many cycles as its most demanding simulation).
    if ((tol > 0.0 && S->res2[cycle] <= tol * tol * S->rhs2) || cycle + 1 >= P.vcycles) S->converged = 1;
  }
}

// cellTopology (pressure.wgsl:208-222): solid, or the sides whose neighbours are not solid.
FP_DEV uint8_t cellTopology(const SimParams& P, const Home& H, int px, int py, int pz, int level) {
  // solidAt at the centre of a level's cell, ((x + .5) s h) / h + .25 with s = 2^level field
  // cells a level-0 cell side (solidSpan), floors to field cell x s + s/2 (x itself for s = 1).
  const int span = (1 << level) * P.solidSpan, half = span >> 1;
  auto blocked = [&](int x, int y, int z) { return solidFine(P, H, x * span + half, y * span + half, z * span + half); };
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

// buildBrickTopology (pressure.wgsl:259-278): the brick levels of the slots granted this
// step, or (ALL) of every slotted brick of the simulations whose geometry changed.
template <bool ALL>
__global__ void __launch_bounds__(128) k_topo_bricks(FpBatch bt) {
  __shared__ int nslot[27];
  // Every slotted brick is on the ascending list of computing bricks.
  const int kind = ALL ? FP_WORK_ACTIVE : FP_WORK_FRESH;
  uint32_t total = workTotal(bt, kind);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = *workSim(bt, kind, item, i).vview;
    if ((P.topoAll != 0) != ALL) continue;  // uniform across the CTA
    uint32_t id;
    int slot;
    if (ALL) {
      id = P.active[i];
      if (__ldg(&P.tileRec[id >> 6]).w == 0) continue;
      slot = entryPage(P.entries[id]);
    } else {
      id = P.zeroList[2 * i];
      slot = (int)P.zeroList[2 * i + 1];
    }
    if (slot < 0) continue;
    // The brick's neighbour slots in shared memory: every solid test stays within them.
    if (!homeOk(P, id)) continue;  // the bounds-checked build only
    Home H = enterBrick(P, id, nslot);
    int bx = H.bx, by = H.by, bz = H.bz;
    // Away from the ground, a brick whose neighbourhood holds no solid cell has every side of
    // every cell open at every brick level: cellTopology would return 63 throughout.
    bool solidNear = P.ground && by == 0;
    if (!solidNear && P.colliderCount > 0) {
      bool any = false;
      for (int q = threadIdx.x; q < 27 * P.W; q += blockDim.x) {
        int s = nslot[q / P.W];
        if (s >= 0 && P.solids[(size_t)s * P.W + q % P.W] != 0u) any = true;
      }
      solidNear = __syncthreads_or(any) != 0;
    }
    if (!solidNear) {
      for (int level = 0; level < P.brickLevels; level++) {
        int s = levelShift(P, level), cells = 1 << (3 * s);
        for (int o = threadIdx.x; o < cells; o += blockDim.x) P.topo[level][(size_t)slot * cells + o] = 63;
      }
      __syncthreads();
      continue;
    }
    for (int level = 0; level < P.brickLevels; level++) {
      int s = levelShift(P, level), side = 1 << s, cells = side * side * side;
      for (int o = threadIdx.x; o < cells; o += blockDim.x) {
        int lx = o & (side - 1), ly = (o >> s) & (side - 1), lz = o >> (2 * s);
        P.topo[level][(size_t)slot * cells + o] = cellTopology(P, H, bx * side + lx, by * side + ly, bz * side + lz, level);
      }
    }
    __syncthreads();
  }
}

// Each tile slot's mask of computing bricks this step (activeCell at the tile levels,
// pressure.wgsl:100-136, asks whether every brick a cell covers has an entry and computes):
// a CTA of 64 threads per tile, a thread per brick.
__global__ void __launch_bounds__(64) k_tile_masks(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_TILES);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t local;
    const SimParams& P = *workSim(bt, FP_WORK_TILES, item, local).vview;
    const int t = P.liveTiles[local];
    const size_t id = (size_t)t * 64 + threadIdx.x;
    const bool slotted = __ldg(&P.tileRec[t]).w != 0 && P.entries[id] >= 0;
    bool on = slotted && P.records[id * FP_RECORD_WORDS + 27] != 0;
    uint32_t half = __ballot_sync(0xffffffffu, on);
    if ((threadIdx.x & 31) == 0) reinterpret_cast<uint32_t*>(P.tileMask)[2 * t + (threadIdx.x >> 5)] = half;
    // The first tile level's right-hand side and first iterate at a brick without a slot: the
    // restriction into that level writes only slotted bricks' cells (no other has an unknown
    // child, so restrictCell would write zero there).
    if (!slotted) {
      const int L = P.brickLevels;
      const bool narrow = narrowLevel(P, L);
      stBf(P.lrhs[L], (long)id, 0.f, narrow);
      stBf(P.lp[L][1], (long)id, 0.f, narrow);
    }
  }
}

// buildTileTopology (pressure.wgsl:281-305): every tile's cells at the tile levels.
__global__ void __launch_bounds__(64) k_topo_tiles(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_TILES);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t local;
    const SimParams& P = *workSim(bt, FP_WORK_TILES, item, local).vview;
    if (!P.topoAll) continue;
    int t = P.liveTiles[local];
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

void fp_launch_topology(const FpBatch& bt, bool anyAll, int sms, cudaStream_t st) {
  k_tile_masks<<<sms * 16, 64, 0, st>>>(bt);
  k_topo_bricks<false><<<sms * 4, 128, 0, st>>>(bt);
  if (anyAll) {
    k_topo_bricks<true><<<sms * 4, 128, 0, st>>>(bt);
    k_topo_tiles<<<sms * 8, 64, 0, st>>>(bt);
  }
}

static const int BOTTOM_SMEM = 200 * 1024;
// Resident CTAs per SM of each staged tile-level instantiation, from the occupancy calculator.
template <int OP, int TS>
static int& tileStagedCtas() {
  static int n = 4;
  return n;
}
template <int OP, int TS>
static void configureTileStaged() {
  using K = TileStaged<OP, TS>;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_level_tiles_staged<OP, TS>, 256, K::SMEM) != cudaSuccess) n = 4;
  tileStagedCtas<OP, TS>() = n > 0 ? n : 1;
}
template <int OP, int TS>
static void tileStagedLaunch(const FpBatch& bt, const MgSel& S, int sms, cudaStream_t st) {
  k_level_tiles_staged<OP, TS><<<sms * tileStagedCtas<OP, TS>(), 256, TileStaged<OP, TS>::SMEM, st>>>(bt, S);
}

// Resident CTAs per SM of each staged instantiation, from the occupancy calculator.
template <int OP, int SB>
static int& stagedCtas() {
  static int n = 4;
  return n;
}
template <int OP, int SB>
static void configureStaged() {
  using K = Staged<OP, SB>;
  cudaFuncSetAttribute(k_level_bricks_staged<OP, SB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_level_bricks_staged<OP, SB>, 256, K::SMEM) != cudaSuccess)
    n = 4;
  stagedCtas<OP, SB>() = n > 0 ? n : 1;
}
void fp_mg_configure(int B) {
  (void)B;
  configureStaged<RELAX, 32>();
  configureStaged<RELAX, 16>();
  configureStaged<RELAX, 8>();
  configureStaged<RELAX, 4>();
  configureStaged<RELAX, 2>();
  configureStaged<RESTRICT, 32>();
  configureStaged<RESTRICT, 16>();
  configureStaged<RESTRICT, 8>();
  configureStaged<RESTRICT, 4>();
  configureStaged<RESTRICT, 2>();
  configureStaged<PROLONG, 16>();
  configureStaged<PROLONG, 8>();
  configureStaged<PROLONG, 4>();
  configureStaged<PROLONG, 2>();
  configureStaged<PROLONG, 1>();
  configureTileStaged<RELAX, 4>();
  configureTileStaged<RESTRICT, 4>();
  configureTileStaged<PROLONG, 2>();
  cudaFuncSetAttribute(k_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, BOTTOM_SMEM);
  cudaFuncSetAttribute(k_bottom_rb, cudaFuncAttributeMaxDynamicSharedMemorySize, BOTTOM_SMEM);
  cudaFuncSetAttribute(k_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, COARSE_SMEM);
}

template <int OP, int SB>
static void stagedLaunch(const FpBatch& bt, const MgSel& S, int sms, cudaStream_t st) {
  k_level_bricks_staged<OP, SB><<<sms * stagedCtas<OP, SB>(), 256, Staged<OP, SB>::SMEM, st>>>(bt, S);
}

// The staged level's cells per brick side for an operation whose output level is `level`,
// in bricks of B velocity cells a side (1: the first tile level).
static int log2i(int v) {
  int s = 0;
  while ((1 << s) < v) s++;
  return s;
}
template <int OP>
static int stagedSide(int level, int B) {
  int bl = log2i(B);
  int stage = OP == PROLONG ? level + 1 : (OP == RESTRICT ? level - 1 : level);
  return stage < bl ? 1 << (bl - stage) : 1;
}

template <int OP>
static void levelLaunch(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st) {
  if constexpr (OP == RESTRICT) {
    // Into the first tile level: a brick's cell there restricts the brick's own 2^3 cells, staged
    // per brick like the brick levels. Cells of bricks without a slot have no unknown child and
    // stay zero (k_tile_masks clears them each step).
    if (tiles && S.level == log2i(B)) {
      stagedLaunch<OP, 2>(bt, S, sms, st);
      return;
    }
  }
  if (tiles) {
    // The tile levels hold 4^3, 2^3 and one cell a tile. Those that read or write the first
    // (a cell a brick) are staged per tile.
    const int below = S.level - log2i(B);
    if (OP == RELAX && below == 0) {
      tileStagedLaunch<RELAX, 4>(bt, S, sms, st);
      return;
    }
    if (OP == RESTRICT && below == 1) {
      tileStagedLaunch<RESTRICT, 4>(bt, S, sms, st);
      return;
    }
    if (OP == PROLONG && below == 0) {
      tileStagedLaunch<PROLONG, 2>(bt, S, sms, st);
      return;
    }
    if (below == 0)
      k_level_tiles<OP, 64><<<sms * 16, 64, 0, st>>>(bt, S);
    else if (below == 1)
      k_level_tiles<OP, 8><<<sms * 16, 64, 0, st>>>(bt, S);
    else
      k_level_tiles<OP, 1><<<sms * 16, 64, 0, st>>>(bt, S);
    return;
  }
  // Relaxation stages sides 32..2, restriction its fine sides 32..4, prolongation 16..1.
  const int sb = stagedSide<OP>(S.level, B);
  if constexpr (OP == RELAX) {
    if (sb == 32) stagedLaunch<OP, 32>(bt, S, sms, st);
    else if (sb == 16) stagedLaunch<OP, 16>(bt, S, sms, st);
    else if (sb == 8) stagedLaunch<OP, 8>(bt, S, sms, st);
    else if (sb == 4) stagedLaunch<OP, 4>(bt, S, sms, st);
    else stagedLaunch<OP, 2>(bt, S, sms, st);
  } else if constexpr (OP == RESTRICT) {
    if (sb == 32) stagedLaunch<OP, 32>(bt, S, sms, st);
    else if (sb == 16) stagedLaunch<OP, 16>(bt, S, sms, st);
    else if (sb == 8) stagedLaunch<OP, 8>(bt, S, sms, st);
    else if (sb == 4) stagedLaunch<OP, 4>(bt, S, sms, st);
    else stagedLaunch<OP, 2>(bt, S, sms, st);
  } else {
    if (sb == 16) stagedLaunch<OP, 16>(bt, S, sms, st);
    else if (sb == 8) stagedLaunch<OP, 8>(bt, S, sms, st);
    else if (sb == 4) stagedLaunch<OP, 4>(bt, S, sms, st);
    else if (sb == 2) stagedLaunch<OP, 2>(bt, S, sms, st);
    else stagedLaunch<OP, 1>(bt, S, sms, st);
  }
}
void fp_launch_relax(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st) {
  levelLaunch<RELAX>(bt, S, tiles, B, sms, st);
}
void fp_launch_restrict(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st) {
  levelLaunch<RESTRICT>(bt, S, tiles, B, sms, st);
}
void fp_launch_prolong(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st) {
  levelLaunch<PROLONG>(bt, S, tiles, B, sms, st);
}
void fp_launch_bottom(const FpBatch& bt, const MgSel& S, int iterations, int sms, cudaStream_t st) {
  k_bottom<<<sms, 1024, BOTTOM_SMEM, st>>>(bt, S, iterations, BOTTOM_SMEM);
}
bool fp_coarse_fits(int liveTiles) { return (long)liveTiles * COARSE_SLOT_BYTES <= COARSE_SMEM; }
void fp_launch_coarse(const FpBatch& bt, const MgSel& S, int iterations, int sms, cudaStream_t st) {
  k_coarse<<<sms, 1024, COARSE_SMEM, st>>>(bt, S, iterations);
}

void fp_launch_residual(const FpBatch& bt, int pSel, int cycle, int sms, cudaStream_t st) {
  k_residual<<<sms * 4, 256, 0, st>>>(bt, pSel, cycle);
  k_converge<<<1, 256, 0, st>>>(bt, cycle);
}

void fp_launch_bottom_rb(const FpBatch& bt, const MgSel& S, int sweeps, int sms, cudaStream_t st) {
  k_bottom_rb<<<sms, 1024, BOTTOM_SMEM, st>>>(bt, S, sweeps, BOTTOM_SMEM);
}

void fp_launch_fcg_begin(const FpBatch& bt, int pSel, int sms, cudaStream_t st) {
  k_fcg<FCG_BEGIN><<<sms * 4, 256, 0, st>>>(bt, pSel, 0);
  k_converge<<<1, 256, 0, st>>>(bt, 0);
}
int fp_fcg_iterate_launches(int cycle) { return cycle > 1 ? 4 : 3; }
void fp_launch_fcg_iterate(const FpBatch& bt, int zSel, int cycle, int sms, cudaStream_t st) {
  if (cycle > 1) k_fcg<FCG_DOT><<<sms * 4, 256, 0, st>>>(bt, zSel, cycle);
  k_fcg<FCG_DIRECTION><<<sms * 4, 256, 0, st>>>(bt, zSel, cycle);
  k_fcg<FCG_UPDATE><<<sms * 4, 256, 0, st>>>(bt, -1, cycle);
  k_converge<<<1, 256, 0, st>>>(bt, cycle);
}
