// Device helpers shared by the step kernels: sparse addressing through the tile directory
// and each brick's 27-neighbour record, trilinear sampling with exact weights, solid tests,
// the emitter, flame and noise functions. Reference semantics are cited per function.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp_types.h"

#define FP_DEV __device__ __forceinline__

// Work lists of a batch (fp_types.h): the simulations in the launch, a list's total, and the
// simulation an item belongs to with the item's index in that simulation's own list.
FP_DEV int batchCount(const FpBatch& b) { return (int)b.work[0]; }
FP_DEV const uint32_t* workRow(const FpBatch& b, int kind) { return b.work + 1 + kind * b.stride; }
FP_DEV uint32_t workTotal(const FpBatch& b, int kind) { return workRow(b, kind)[batchCount(b)]; }
FP_DEV const SimParams& workSim(const FpBatch& b, int kind, uint32_t item, uint32_t& local) {
  const uint32_t* row = workRow(b, kind);
  int lo = 0, hi = batchCount(b) - 1;
  while (lo < hi) {  // the last simulation whose first item is at or before `item`
    int mid = (lo + hi + 1) >> 1;
    if (row[mid] <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  local = item - row[lo];
  return b.sims[lo];
}

// Storage of the scalar pools (FP16 in FP_PRECISION_MIXED) and of the coarse multigrid levels
// (BF16): loads widen to FP32, stores round to nearest even. `narrow` is uniform per launch.
FP_DEV float ldHalf(const float* pool, size_t i, bool narrow) {
  return narrow ? __half2float(reinterpret_cast<const __half*>(pool)[i]) : pool[i];
}
FP_DEV void stHalf(float* pool, size_t i, float v, bool narrow) {
  if (narrow)
    reinterpret_cast<__half*>(pool)[i] = __float2half_rn(v);
  else
    pool[i] = v;
}
FP_DEV float ldBf(const float* p, long i, bool narrow) {
  return narrow ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(p)[i]) : p[i];
}
FP_DEV void stBf(float* p, long i, float v, bool narrow) {
  if (narrow)
    reinterpret_cast<__nv_bfloat16*>(p)[i] = __float2bfloat16_rn(v);
  else
    p[i] = v;
}

// Sum of a double over the CTA (blockDim a multiple of 32, at most 1024), in a fixed order;
// thread 0 holds it. Every thread of the CTA must call it.
FP_DEV double blockSum(double v, double* scratch) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += scratch[w];
  __syncthreads();
  return s;
}

FP_DEV int nbrIndex(int dx, int dy, int dz) { return (dz + 1) * 9 + (dy + 1) * 3 + dx + 1; }
FP_DEV int entryPage(int e) { return e < 0 ? -1 : (e & 0xffffff); }

// The bounds-checked build (FP_BOUNDS, FpBounds in fp_types.h). checkSlot / checkTile pass an
// index read out of a table through when it is -1 (none) or within the table, and otherwise
// record it and return -1, so the access it would have made is skipped. homeOk tells a CTA
// whether its brick id and the brick's own slot are usable; a CTA whose home is not returns
// before any work. Without FP_BOUNDS every check compiles to nothing.
#ifdef FP_BOUNDS
static __device__ __noinline__ void boundsFail(FpBounds* b, int site, long long index, long long limit) {
  if (!b) return;
  if (atomicAdd(&b->count, 1u) == 0u) {
    b->site = site;
    b->index = index;
    b->limit = limit;
  }
}
FP_DEV int checkIndex(const SimParams& P, int site, int v, long long limit) {
  if (v < -1 || (long long)v >= limit) {
    boundsFail(P.bounds, site, v, limit);
    return -1;
  }
  return v;
}
#else
FP_DEV int checkIndex(const SimParams&, int, int v, long long) { return v; }
#endif
FP_DEV int checkSlot(const SimParams& P, int site, int slot) { return checkIndex(P, site, slot, (long long)P.slots); }
FP_DEV int checkTile(const SimParams& P, int site, int tile) { return checkIndex(P, site, tile, (long long)P.capacity); }
FP_DEV bool homeOk(const SimParams& P, uint32_t id) {
#ifdef FP_BOUNDS
  if ((long long)id >= (long long)P.capacity * 64) {
    boundsFail(P.bounds, FP_SITE_BRICK_ID, id, (long long)P.capacity * 64);
    return false;
  }
  return checkSlot(P, FP_SITE_ENTRY, entryPage(P.entries[id])) >= 0;
#else
  (void)P;
  (void)id;
  return true;
#endif
}

// tileHash (tiles.wgsl:166-169).
FP_DEV uint32_t tileHash(int x, int y, int z) {
  return ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349663u) ^ ((uint32_t)z * 83492791u);
}
// findTile (tiles.wgsl:172-187): the slot of tile t, or -1. The table is at most half full.
FP_DEV int hashFind(const SimParams& P, int x, int y, int z) {
  uint32_t mask = P.hashMask;
  uint32_t h = tileHash(x, y, z) & mask;
  for (uint32_t probe = 0; probe <= mask; probe++) {
    int4 e = __ldg(&P.hash[h]);
    if (e.w < 0) break;
    if (e.x == x && e.y == y && e.z == z) return checkTile(P, FP_SITE_HASH, e.w);
    h = (h + 1) & mask;
  }
  return -1;
}

// Where a CTA works: its home brick, whose 27 neighbour slots sit in shared memory, and the
// home tile, whose 27 neighbour tiles are in tileNbr (tiles.wgsl:211-295).
struct Home {
  int bx, by, bz;    // home brick
  int tx, ty, tz;    // home tile
  int tile;          // home tile slot, -1 without one
  const int* nslot;  // shared: slot of each of the 27 neighbour bricks, or -1
};

FP_DEV int tileAt(const SimParams& P, const Home& H, int x, int y, int z) {
  if (H.tile >= 0) {
    int dx = x - H.tx, dy = y - H.ty, dz = z - H.tz;
    if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1)
      return checkTile(P, FP_SITE_TILE_NBR, __ldg(&P.tileNbr[H.tile * 27 + nbrIndex(dx, dy, dz)]));
  }
  return hashFind(P, x, y, z);
}
FP_DEV int brickIdAt(const SimParams& P, const Home& H, int bx, int by, int bz) {
  int t = tileAt(P, H, bx >> 2, by >> 2, bz >> 2);
  if (t < 0) return -1;
  return t * 64 + (((bz & 3) * 4 + (by & 3)) * 4 + (bx & 3));
}
// The entry of world brick b (tiles.wgsl:275-290), through the directory.
FP_DEV int brickEntryG(const SimParams& P, const Home& H, int bx, int by, int bz) {
  int id = brickIdAt(P, H, bx, by, bz);
  return id < 0 ? -1 : P.entries[id];
}
// The slot of world brick b, or -1 without one.
FP_DEV int brickSlot(const SimParams& P, const Home& H, int bx, int by, int bz) {
  int dx = bx - H.bx, dy = by - H.by, dz = bz - H.bz;
  if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) return H.nslot[nbrIndex(dx, dy, dz)];
  return checkSlot(P, FP_SITE_ENTRY, entryPage(brickEntryG(P, H, bx, by, bz)));
}
FP_DEV int localCell(const SimParams& P, int x, int y, int z) {
  int m = P.B - 1;
  return (((z & m) << P.shift | (y & m)) << P.shift) | (x & m);
}
// Cell (x,y,z) of a pool of `ch` channels: zero in a brick without a slot
// (fluid-sampling.wgsl:68-75).
FP_DEV float cellAt(const SimParams& P, const Home& H, const float* pool, int ch, int c, int x, int y, int z,
                    bool half = false) {
  int s = brickSlot(P, H, x >> P.shift, y >> P.shift, z >> P.shift);
  if (s < 0) return 0.f;
  return ldHalf(pool, ((size_t)s * ch + c) * P.N + localCell(P, x, y, z), half);
}

// a + t (b - a): exact at t = 0 and wherever a == b, so a constant field samples exactly.
FP_DEV float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }
// Trilinear blend of the 2x2x2 corner values t (x fastest, then y, then z).
FP_DEV float blend8(const float* t, float fx, float fy, float fz) {
  return lerpf(lerpf(lerpf(t[0], t[1], fx), lerpf(t[2], t[3], fx), fy),
               lerpf(lerpf(t[4], t[5], fx), lerpf(t[6], t[7], fx), fy), fz);
}

// Trilinear sample of one channel at `pos` in cell units, centres at .5
// (fluid-sampling.wgsl:85-114): bricks without a slot read zero.
FP_DEV float sampleCells(const SimParams& P, const Home& H, const float* pool, int ch, int c, float px, float py,
                         float pz, bool half = false) {
  float qx = px - 0.5f, qy = py - 0.5f, qz = pz - 0.5f;
  int x0 = (int)floorf(qx), y0 = (int)floorf(qy), z0 = (int)floorf(qz);
  float fx = qx - (float)x0, fy = qy - (float)y0, fz = qz - (float)z0;
  int sh = P.shift;
  int bx0 = x0 >> sh, bx1 = (x0 + 1) >> sh, by0 = y0 >> sh, by1 = (y0 + 1) >> sh, bz0 = z0 >> sh,
      bz1 = (z0 + 1) >> sh;
  float t[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    int dx = j & 1, dy = (j >> 1) & 1, dz = j >> 2;
    int s = brickSlot(P, H, dx ? bx1 : bx0, dy ? by1 : by0, dz ? bz1 : bz0);
    t[j] = s < 0 ? 0.f : ldHalf(pool, ((size_t)s * ch + c) * P.N + localCell(P, x0 + dx, y0 + dy, z0 + dz), half);
  }
  return blend8(t, fx, fy, fz);
}

// velocityCellAverage (fluid-sampling.wgsl:268-285): the mean of the field cells under velocity
// cell (x,y,z) when the velocity divisor d is above 1, through the field view F: a trilinear
// sample on the shared corner of a 2x2x2 block of field cells is that block's mean.
static __device__ __noinline__ float fieldAverage(const SimParams& F, const Home& H, const float* pool, int ch, int c, int x,
                                           int y, int z, bool half) {
  const int d = F.velDiv, blocks = d >> 1;
  float sum = 0.f;
  for (int k = 0; k < blocks; k++)
    for (int j = 0; j < blocks; j++)
      for (int i = 0; i < blocks; i++)
        sum += sampleCells(F, H, pool, ch, c, (float)(x * d + 1 + 2 * i), (float)(y * d + 1 + 2 * j),
                           (float)(z * d + 1 + 2 * k), half);
  return sum / (float)(blocks * blocks * blocks);
}

// The coarse smoke grid (fluid-sampling.wgsl:4-20: every grid shares the brick footprint with
// its own cells a side, here 2^P.smokeShift): cell (x,y,z) of a [slot][smokeCells] pool, zero
// in a brick without a slot, and the trilinear sample at `q` in its cells, centres at .5.
FP_DEV float smokeCell(const SimParams& P, const Home& H, const float* pool, int x, int y, int z, bool half) {
  const int sh = P.smokeShift, m = (1 << sh) - 1;
  int s = brickSlot(P, H, x >> sh, y >> sh, z >> sh);
  if (s < 0) return 0.f;
  return ldHalf(pool, (size_t)s * P.smokeCells + ((((z & m) << sh) | (y & m)) << sh | (x & m)), half);
}
FP_DEV float smokeSample(const SimParams& P, const Home& H, const float* pool, float px, float py, float pz,
                         bool half) {
  float qx = px - 0.5f, qy = py - 0.5f, qz = pz - 0.5f;
  float gx = floorf(qx), gy = floorf(qy), gz = floorf(qz);
  int x0 = (int)gx, y0 = (int)gy, z0 = (int)gz;
  float t[8];
#pragma unroll
  for (int j = 0; j < 8; j++) t[j] = smokeCell(P, H, pool, x0 + (j & 1), y0 + ((j >> 1) & 1), z0 + (j >> 2), half);
  return blend8(t, qx - gx, qy - gy, qz - gz);
}

// meshSourceAt (fluid-sources.wgsl:9-22) for field cell (x,y,z): its mesh emission record,
// or null where none (record 0, all zero, changes nothing).
FP_DEV const FpMeshSource* meshSourceAt(const SimParams& P, const Home& H, int x, int y, int z) {
  if (P.meshCount == 0) return nullptr;
  int id = brickIdAt(P, H, x >> P.shift, y >> P.shift, z >> P.shift);
  if (id < 0) return nullptr;
  int table = P.meshTables[id];
  if (table < 0) return nullptr;
  const int m = P.B - 1, sh = P.shift;
  size_t index = (((((size_t)table << sh) | (size_t)(z & m)) << sh | (size_t)(y & m)) << sh) | (size_t)(x & m);
  int r = P.meshTables[(size_t)P.capacity * 64 + index];
  return r > 0 ? &P.meshSources[r] : nullptr;
}

// solidCell (solids.wgsl:15-31) of field cell (x,y,z): the ground, then colliders drawn into
// each slot's bits.
FP_DEV bool solidFine(const SimParams& P, const Home& H, int x, int y, int z) {
  if (P.ground && y < 0) return true;
  if (P.colliderCount == 0) return false;
  const int fs = P.fshift, m = (1 << fs) - 1;
  int s = brickSlot(P, H, x >> fs, y >> fs, z >> fs);
  if (s < 0) return false;
  int bit = (((z & m) << fs | (y & m)) << fs) | (x & m);
  return ((P.solids[(size_t)s * P.W + (bit >> 5)] >> (bit & 31)) & 1u) != 0u;
}
// The same on a coarser lattice of s field cells a side (solidSpan): the field cell under its
// centre. Out of line: only the velocity view of a divided lattice calls it.
static __device__ __noinline__ bool solidScaled(const SimParams& P, const Home& H, int x, int y, int z) {
  const int s = P.solidSpan, o = s >> 1;
  return solidFine(P, H, x * s + o, y * s + o, z * s + o);
}
// solidAt at the centre of cell (x,y,z) of this lattice: ((x + .5) s h) / h + .25 floors to
// field cell x s + s/2 (s = solidSpan; x itself on the field lattice).
// ONE: this view is known at compile time to be the field lattice (velocity divisor 1).
template <bool ONE = false>
FP_DEV bool solidCell(const SimParams& P, const Home& H, int x, int y, int z) {
  if (!ONE && P.solidSpan > 1) return solidScaled(P, H, x, y, z);
  // this view is the field lattice
  if (P.ground && y < 0) return true;
  if (P.colliderCount == 0) return false;
  int s = brickSlot(P, H, x >> P.shift, y >> P.shift, z >> P.shift);
  if (s < 0) return false;
  int bit = localCell(P, x, y, z);
  return ((P.solids[(size_t)s * P.W + (bit >> 5)] >> (bit & 31)) & 1u) != 0u;
}
// fieldCell (solids.wgsl:7-9) and solidAt (:33-35).
FP_DEV bool solidAt(const SimParams& P, const Home& H, float wx, float wy, float wz) {
  return solidFine(P, H, (int)floorf(wx / P.fineH + 0.25f), (int)floorf(wy / P.fineH + 0.25f),
                   (int)floorf(wz / P.fineH + 0.25f));
}

FP_DEV float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }
FP_DEV float clamp01(float x) { return fminf(fmaxf(x, 0.f), 1.f); }
FP_DEV float smooth(float e0, float e1, float x) {
  float t = clamp01((x - e0) / (e1 - e0));
  return t * t * (3.f - 2.f * t);
}

// The home tile's list of `kind`: first index and count (fluid-common.wgsl:88-95).
FP_DEV uint2 tileList(const SimParams& P, int tile, int kind) {
  const uint32_t* h = P.tileLists + tile * 8 + kind * 2;
  return make_uint2(__ldg(h), __ldg(h + 1));
}

// emitterWeight (fluid-sources.wgsl:24-37).
FP_DEV float emitterWeight(const FpEmitter& e, float px, float py, float pz) {
  float dx = (px - e.pos[0]) / fmaxf(e.size[0], 0.03f), dy = (py - e.pos[1]) / fmaxf(e.size[1], 0.03f),
        dz = (pz - e.pos[2]) / fmaxf(e.size[2], 0.03f);
  float r = e.box > 0.5f ? fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))) : sqrtf(dx * dx + dy * dy + dz * dz);
  if (r >= 1.f || e.enabled < 0.5f) return 0.f;
  return 1.f - smooth(0.5f, 1.f, r);
}

// burstGradient / burstPerlin / burstPattern (fluid-sources.wgsl:41-71).
FP_DEV float burstGradient(int cx, int cy, int cz, float ox, float oy, float oz, uint32_t seed) {
  uint32_t h = (uint32_t)cx * 374761393u + (uint32_t)cy * 668265263u + (uint32_t)cz * 2246822519u + seed * 3266489917u;
  h = (h ^ (h >> 13u)) * 1274126177u;
  h = (h ^ (h >> 16u)) & 15u;
  float a = h < 8u ? ox : oy;
  float b = h < 4u ? oy : ((h == 12u || h == 14u) ? ox : oz);
  return ((h & 1u) == 0u ? a : -a) + ((h & 2u) == 0u ? b : -b);
}
FP_DEV float burstPerlin(float px, float py, float pz, uint32_t seed) {
  int cx = (int)floorf(px), cy = (int)floorf(py), cz = (int)floorf(pz);
  float fx = px - floorf(px), fy = py - floorf(py), fz = pz - floorf(pz);
  float sx = fx * fx * fx * (fx * (fx * 6.f - 15.f) + 10.f), sy = fy * fy * fy * (fy * (fy * 6.f - 15.f) + 10.f),
        sz = fz * fz * fz * (fz * (fz * 6.f - 15.f) + 10.f);
  float a = burstGradient(cx, cy, cz, fx, fy, fz, seed);
  float b = burstGradient(cx + 1, cy, cz, fx - 1, fy, fz, seed);
  float c = burstGradient(cx, cy + 1, cz, fx, fy - 1, fz, seed);
  float d = burstGradient(cx + 1, cy + 1, cz, fx - 1, fy - 1, fz, seed);
  float e = burstGradient(cx, cy, cz + 1, fx, fy, fz - 1, seed);
  float g = burstGradient(cx + 1, cy, cz + 1, fx - 1, fy, fz - 1, seed);
  float hh = burstGradient(cx, cy + 1, cz + 1, fx, fy - 1, fz - 1, seed);
  float j = burstGradient(cx + 1, cy + 1, cz + 1, fx - 1, fy - 1, fz - 1, seed);
  return mixf(mixf(mixf(a, b, sx), mixf(c, d, sx), sy), mixf(mixf(e, g, sx), mixf(hh, j, sx), sy), sz);
}
FP_DEV float burstPattern(float px, float py, float pz, uint32_t seed) {
  float n = (burstPerlin(px, py, pz, seed) + 0.35f * burstPerlin(px * 2.f + 5.2f, py * 2.f + 9.7f, pz * 2.f + 3.1f, seed)) /
            1.35f;
  return clamp01(0.5f + 0.5f * n);
}
// burstVariation (fluid-sources.wgsl:73-82): heat and lifetime multipliers.
FP_DEV float2 burstVariation(const FpEmitter& e, float px, float py, float pz, uint32_t seed) {
  if (e.strength == 0.f) return make_float2(1.f, 1.f);
  float qx = (px - e.pos[0]) / e.period + 3.17f, qy = (py - e.pos[1]) / e.period + 7.53f,
        qz = (pz - e.pos[2]) / e.period + 11.29f;
  return make_float2(1.f - e.strength * burstPattern(qx, qy, qz, seed),
                     1.f - e.strength * burstPattern(qx + 17.3f, qy + 2.8f, qz + 8.6f, seed));
}

// rampIntegral / evaluateFlame (flame-common.wgsl:14-42).
FP_DEV float rampIntegral(const FpFlame& F, int ch, float lo, float hi) {
  float area = 0.f;
  for (int i = 1; i < F.counts[ch]; i++) {
    float ax = F.knots[ch][i - 1][0], ay = F.knots[ch][i - 1][1], bx = F.knots[ch][i][0], by = F.knots[ch][i][1];
    float left = fmaxf(lo, ax), right = fminf(hi, bx);
    if (right > left) {
      float y0 = mixf(ay, by, (left - ax) / (bx - ax));
      float y1 = mixf(ay, by, (right - ax) / (bx - ax));
      area += (right - left) * (y0 + y1) * 0.5f;
    }
  }
  return area;
}

// curlNoise (fluid-forces.wgsl:3-9): repeat-addressed trilinear fetch of the 64^3 table,
// rotated in and out.
FP_DEV float3 curlNoise(const SimParams& P, float px, float py, float pz) {
  // rotation columns (.36,-.8,.48), (.48,.6,.64), (-.8,0,.6)
  float u = (0.36f * px + 0.48f * py + -0.8f * pz) / 16.f;
  float v = (-0.8f * px + 0.6f * py + 0.f * pz) / 16.f;
  float w = (0.48f * px + 0.64f * py + 0.6f * pz) / 16.f;
  float tx = u * 64.f - 0.5f, ty = v * 64.f - 0.5f, tz = w * 64.f - 0.5f;
  int ix = (int)floorf(tx), iy = (int)floorf(ty), iz = (int)floorf(tz);
  float fx = tx - floorf(tx), fy = ty - floorf(ty), fz = tz - floorf(tz);
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
  for (int dz = 0; dz < 2; dz++)
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
      for (int dx = 0; dx < 2; dx++) {
        float wt = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
        float4 n = __ldg(&P.noise[(((iz + dz) & 63) * 64 + ((iy + dy) & 63)) * 64 + ((ix + dx) & 63)]);
        sx += n.x * wt;
        sy += n.y * wt;
        sz += n.z * wt;
      }
  // transpose(rotation) * s: the dot of each column with s.
  return make_float3(0.36f * sx + -0.8f * sy + 0.48f * sz, 0.48f * sx + 0.6f * sy + 0.64f * sz,
                     -0.8f * sx + 0.f * sy + 0.6f * sz);
}

// Load a brick's home record (its 27 neighbour entries) into shared memory as slots.
// Every thread of the block must call this.
// The home brick and tile of brick `id`; `nslot` is filled by the caller.
FP_DEV Home homeOf(const SimParams& P, uint32_t id, const int* nslot) {
  Home H;
  int tile = (int)(id >> 6);
  int4 t = __ldg(&P.tileRec[tile]);
  int l = id & 63;
  H.tile = tile;
  H.tx = t.x;
  H.ty = t.y;
  H.tz = t.z;
  H.bx = t.x * 4 + (l & 3);
  H.by = t.y * 4 + ((l >> 2) & 3);
  H.bz = t.z * 4 + (l >> 4);
  H.nslot = nslot;
  return H;
}

FP_DEV Home enterBrick(const SimParams& P, uint32_t id, int* nslot) {
  Home H;
  int tile = (int)(id >> 6);
  int4 t = __ldg(&P.tileRec[tile]);
  int l = id & 63;
  H.tile = tile;
  H.tx = t.x;
  H.ty = t.y;
  H.tz = t.z;
  H.bx = t.x * 4 + (l & 3);
  H.by = t.y * 4 + ((l >> 2) & 3);
  H.bz = t.z * 4 + (l >> 4);
  H.nslot = nslot;
  if (threadIdx.x < 27)
    nslot[threadIdx.x] = checkSlot(P, FP_SITE_RECORD, entryPage(P.records[(size_t)id * FP_RECORD_WORDS + threadIdx.x]));
  __syncthreads();
  return H;
}
