// Volume rendering of a simulation's state, headless: restates the renderer's compute passes
// (src/engine/shaders/lighting.wgsl smoothSmoke 69-99, buildOccupancy 149-244, incidentLight
// 257-310, lightSlot 312-347) and the camera march (volume-march.wgsl fireProRay 18-24,
// fireProHit 28-35, fireProStep 77-79, fireProJitter 94-102, fireProShade 106-138,
// fireProDirect 141-146, fireProMarch 178-268; scene-volume.wgsl 39-44 and 160-167 with no
// scene depth and half resolution off), the optical model (fire-emission.wgsl) and the
// reconstruction filters (volume-reconstruction.wgsl).
//
// Where the reference reads a pool slot's apron (a copy of the +1 neighbours), these kernels
// read the neighbour's slot; a neighbour without a slot reads what the apron would hold: the
// smoothed density computed on the spot for the render field, the incident light computed on
// the spot for the lighting pool. The render marches one box per cluster of tiles that holds
// content or sources (FluidSimulation.ts:916-957, TileDirectory.ts:189-245): a sample reads the
// pages of the box it lies in only, clamped to that box, and a ray crosses the boxes in order
// (volume-march.wgsl fireProSpan, fireProNext, fireProEnter).
#include "fp_device.cuh"
#include "fp_render.h"

namespace {

constexpr int RTHREADS = 128;

// A thread's current box (the pages its samples read) and its last two brick lookups (samples
// near a brick's face alternate between two bricks).
struct SlotCache {
  int bx, by, bz, slot;
  int bx2, by2, bz2, slot2;
  int lo[3], hi[3];  // the current box in bricks, inclusive
};
FP_DEV SlotCache noBox() {
  SlotCache c;
  c.bx = c.bx2 = 1 << 30;
  c.by = c.bz = c.by2 = c.bz2 = 0;
  c.slot = c.slot2 = -1;
  for (int a = 0; a < 3; a++) {
    c.lo[a] = 0;
    c.hi[a] = -1;
  }
  return c;
}
// Box k becomes the current one; the lookup cache starts over (pages are per box).
FP_DEV void useBox(const FpRender& R, SlotCache& c, int k) {
  for (int a = 0; a < 3; a++) {
    c.lo[a] = R.boxes[6 * k + a];
    c.hi[a] = R.boxes[6 * k + 3 + a];
  }
  c.bx = c.bx2 = 1 << 30;
}
FP_DEV bool inBox(const SlotCache& c, int bx, int by, int bz) {
  return bx >= c.lo[0] && bx <= c.hi[0] && by >= c.lo[1] && by <= c.hi[1] && bz >= c.lo[2] && bz <= c.hi[2];
}
// fireProPage: the slot of world brick b inside the current box, or -1.
FP_DEV int slotAt(const SimParams& P, const FpRender& R, SlotCache& c, int bx, int by, int bz) {
  if (bx == c.bx && by == c.by && bz == c.bz) return c.slot;
  if (bx == c.bx2 && by == c.by2 && bz == c.bz2) return c.slot2;
  c.bx2 = c.bx;
  c.by2 = c.by;
  c.bz2 = c.bz;
  c.slot2 = c.slot;
  int s = -1;
  if (inBox(c, bx, by, bz)) {
    int t = hashFind(P, bx >> 2, by >> 2, bz >> 2);
    if (t >= 0) s = checkSlot(P, FP_SITE_ENTRY, entryPage(P.entries[t * 64 + (((bz & 3) * 4 + (by & 3)) * 4 + (bx & 3))]));
  }
  c.bx = bx;
  c.by = by;
  c.bz = bz;
  c.slot = s;
  return s;
}

FP_DEV float glowOf(float life) { return fminf(fmaxf(life * 5.f, 0.f), 1.f); }  // fireProGlow

// The simulation's smoke at a world cell: zero outside the box or without a slot.
FP_DEV float rawSmoke(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z) {
  int s = slotAt(P, R, c, x >> P.shift, y >> P.shift, z >> P.shift);
  if (s < 0) return 0.f;
  return ldHalf(P.fld, (size_t)s * 4 * P.N + localCell(P, x, y, z), P.scalarHalf != 0);
}
// fireProField of the smoke at `q` in cells: clamped to the box, trilinear.
FP_DEV float smokeSample(const SimParams& P, const FpRender& R, SlotCache& c, float qx, float qy, float qz) {
  float B = (float)P.B;
  qx = fminf(fmaxf(qx, (float)c.lo[0] * B + .5f), (float)(c.hi[0] + 1) * B - .5f);
  qy = fminf(fmaxf(qy, (float)c.lo[1] * B + .5f), (float)(c.hi[1] + 1) * B - .5f);
  qz = fminf(fmaxf(qz, (float)c.lo[2] * B + .5f), (float)(c.hi[2] + 1) * B - .5f);
  float gx = qx - .5f, gy = qy - .5f, gz = qz - .5f;
  int x0 = (int)floorf(gx), y0 = (int)floorf(gy), z0 = (int)floorf(gz);
  float fx = gx - (float)x0, fy = gy - (float)y0, fz = gz - (float)z0;
  float v = 0.f;
  for (int k = 0; k < 8; k++) {
    int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
    float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
    v += rawSmoke(P, R, c, x0 + dx, y0 + dy, z0 + dz) * w;
  }
  return v;
}
// smoothSmoke's [1,2,1]/4 density at a world cell: eight half-offset samples.
FP_DEV float smoothedSmoke(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z) {
  float d = 0.f;
  for (int k = 0; k < 8; k++)
    d += smokeSample(P, R, c, (float)(x + (k & 1)), (float)(y + ((k >> 1) & 1)), (float)(z + (k >> 2)));
  return fmaxf(0.f, d * .125f);
}

// The coarse smoke grid (smoke_divisor d > 1): 2^P.smokeShift cells a brick side.
// The simulation's coarse density at a coarse cell: zero outside the box or without a slot.
FP_DEV float rawCoarse(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z) {
  const int sh = P.smokeShift, m = (1 << sh) - 1;
  int s = slotAt(P, R, c, x >> sh, y >> sh, z >> sh);
  if (s < 0) return 0.f;
  return ldHalf(P.smk, (size_t)s * P.smokeCells + (((z & m) << sh | (y & m)) << sh | (x & m)), P.scalarHalf != 0);
}
// fireProField of the coarse density at `q` in coarse cells: clamped to the box, trilinear.
FP_DEV float coarseSample(const SimParams& P, const FpRender& R, SlotCache& c, float qx, float qy, float qz) {
  float S = (float)(1 << P.smokeShift);
  qx = fminf(fmaxf(qx, (float)c.lo[0] * S + .5f), (float)(c.hi[0] + 1) * S - .5f);
  qy = fminf(fmaxf(qy, (float)c.lo[1] * S + .5f), (float)(c.hi[1] + 1) * S - .5f);
  qz = fminf(fmaxf(qz, (float)c.lo[2] * S + .5f), (float)(c.hi[2] + 1) * S - .5f);
  float gx = qx - .5f, gy = qy - .5f, gz = qz - .5f;
  int x0 = (int)floorf(gx), y0 = (int)floorf(gy), z0 = (int)floorf(gz);
  float fx = gx - (float)x0, fy = gy - (float)y0, fz = gz - (float)z0;
  float v = 0.f;
  for (int k = 0; k < 8; k++) {
    int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
    float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
    v += rawCoarse(P, R, c, x0 + dx, y0 + dy, z0 + dz) * w;
  }
  return v;
}
// smoothCoarseSmoke (lighting.wgsl:104-129): the [1,2,1]/4 density at a coarse cell.
FP_DEV float smoothedCoarse(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z) {
  float d = 0.f;
  for (int k = 0; k < 8; k++)
    d += coarseSample(P, R, c, (float)(x + (k & 1)), (float)(y + ((k >> 1) & 1)), (float)(z + (k >> 2)));
  return fmaxf(0.f, d * .125f);
}
// The smoothed coarse density at a coarse cell: the pool in a brick with a slot, else what a
// sample based in a slotted brick reads from its apron (`apron`), else zero.
FP_DEV float renderSmokeCell(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z, bool apron) {
  const int sh = P.smokeShift, m = (1 << sh) - 1;
  int s = slotAt(P, R, c, x >> sh, y >> sh, z >> sh);
  if (s >= 0) return R.renderSmoke[(size_t)s * P.smokeCells + (((z & m) << sh | (y & m)) << sh | (x & m))];
  return apron ? smoothedCoarse(P, R, c, x, y, z) : 0.f;
}
// renderSmokeAt (volume-common.wgsl:74-78): fireProField of the smoothed coarse density at `q`
// in coarse cells.
FP_DEV float renderSmokeAt(const SimParams& P, const FpRender& R, SlotCache& c, float qx, float qy, float qz) {
  const int sh = P.smokeShift;
  float S = (float)(1 << sh);
  qx = fminf(fmaxf(qx, (float)c.lo[0] * S + .5f), (float)(c.hi[0] + 1) * S - .5f);
  qy = fminf(fmaxf(qy, (float)c.lo[1] * S + .5f), (float)(c.hi[1] + 1) * S - .5f);
  qz = fminf(fmaxf(qz, (float)c.lo[2] * S + .5f), (float)(c.hi[2] + 1) * S - .5f);
  float gx = qx - .5f, gy = qy - .5f, gz = qz - .5f;
  int x0 = (int)floorf(gx), y0 = (int)floorf(gy), z0 = (int)floorf(gz);
  float fx = gx - (float)x0, fy = gy - (float)y0, fz = gz - (float)z0;
  bool based = slotAt(P, R, c, x0 >> sh, y0 >> sh, z0 >> sh) >= 0;
  float v = 0.f;
  for (int k = 0; k < 8; k++) {
    int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
    float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
    v += renderSmokeCell(P, R, c, x0 + dx, y0 + dy, z0 + dz, based) * w;
  }
  return v;
}
// cachedSmokeCell (lighting.wgsl:133-156): the smoothed coarse density a conservative bound
// reads at coarse cell (x,y,z): the pool, else the apron a previous neighbour holds.
FP_DEV float cachedSmokeCell(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z) {
  const int sh = P.smokeShift, m = (1 << sh) - 1;
  int bx = x >> sh, by = y >> sh, bz = z >> sh;
  int s = slotAt(P, R, c, bx, by, bz);
  if (s >= 0) return R.renderSmoke[(size_t)s * P.smokeCells + (((z & m) << sh | (y & m)) << sh | (x & m))];
  const int l[3] = {x & m, y & m, z & m};
  for (int k = 1; k < 8; k++) {
    if (((k & 1) && l[0] != 0) || ((k & 2) && l[1] != 0) || ((k & 4) && l[2] != 0)) continue;
    if (slotAt(P, R, c, bx - (k & 1), by - ((k >> 1) & 1), bz - ((k >> 2) & 1)) >= 0)
      return smoothedCoarse(P, R, c, x, y, z);
  }
  return 0.f;
}

// The render field at a world cell. A cell of a brick with a slot reads the pool. A cell in a
// brick without one reads as the apron of a sample based in a slotted brick would hold it
// (`apron`: the smoothed density, no heat, flame or fuel; all zero with coarse smoke, whose
// field apron holds no neighbour), else zero.
FP_DEV float4 renderCell(const SimParams& P, const FpRender& R, SlotCache& c, int x, int y, int z, bool apron) {
  int s = slotAt(P, R, c, x >> P.shift, y >> P.shift, z >> P.shift);
  if (s >= 0) {
    size_t i = (size_t)s * 4 * P.N + localCell(P, x, y, z);
    return make_float4(R.renderField[i], R.renderField[i + P.N], R.renderField[i + 2 * P.N], R.renderField[i + 3 * P.N]);
  }
  if (!apron || P.smokeDiv > 1) return make_float4(0.f, 0.f, 0.f, 0.f);
  return make_float4(smoothedSmoke(P, R, c, x, y, z), 0.f, 0.f, 0.f);
}
FP_DEV void add4(float4& a, const float4& b, float w) {
  a.x += b.x * w;
  a.y += b.y * w;
  a.z += b.z * w;
  a.w += b.w * w;
}
// fireProField of the render field at `q` in cells (fireProSample, volume-bricks.wgsl).
FP_DEV float4 renderSample(const SimParams& P, const FpRender& R, SlotCache& c, float qx, float qy, float qz) {
  float B = (float)P.B;
  qx = fminf(fmaxf(qx, (float)c.lo[0] * B + .5f), (float)(c.hi[0] + 1) * B - .5f);
  qy = fminf(fmaxf(qy, (float)c.lo[1] * B + .5f), (float)(c.hi[1] + 1) * B - .5f);
  qz = fminf(fmaxf(qz, (float)c.lo[2] * B + .5f), (float)(c.hi[2] + 1) * B - .5f);
  float gx = qx - .5f, gy = qy - .5f, gz = qz - .5f;
  int x0 = (int)floorf(gx), y0 = (int)floorf(gy), z0 = (int)floorf(gz);
  float fx = gx - (float)x0, fy = gy - (float)y0, fz = gz - (float)z0;
  bool based = slotAt(P, R, c, x0 >> P.shift, y0 >> P.shift, z0 >> P.shift) >= 0;
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int k = 0; k < 8; k++) {
    int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
    float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
    add4(v, renderCell(P, R, c, x0 + dx, y0 + dy, z0 + dz, based), w);
  }
  return v;
}

// fireProReconstruct (volume-reconstruction.wgsl:5-95): 0 trilinear; 1 quadratic and 2 cubic
// B-splines from eight trilinear samples.
FP_DEV float4 reconstruct(const SimParams& P, const FpRender& R, SlotCache& c, float px, float py, float pz, int mode) {
  if (mode == 0) return renderSample(P, R, c, px, py, pz);
  float pos[2][3], wt[2][3];
  float p[3] = {px, py, pz};
  for (int a = 0; a < 3; a++) {
    float g = p[a] - .5f;
    if (mode == 1) {
      float center = floorf(g + .5f), delta = g - center;
      float w0 = .5f * (.5f - delta) * (.5f - delta), w1 = .75f - delta * delta, w2 = .5f * (.5f + delta) * (.5f + delta);
      wt[0][a] = w0 + w1;
      wt[1][a] = w2;
      pos[0][a] = center - .5f + w1 / wt[0][a];
      pos[1][a] = center + 1.5f;
    } else {
      float base = floorf(g), q = g - floorf(g), inv = 1.f - q;
      float w0 = inv * inv * inv / 6.f, w1 = (3.f * q * q * q - 6.f * q * q + 4.f) / 6.f;
      float w2 = (-3.f * q * q * q + 3.f * q * q + 3.f * q + 1.f) / 6.f, w3 = q * q * q / 6.f;
      wt[0][a] = w0 + w1;
      wt[1][a] = w2 + w3;
      pos[0][a] = base - .5f + w1 / wt[0][a];
      pos[1][a] = base + 1.5f + w3 / wt[1][a];
    }
  }
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  // The reference's order: x outermost, then y, then z.
  for (int i = 0; i < 8; i++) {
    int ix = (i >> 2) & 1, iy = (i >> 1) & 1, iz = i & 1;
    add4(v, renderSample(P, R, c, pos[ix][0], pos[iy][1], pos[iz][2]), wt[ix][0] * wt[iy][1] * wt[iz][2]);
  }
  return make_float4(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f), fmaxf(v.z, 0.f), fmaxf(v.w, 0.f));
}

// fireProExtinction and fireProEmission (fire-emission.wgsl:18-56).
FP_DEV float extinctionOf(const FpRender& R, const float4& f) {
  return fmaxf(0.f, f.x) * R.optical[0] + glowOf(f.z) * R.flameOpacity;
}
FP_DEV float3 emissionOf(const FpRender& R, const float4& f) {
  if (R.optical[1] <= 0.f) return make_float3(0.f, 0.f, 0.f);
  float s = fmaxf(0.f, f.x) * R.optical[0], flame = glowOf(f.z) * R.flameOpacity;
  float3 source = make_float3((1.f - R.smoke[0]) * s * R.smoke[3] + flame, (1.f - R.smoke[1]) * s * R.smoke[3] + flame,
                              (1.f - R.smoke[2]) * s * R.smoke[3] + flame);
  if (source.x == 0.f && source.y == 0.f && source.z == 0.f) return make_float3(0.f, 0.f, 0.f);
  float heat = fmaxf(0.f, f.y);
  float kelvin = 800.f + heat / (heat + 2.f) * (R.fire[3] - 800.f);
  float u = fminf(fmaxf((kelvin - 500.f) / 9500.f, 0.f), 1.f) * (float)(FP_BLACKBODY_SIZE - 1);
  int i0 = (int)floorf(u);
  int i1 = min(i0 + 1, FP_BLACKBODY_SIZE - 1);
  float fr = u - (float)i0;
  float4 a = __ldg(&R.lut[i0]), b = __ldg(&R.lut[i1]);
  float4 spec = make_float4(mixf(a.x, b.x, fr), mixf(a.y, b.y, fr), mixf(a.z, b.z, fr), mixf(a.w, b.w, fr));
  float scale = exp2f(fminf(fmaxf(spec.w, -24.f), 10.f));
  float3 thermal = make_float3(spec.x * scale, spec.y * scale, spec.z * scale);
  float tintPeak = fmaxf(R.fire[0], fmaxf(R.fire[1], R.fire[2]));
  float saturation = 1.f - fminf(R.fire[0], fminf(R.fire[1], R.fire[2])) / fmaxf(tintPeak, 1e-6f);
  float peak = fmaxf(thermal.x, fmaxf(thermal.y, thermal.z));
  float k = R.optical[1];
  return make_float3(mixf(thermal.x * tintPeak, R.fire[0] * peak, saturation) * source.x * k,
                     mixf(thermal.y * tintPeak, R.fire[1] * peak, saturation) * source.y * k,
                     mixf(thermal.z * tintPeak, R.fire[2] * peak, saturation) * source.z * k);
}

// sampleWorld (volume-common.wgsl:33-43): the render field at world point p, zero outside
// the box.
FP_DEV float4 sampleWorld(const SimParams& P, const FpRender& R, SlotCache& c, float px, float py, float pz) {
  float size = (float)P.B * P.h;
  if (px < (float)c.lo[0] * size || py < (float)c.lo[1] * size || pz < (float)c.lo[2] * size ||
      px > (float)(c.hi[0] + 1) * size || py > (float)(c.hi[1] + 1) * size || pz > (float)(c.hi[2] + 1) * size)
    return make_float4(0.f, 0.f, 0.f, 0.f);
  float4 f = renderSample(P, R, c, px / P.h, py / P.h, pz / P.h);
  if (P.smokeDiv > 1) {
    const float r = 1.f / (float)P.smokeDiv;  // fine cells to coarse: a power of two, exact
    f.x = renderSmokeAt(P, R, c, px / P.h * r, py / P.h * r, pz / P.h * r);
  }
  return f;
}

// exitDistance (lighting.wgsl:248-255).
FP_DEV float exitDistance(const SimParams& P, const SlotCache& c, float px, float py, float pz, float dx, float dy,
                          float dz) {
  float size = (float)P.B * P.h;
  float p[3] = {px, py, pz}, d[3] = {dx, dy, dz}, m = 1e30f;
  for (int a = 0; a < 3; a++) {
    if (!(fabsf(d[a]) > 1e-6f)) continue;
    float edge = (d[a] > 0.f ? (float)(c.hi[a] + 1) : (float)c.lo[a]) * size;
    m = fminf(m, (edge - p[a]) / d[a]);
  }
  return fmaxf(0.f, m);
}

// integratedTransmission (volume-common.wgsl:47-53).
FP_DEV float integratedTransmission(float extinction, float distance, float attenuation) {
  float depth = extinction * distance;
  if (depth < .001f) return distance * (1.f - .5f * depth + depth * depth / 6.f);
  return (1.f - attenuation) / extinction;
}

// incidentLight (lighting.wgsl:257-310): glow RGB and the sun's transmittance at p.
FP_DEV float4 incidentLight(const SimParams& P, const FpRender& R, SlotCache& c, float px, float py, float pz) {
  float4 local = sampleWorld(P, R, c, px, py, pz);
  if (local.x + glowOf(local.z) < 1e-5f) return make_float4(0.f, 0.f, 0.f, 1.f);
  float ln = sqrtf(R.light[0] * R.light[0] + R.light[1] * R.light[1] + R.light[2] * R.light[2]);
  float sx = R.light[0] / ln, sy = R.light[1] / ln, sz = R.light[2] / ln;
  int count = R.shadowSamples;
  float ds = exitDistance(P, c, px, py, pz, sx, sy, sz) / (float)count;
  float depth = 0.f;
  if (R.light[3] > 0.f) {
    for (int i = 0; i < count; i++) {
      float t = ((float)i + .5f) * ds;
      float4 f = sampleWorld(P, R, c, px + sx * t, py + sy * t, pz + sz * t);
      depth += (fmaxf(0.f, f.x) * R.optical[2] + glowOf(f.z) * R.flameOpacity) * ds;
      if (depth > 9.f) break;
    }
  }
  const float dirs[6][3] = {{.36f, .48f, -.8f}, {-.36f, -.48f, .8f}, {-.8f, .6f, 0.f},
                            {.8f, -.6f, 0.f},   {.48f, .64f, .6f},   {-.48f, -.64f, -.6f}};
  float3 glow = make_float3(0.f, 0.f, 0.f);
  if (R.optical[1] > 0.f && local.x > 1e-5f) {
    for (int d = 0; d < 6; d++) {
      float t = 0.f, interval = .075f, transmission = 1.f;
      for (int s = 0; s < 6; s++) {
        float q = t + interval * .5f;
        float4 f = sampleWorld(P, R, c, px + dirs[d][0] * q, py + dirs[d][1] * q, pz + dirs[d][2] * q);
        float ext = extinctionOf(R, f);
        float att = expf(-ext * interval);
        float3 e = emissionOf(R, f);
        float w = transmission * integratedTransmission(ext, interval, att) / 6.f;
        glow.x += e.x * w;
        glow.y += e.y * w;
        glow.z += e.z * w;
        transmission *= att;
        t += interval;
        interval *= 1.65f;
      }
    }
  }
  return make_float4(glow.x, glow.y, glow.z, expf(-depth));
}

// incidentLight with a whole warp, every lane passing the same position (and its own copy of
// the same cursor): the lanes take the shadow samples (32 at a time) and the six glow
// directions, and every lane then adds their terms in the order of the serial loops, with the
// serial early stop of the shadow sum, so all lanes return the serial result's value.
FP_DEV float4 incidentLightWarp(const SimParams& P, const FpRender& R, SlotCache& c, float px, float py, float pz) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float4 local = sampleWorld(P, R, c, px, py, pz);
  if (local.x + glowOf(local.z) < 1e-5f) return make_float4(0.f, 0.f, 0.f, 1.f);
  float ln = sqrtf(R.light[0] * R.light[0] + R.light[1] * R.light[1] + R.light[2] * R.light[2]);
  float sx = R.light[0] / ln, sy = R.light[1] / ln, sz = R.light[2] / ln;
  int count = R.shadowSamples;
  float ds = exitDistance(P, c, px, py, pz, sx, sy, sz) / (float)count;
  float depth = 0.f;
  if (R.light[3] > 0.f) {
    bool stop = false;
    for (int base = 0; base < count && !stop; base += 32) {
      const int i = base + lane;
      float v = 0.f;
      if (i < count) {
        float t = ((float)i + .5f) * ds;
        float4 f = sampleWorld(P, R, c, px + sx * t, py + sy * t, pz + sz * t);
        v = (fmaxf(0.f, f.x) * R.optical[2] + glowOf(f.z) * R.flameOpacity) * ds;
      }
      const int n = min(32, count - base);
      for (int j = 0; j < n; j++) {
        const float vj = __shfl_sync(full, v, j);
        if (!stop) {
          depth += vj;
          stop = depth > 9.f;
        }
      }
    }
  }
  float3 glow = make_float3(0.f, 0.f, 0.f);
  if (R.optical[1] > 0.f && local.x > 1e-5f) {
    const float dirs[6][3] = {{.36f, .48f, -.8f}, {-.36f, -.48f, .8f}, {-.8f, .6f, 0.f},
                              {.8f, -.6f, 0.f},   {.48f, .64f, .6f},   {-.48f, -.64f, -.6f}};
    float ex[6], ey[6], ez[6], ew[6];  // lane d < 6: direction d's six steps
#pragma unroll
    for (int k = 0; k < 6; k++) ex[k] = ey[k] = ez[k] = ew[k] = 0.f;
    if (lane < 6) {
      float t = 0.f, interval = .075f, transmission = 1.f;
#pragma unroll
      for (int k = 0; k < 6; k++) {
        float q = t + interval * .5f;
        float4 f = sampleWorld(P, R, c, px + dirs[lane][0] * q, py + dirs[lane][1] * q, pz + dirs[lane][2] * q);
        float ext = extinctionOf(R, f);
        float att = expf(-ext * interval);
        float3 e = emissionOf(R, f);
        ew[k] = transmission * integratedTransmission(ext, interval, att) / 6.f;
        ex[k] = e.x;
        ey[k] = e.y;
        ez[k] = e.z;
        transmission *= att;
        t += interval;
        interval *= 1.65f;
      }
    }
    for (int d = 0; d < 6; d++) {
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const float w = __shfl_sync(full, ew[k], d);
        glow.x += __shfl_sync(full, ex[k], d) * w;
        glow.y += __shfl_sync(full, ey[k], d) * w;
        glow.z += __shfl_sync(full, ez[k], d) * w;
      }
    }
  }
  return make_float4(glow.x, glow.y, glow.z, expf(-depth));
}

// The brick of computing brick `i` inside a box, that box made the current one, with its
// slot; false when no box holds it.
FP_DEV bool boxBrick(const SimParams& P, const FpRender& R, SlotCache& c, uint32_t i, int& bx, int& by, int& bz,
                     int& slot) {
  uint32_t id = P.active[i];
  if (!homeOk(P, id)) return false;  // the bounds-checked build only
  int4 t = __ldg(&P.tileRec[id >> 6]);
  int l = id & 63;
  bx = t.x * 4 + (l & 3);
  by = t.y * 4 + ((l >> 2) & 3);
  bz = t.z * 4 + (l >> 4);
  int k = 0;
  for (; k < R.boxCount; k++) {
    const int* b = R.boxes + 6 * k;
    if (bx >= b[0] && bx <= b[3] && by >= b[1] && by <= b[4] && bz >= b[2] && bz <= b[5]) break;
  }
  if (k == R.boxCount) return false;
  useBox(R, c, k);
  slot = slotAt(P, R, c, bx, by, bz);
  return slot >= 0;
}

// smoothSmoke: each boxed brick's render field, the smoothed density with heat, lifetime and
// fuel as they are.
__global__ void __launch_bounds__(RTHREADS) k_render_field(const SimParams* __restrict__ Pp, FpRender R) {
  const SimParams& P = *Pp;
  uint32_t total = P.counters->active;
  const bool half = P.scalarHalf != 0;
  for (uint32_t i = blockIdx.x; i < total; i += gridDim.x) {
    SlotCache c = noBox();
    int bx, by, bz, slot;
    if (!boxBrick(P, R, c, i, bx, by, bz, slot)) continue;
    for (int k = threadIdx.x; k < P.N; k += blockDim.x) {
      int x = bx * P.B + (k & (P.B - 1)), y = by * P.B + ((k >> P.shift) & (P.B - 1)), z = bz * P.B + (k >> (2 * P.shift));
      size_t o = (size_t)slot * 4 * P.N + k;
      R.renderField[o] = P.smokeDiv > 1 ? ldHalf(P.fld, o, half) : smoothedSmoke(P, R, c, x, y, z);
      R.renderField[o + P.N] = ldHalf(P.fld, o + P.N, half);
      R.renderField[o + 2 * P.N] = ldHalf(P.fld, o + 2 * P.N, half);
      R.renderField[o + 3 * P.N] = ldHalf(P.fld, o + 3 * P.N, half);
    }
    if (P.smokeDiv > 1) {  // smoothCoarseSmoke on the brick's coarse cells
      const int sh = P.smokeShift, S = 1 << sh;
      for (int k = threadIdx.x; k < P.smokeCells; k += blockDim.x) {
        int x = bx * S + (k & (S - 1)), y = by * S + ((k >> sh) & (S - 1)), z = bz * S + (k >> (2 * sh));
        R.renderSmoke[(size_t)slot * P.smokeCells + k] = smoothedCoarse(P, R, c, x, y, z);
      }
    }
  }
}

// buildOccupancy and buildLighting of each boxed brick, from the render field.
__global__ void __launch_bounds__(RTHREADS) k_render_light(const SimParams* __restrict__ Pp, FpRender R) {
  const SimParams& P = *Pp;
  __shared__ int flags;
  __shared__ int glowBits, smokeBits;  // the coarse bound's maxima (nonnegative floats' bits)
  if (threadIdx.x == 0) glowBits = smokeBits = 0;
  uint32_t total = P.counters->active;
  const int L = 1 << R.lightShift, L3 = L * L * L;
  const float texel = P.h * (float)(P.B >> R.lightShift);
  const int per = P.B / 8, blocks = per * per * per;
  for (uint32_t i = blockIdx.x; i < total; i += gridDim.x) {
    SlotCache c = noBox();
    int bx, by, bz, slot;
    if (!boxBrick(P, R, c, i, bx, by, bz, slot)) continue;  // the same for the whole CTA
    // Each 8-cell block with a halo of two cells, in units of 2x2x2 cells: a unit in a
    // slotted brick looks at its corner cells of the render field.
    for (int b = 0; b < blocks; b++) {
      if (threadIdx.x == 0) flags = 0;
      __syncthreads();
      int ox = bx * P.B + (b % per) * 8 - 2, oy = by * P.B + ((b / per) % per) * 8 - 2, oz = bz * P.B + (b / (per * per)) * 8 - 2;
      int mine = 0;
      const bool coarse = P.smokeDiv > 1;
      float glowMax = 0.f, smokeMax = 0.f;
      for (int u = threadIdx.x; u < 216; u += blockDim.x) {
        int ux = ox + (u % 6) * 2, uy = oy + ((u / 6) % 6) * 2, uz = oz + (u / 36) * 2;
        if (slotAt(P, R, c, ux >> P.shift, uy >> P.shift, uz >> P.shift) < 0) continue;
        for (int k = 0; k < 8; k++) {
          float4 f = renderCell(P, R, c, ux + (k & 1), uy + ((k >> 1) & 1), uz + (k >> 2), true);
          float g = glowOf(f.z);
          mine |= (g > .002f ? 1 : 0) | ((coarse ? 0.f : f.x) + g > .002f ? 2 : 0);
          glowMax = fmaxf(glowMax, g);
        }
      }
      if (coarse) {
        // Every trilinear donor of coarse density in the block and halo (lighting.wgsl:222-238).
        const int d = P.smokeDiv, S = 1 << P.smokeShift;
        const float ratio = (float)d;
        int lo[3], hi[3], size[3], boxLo[3], boxHi[3];
        const int o[3] = {ox, oy, oz};
        for (int a = 0; a < 3; a++) {
          lo[a] = (int)floorf((float)o[a] / ratio - .5f);
          hi[a] = (int)floorf((float)(o[a] + 12) / ratio - .5f) + 1;
          size[a] = hi[a] - lo[a] + 1;
          boxLo[a] = c.lo[a] * S;
          boxHi[a] = (c.hi[a] + 1) * S - 1;
        }
        for (int q = threadIdx.x; q < size[0] * size[1] * size[2]; q += blockDim.x) {
          int cq[3] = {lo[0] + q % size[0], lo[1] + (q / size[0]) % size[1], lo[2] + q / (size[0] * size[1])};
          for (int a = 0; a < 3; a++) cq[a] = min(max(cq[a], boxLo[a]), boxHi[a]);
          smokeMax = fmaxf(smokeMax, cachedSmokeCell(P, R, c, cq[0], cq[1], cq[2]));
        }
        glowMax = fmaxf(glowMax, __shfl_xor_sync(0xffffffffu, glowMax, 16));
        for (int w = 8; w > 0; w >>= 1) glowMax = fmaxf(glowMax, __shfl_xor_sync(0xffffffffu, glowMax, w));
        for (int w = 16; w > 0; w >>= 1) smokeMax = fmaxf(smokeMax, __shfl_xor_sync(0xffffffffu, smokeMax, w));
        if ((threadIdx.x & 31) == 0) {
          atomicMax(&glowBits, __float_as_int(glowMax));
          atomicMax(&smokeBits, __float_as_int(smokeMax));
        }
      }
      if (mine) atomicOr(&flags, mine);
      __syncthreads();
      if (coarse && threadIdx.x == 0 && __int_as_float(smokeBits) + __int_as_float(glowBits) > .002f) flags |= 2;
      if (threadIdx.x == 0) {
        R.occupancy[(size_t)slot * blocks + b] = (uint8_t)flags;
        glowBits = 0;
        smokeBits = 0;
      }
      __syncthreads();
    }
    // The brick's texels of the lighting lattice, a warp a texel.
    for (int k = threadIdx.x >> 5; k < L3; k += blockDim.x >> 5) {
      int lx = k % L, ly = (k / L) % L, lz = k / (L * L);
      float4 light = incidentLightWarp(P, R, c, ((float)(bx * L + lx) + .5f) * texel,
                                       ((float)(by * L + ly) + .5f) * texel, ((float)(bz * L + lz) + .5f) * texel);
      if ((threadIdx.x & 31) == 0) {
        size_t o = (size_t)slot * 4 * L3 + k;
        R.lighting[o] = light.x;
        R.lighting[o + L3] = light.y;
        R.lighting[o + 2 * L3] = light.z;
        R.lighting[o + 3 * L3] = light.w;
      }
    }
  }
}

// fireProLight (volume-bricks.wgsl:158-178) at `q` in lighting texels.
FP_DEV float4 lightSample(const SimParams& P, const FpRender& R, SlotCache& c, float qx, float qy, float qz) {
  const int L = 1 << R.lightShift, L3 = L * L * L;
  const float texel = P.h * (float)(P.B >> R.lightShift);
  qx = fminf(fmaxf(qx, (float)c.lo[0] * L + .5f), (float)(c.hi[0] + 1) * L - .5f);
  qy = fminf(fmaxf(qy, (float)c.lo[1] * L + .5f), (float)(c.hi[1] + 1) * L - .5f);
  qz = fminf(fmaxf(qz, (float)c.lo[2] * L + .5f), (float)(c.hi[2] + 1) * L - .5f);
  float gx = qx - .5f, gy = qy - .5f, gz = qz - .5f;
  int x0 = (int)floorf(gx), y0 = (int)floorf(gy), z0 = (int)floorf(gz);
  if (slotAt(P, R, c, x0 >> R.lightShift, y0 >> R.lightShift, z0 >> R.lightShift) < 0)
    return make_float4(0.f, 0.f, 0.f, 1.f);
  float fx = gx - (float)x0, fy = gy - (float)y0, fz = gz - (float)z0;
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int k = 0; k < 8; k++) {
    int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
    int x = x0 + dx, y = y0 + dy, z = z0 + dz;
    float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
    int s = slotAt(P, R, c, x >> R.lightShift, y >> R.lightShift, z >> R.lightShift);
    float4 t;
    if (s >= 0) {
      int m = L - 1;
      size_t o = (size_t)s * 4 * L3 + (((z & m) * L + (y & m)) * L + (x & m));
      t = make_float4(R.lighting[o], R.lighting[o + L3], R.lighting[o + 2 * L3], R.lighting[o + 3 * L3]);
    } else {  // the apron of a neighbour without a slot: lit where it stands
      t = incidentLight(P, R, c, ((float)x + .5f) * texel, ((float)y + .5f) * texel, ((float)z + .5f) * texel);
    }
    add4(v, t, w);
  }
  return v;
}

// fireProJitter (volume-march.wgsl:94-102).
FP_DEV float jitterOf(uint32_t px, uint32_t py, float time) {
  uint32_t s0 = px * 1664525u + 1013904223u, s1 = py * 1664525u + 1013904223u,
           s2 = (uint32_t)(time * 60.f) * 1664525u + 1013904223u;
  s0 += s1 * s2;
  s1 += s2 * s0;
  s2 += s0 * s1;
  s0 ^= s0 >> 16u;
  s1 ^= s1 >> 16u;
  s2 ^= s2 >> 16u;
  s0 += s1 * s2;
  return (float)(s0 >> 8u) / 16777216.f;
}

// A pixel's march (fireProSceneVolume with fireProMarch), a thread a pixel.
// A camera ray through the boxes (fireProRay, fireProSpan) and what its march keeps fixed.
struct Ray {
  float ro[3], rd[3], safe[3], exitSide[3];
  float lo, hi;  // the first box entry and the last exit
  float stepSize, jitter, direct[3];
};
// fireProHit: where the ray enters and leaves box k (entry after exit when it misses).
FP_DEV float2 boxHit(const FpRender& R, const Ray& r, int k, float brickSize) {
  const int* b = R.boxes + 6 * k;
  float lo = 0.f, hi = 1e30f;
  for (int a = 0; a < 3; a++) {
    float ta = ((float)b[a] * brickSize - r.ro[a]) / r.safe[a];
    float tb = ((float)(b[3 + a] + 1) * brickSize - r.ro[a]) / r.safe[a];
    lo = fmaxf(lo, fminf(ta, tb));
    hi = fminf(hi, fmaxf(ta, tb));
  }
  return make_float2(lo, hi);
}
// The ray of viewport point (ux, uy) in [0,1]^2, its span through the boxes and step; false
// when it misses them all.
FP_DEV bool rayOf(const SimParams& P, const FpRender& R, float ux, float uy, Ray& r) {
  float cx = ux * 2.f - 1.f, cy = 1.f - uy * 2.f;
  const float* M = R.ivp;
  float nh[4], fh[4];
  for (int k = 0; k < 4; k++) {
    nh[k] = M[k] * cx + M[4 + k] * cy + M[8 + k] * 0.f + M[12 + k];
    fh[k] = M[k] * cx + M[4 + k] * cy + M[8 + k] * .99999f + M[12 + k];
  }
  for (int a = 0; a < 3; a++) {
    r.ro[a] = nh[a] / nh[3];
    r.rd[a] = fh[a] / fh[3] - r.ro[a];
  }
  float rl = sqrtf(r.rd[0] * r.rd[0] + r.rd[1] * r.rd[1] + r.rd[2] * r.rd[2]);
  for (int a = 0; a < 3; a++) r.rd[a] /= rl;
  const float brickSize = P.h * (float)P.B;
  for (int a = 0; a < 3; a++) {
    r.safe[a] = fabsf(r.rd[a]) > 1e-6f ? r.rd[a] : 1e-6f;
    r.exitSide[a] = r.rd[a] > 0.f ? 1.f : 0.f;
  }
  // fireProSpan: the first entry, the last exit and the length inside every box.
  r.lo = 1e30f;
  r.hi = 0.f;
  float length = 0.f;
  for (int k = 0; k < R.boxCount; k++) {
    float2 hit = boxHit(R, r, k, brickSize);
    if (hit.y > hit.x) {
      r.lo = fminf(r.lo, hit.x);
      r.hi = fmaxf(r.hi, hit.y);
      length += hit.y - hit.x;
    }
  }
  if (!(r.hi > r.lo)) return false;
  r.stepSize = fmaxf(P.h * .5f, length / (float)R.raySteps);
  // fireProDirect
  float ln = sqrtf(R.light[0] * R.light[0] + R.light[1] * R.light[1] + R.light[2] * R.light[2]);
  float g = R.optical[3];
  float mu = (r.rd[0] * R.light[0] + r.rd[1] * R.light[1] + r.rd[2] * R.light[2]) / ln;
  float phase = (1.f - g * g) / powf(fmaxf(.05f, 1.f + g * g - 2.f * g * mu), 1.5f);
  float dk = R.light[3] * (.35f + phase * .3f);
  for (int a = 0; a < 3; a++) r.direct[a] = R.sceneLight[a] * dk;
  return true;
}

// fireProEnter (fireProNext): the box the ray is in at t, or the next one it enters, becomes the
// current one with its exit, and t moves to its entry; false past the last box. Boxes never
// overlap, so of the boxes the ray has not left, the one it enters first is the one.
FP_DEV bool enterBox(const SimParams& P, const FpRender& R, const Ray& r, float& t, float& exit, SlotCache& c) {
  const float brickSize = P.h * (float)P.B;
  float entry = 1e30f, out = 0.f;
  int best = -1;
  for (int k = 0; k < R.boxCount; k++) {
    float2 hit = boxHit(R, r, k, brickSize);
    if (hit.y > hit.x && hit.y > t && hit.x < entry) {
      entry = hit.x;
      out = hit.y;
      best = k;
    }
  }
  if (best < 0) return false;
  useBox(R, c, best);
  exit = out;
  t = fmaxf(t, entry);
  return true;
}

// One step of fireProMarch (volume-march.wgsl:178-268) at t, ds long, in the current box (which
// the ray leaves at `exit`): past an empty block a skip of whole steps up to the exit, else the
// shaded sample. Returns the next t.
FP_DEV float marchStep(const SimParams& P, const FpRender& R, SlotCache& c, const Ray& r, float t, float ds, float exit,
                       float& trans, float* rad) {
  const float brickSize = P.h * (float)P.B, lightRatio = (float)(P.B >> R.lightShift);
  float tt = t + r.jitter * ds;
  float p[3] = {r.ro[0] + r.rd[0] * tt, r.ro[1] + r.rd[1] * tt, r.ro[2] + r.rd[2] * tt};
  float cell[3] = {p[0] / P.h, p[1] / P.h, p[2] / P.h};
  int ci[3] = {(int)floorf(cell[0]), (int)floorf(cell[1]), (int)floorf(cell[2])};
  int slot = slotAt(P, R, c, ci[0] >> P.shift, ci[1] >> P.shift, ci[2] >> P.shift);
  float size = brickSize;
  int flags = 0;
  if (slot >= 0) {  // fireProOccupancy: the sample's 8-cell block of the brick
    const int per = P.B / 8, m = P.B - 1;
    int block = ((((ci[2] & m) >> 3) * per) + ((ci[1] & m) >> 3)) * per + ((ci[0] & m) >> 3);
    flags = R.occupancy[(size_t)slot * per * per * per + block];
    size = P.h * 8.f;
  }
  if (!(flags & 2)) {
    // Skip whole steps past the empty block, keeping the lattice.
    float dist = 1e30f;
    for (int a = 0; a < 3; a++) dist = fminf(dist, ((floorf(p[a] / size) + r.exitSide[a]) * size - p[a]) / r.safe[a]);
    return fminf(t + fmaxf(1.f, floorf(dist / r.stepSize) + 1.f) * r.stepSize, exit);
  }
  float4 f = reconstruct(P, R, c, cell[0], cell[1], cell[2], (flags & 1) ? R.filter : 0);
  if (P.smokeDiv > 1) {  // fireProRenderField: the smoothed coarse density, trilinear
    const float q = 1.f / (float)P.smokeDiv;
    f.x = renderSmokeAt(P, R, c, cell[0] * q, cell[1] * q, cell[2] * q);
  }
  if (f.x + glowOf(f.z) > .002f) {
    // fireProShade
    float3 glow = emissionOf(R, f);
    float density = fmaxf(0.f, f.x) * R.optical[0];
    float sc[3] = {0.f, 0.f, 0.f};
    if (density > 0.f) {
      float4 inc = lightSample(P, R, c, cell[0] / lightRatio, cell[1] / lightRatio, cell[2] / lightRatio);
      sc[0] = R.smoke[0] * (R.ambient[0] + r.direct[0] * inc.w + inc.x * .65f) * density;
      sc[1] = R.smoke[1] * (R.ambient[1] + r.direct[1] * inc.w + inc.y * .65f) * density;
      sc[2] = R.smoke[2] * (R.ambient[2] + r.direct[2] * inc.w + inc.z * .65f) * density;
    }
    float ext = extinctionOf(R, f);
    float tau = ext * ds;
    float integral = ds * (1.f - .5f * tau + tau * tau / 6.f);
    if (tau >= .001f) integral = (1.f - expf(-tau)) / ext;
    rad[0] += trans * (sc[0] + glow.x) * integral;
    rad[1] += trans * (sc[1] + glow.y) * integral;
    rad[2] += trans * (sc[2] + glow.z) * integral;
    trans *= 1.f - fminf(1.f, ext * integral);
  }
  return t + ds;
}

// buildSlices (volume-slices.wgsl:28-122): a ray per half-resolution pixel marches from the
// first box entry to the last exit, box by box, recording radiance and opacity at FP_SLICES
// evenly spaced depths; depths passed by a skip or a jump between boxes keep the values of the
// moment, those past the exit or an opaque ray the final ones.
__global__ void __launch_bounds__(RTHREADS) k_slices(const SimParams* __restrict__ Pp, FpRender R) {
  const SimParams& P = *Pp;
  int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= R.sliceW * R.sliceH) return;
  int px = pix % R.sliceW, py = pix / R.sliceW;
  float4* out = reinterpret_cast<float4*>(R.slices) + (size_t)pix * FP_SLICES;
  float trans = 1.f, rad[3] = {0.f, 0.f, 0.f};
  int recorded = 0;
  Ray r;
  if (R.boxCount > 0 && rayOf(P, R, ((float)px + .5f) / (float)R.sliceW, ((float)py + .5f) / (float)R.sliceH, r)) {
    r.jitter = jitterOf((uint32_t)px, (uint32_t)py, R.time);
    const float spacing = fmaxf(r.hi - r.lo, 0.f) / (float)FP_SLICES;
    SlotCache c = noBox();
    float t = r.lo, depth = r.lo + spacing, exit = t;
    while (recorded < FP_SLICES && t < r.hi && trans >= .008f) {
      if (t >= exit) {
        if (!enterBox(P, R, r, t, exit, c)) break;
      } else {
        float ds = fminf(r.stepSize, fminf(depth, exit) - t);
        t = marchStep(P, R, c, r, t, ds, exit, trans, rad);
      }
      while (recorded < FP_SLICES && t >= depth) {
        out[recorded] = make_float4(rad[0], rad[1], rad[2], 1.f - trans);
        recorded++;
        depth = r.lo + spacing * (float)(recorded + 1);
      }
    }
  }
  for (; recorded < FP_SLICES; recorded++) out[recorded] = make_float4(rad[0], rad[1], rad[2], 1.f - trans);
}

// fireProSceneVolume (scene-volume.wgsl:39-44, 146-167): the march of each pixel's ray up to
// the scene's depth through the boxes, from the last half-resolution slice in front of it when
// slices exist.
__global__ void __launch_bounds__(RTHREADS) k_march(const SimParams* __restrict__ Pp, FpRender R) {
  const SimParams& P = *Pp;
  int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= R.width * R.height) return;
  int px = pix % R.width, py = pix / R.width;
  float4* out = reinterpret_cast<float4*>(R.image) + pix;
  *out = make_float4(0.f, 0.f, 0.f, 0.f);
  if (R.boxCount == 0) return;
  const float ux = ((float)px + .5f) / (float)R.width, uy = ((float)py + .5f) / (float)R.height;
  Ray r;
  if (!rayOf(P, R, ux, uy, r)) return;
  // fireProSceneDistance (volume-march.wgsl:76-89): the scene's depth ends the ray.
  float end = r.hi;
  if (R.depth) {
    const float d = R.depth[pix];
    if (d < .999999f) {
      const float cx = ux * 2.f - 1.f, cy = 1.f - uy * 2.f;
      const float* M = R.ivp;
      float hit[4];
      for (int k = 0; k < 4; k++) hit[k] = M[k] * cx + M[4 + k] * cy + M[8 + k] * d + M[12 + k];
      float dist = 0.f;
      for (int a = 0; a < 3; a++) dist += (hit[a] / hit[3] - r.ro[a]) * r.rd[a];
      end = fminf(end, dist);
    }
  }
  if (end <= r.lo) return;
  r.jitter = jitterOf((uint32_t)px, (uint32_t)py, R.time);
  float t = r.lo, trans = 1.f;
  float rad[3] = {0.f, 0.f, 0.f};
  if (R.slices) {
    // Resume from the last slice in front of the scene: the half-resolution texels
    // interpolated bilinearly (clamped at the edges) on that slice.
    const float count = (float)FP_SLICES;
    const float slice = floorf((end - r.lo) / (r.hi - r.lo) * count);
    if (slice >= 1.f) {
      const int layer = (int)fminf(slice, count) - 1;
      float gx = ux * (float)R.sliceW - .5f, gy = uy * (float)R.sliceH - .5f;
      float fx0 = floorf(gx), fy0 = floorf(gy);
      float wx = gx - fx0, wy = gy - fy0;
      int x0 = (int)fx0, y0 = (int)fy0;
      int xs[2] = {min(max(x0, 0), R.sliceW - 1), min(max(x0 + 1, 0), R.sliceW - 1)};
      int ys[2] = {min(max(y0, 0), R.sliceH - 1), min(max(y0 + 1, 0), R.sliceH - 1)};
      const float4* S = reinterpret_cast<const float4*>(R.slices);
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int k = 0; k < 4; k++) {
        int ix = k & 1, iy = k >> 1;
        add4(v, S[((size_t)ys[iy] * R.sliceW + xs[ix]) * FP_SLICES + layer], (ix ? wx : 1.f - wx) * (iy ? wy : 1.f - wy));
      }
      t = r.lo + (r.hi - r.lo) * fminf(slice, count) / count;
      trans = 1.f - v.w;
      rad[0] = v.x;
      rad[1] = v.y;
      rad[2] = v.z;
    }
  }
  // fireProMarch: the cursor starts exited, so the first pass enters the box at t.
  SlotCache c = noBox();
  float exit = t;
  while (t < end && trans >= .008f) {
    if (t >= exit) {
      if (!enterBox(P, R, r, t, exit, c)) break;
      continue;
    }
    float ds = fminf(r.stepSize, fminf(end, exit) - t);
    t = marchStep(P, R, c, r, t, ds, exit, trans, rad);
  }
  *out = make_float4(rad[0], rad[1], rad[2], 1.f - trans);
}

// collectLights (scene-lights.wgsl:37-106): a CTA of 64 lanes per computing brick, a lane per
// cell of the brick's 4^3 sample lattice (stride B/4, at the stride's middle). The brick's
// anchor is the nearest to its centre (height above an anchor counting a quarter; ties to the
// lower index); the lanes' luminance, luminance-weighted offsets and RGB are summed in shared
// memory and seven lanes add the totals to the anchor's floats.
__global__ void __launch_bounds__(64) k_collect_lights(const SimParams* __restrict__ Pp, FpRender R,
                                                       const float* __restrict__ anchors, int count, float* sums) {
  const SimParams& P = *Pp;
  __shared__ float2 nearest[64];
  __shared__ float4 positions[64];
  __shared__ float4 colors[64];
  const uint32_t total = P.counters->active;
  const int lane = threadIdx.x, stride = P.B >> 2;
  const bool half = P.scalarHalf != 0;
  const float side = (float)P.B * P.h;
  for (uint32_t i = blockIdx.x; i < total; i += gridDim.x) {
    const uint32_t id = P.active[i];
    if (!homeOk(P, id)) continue;  // the bounds-checked build only
    const int e = P.entries[id];
    if (e < 0) continue;  // the same for the whole CTA
    const int slot = entryPage(e);
    const int4 t = __ldg(&P.tileRec[id >> 6]);
    const int l = id & 63;
    const int b[3] = {t.x * 4 + (l & 3), t.y * 4 + ((l >> 2) & 3), t.z * 4 + (l >> 4)};
    const int lx = (lane & 3) * stride + stride / 2, ly = ((lane >> 2) & 3) * stride + stride / 2,
              lz = (lane >> 4) * stride + stride / 2;
    const size_t o = (size_t)slot * 4 * P.N + (size_t)((lz * P.B + ly) * P.B + lx);
    float4 f = make_float4(ldHalf(P.fld, o, half), ldHalf(P.fld, o + P.N, half), ldHalf(P.fld, o + 2 * P.N, half),
                           ldHalf(P.fld, o + 3 * P.N, half));
    if (P.smokeDiv > 1) {
      // The coarse density sampled trilinearly at the cell's centre on the smoke lattice
      // (scene-lights.wgsl:59-65): a tap past the brick reads the +1 neighbour (the slot's
      // apron), zero without a slot; taps before the brick read zero.
      const int sh = P.smokeShift, S = 1 << sh, m = S - 1;
      const float r = 1.f / (float)P.smokeDiv;
      const float q[3] = {((float)lx + .5f) * r - .5f, ((float)ly + .5f) * r - .5f, ((float)lz + .5f) * r - .5f};
      int c0[3];
      float fr[3];
      for (int a = 0; a < 3; a++) {
        float g = floorf(q[a]);
        c0[a] = (int)g;
        fr[a] = q[a] - g;
      }
      float v = 0.f;
      for (int k = 0; k < 8; k++) {
        int d[3] = {k & 1, (k >> 1) & 1, k >> 2};
        int cl[3] = {c0[0] + d[0], c0[1] + d[1], c0[2] + d[2]};
        if (cl[0] < 0 || cl[1] < 0 || cl[2] < 0) continue;
        int nb[3] = {b[0] + (cl[0] >> sh), b[1] + (cl[1] >> sh), b[2] + (cl[2] >> sh)};
        int t = hashFind(P, nb[0] >> 2, nb[1] >> 2, nb[2] >> 2);
        int s = t < 0 ? -1 : checkSlot(P, FP_SITE_ENTRY, entryPage(P.entries[t * 64 + (((nb[2] & 3) * 4 + (nb[1] & 3)) * 4 + (nb[0] & 3))]));
        if (s < 0) continue;
        float w = (d[0] ? fr[0] : 1.f - fr[0]) * (d[1] ? fr[1] : 1.f - fr[1]) * (d[2] ? fr[2] : 1.f - fr[2]);
        v += ldHalf(P.smk, (size_t)s * P.smokeCells + ((((cl[2] & m) << sh) | (cl[1] & m)) << sh | (cl[0] & m)), half) * w;
      }
      f.x = v;
    }
    const float3 rgb = emissionOf(R, f);
    const float luminance = rgb.x * .2126f + rgb.y * .7152f + rgb.z * .0722f;
    const float cx = ((float)b[0] + .5f) * side, cy = ((float)b[1] + .5f) * side, cz = ((float)b[2] + .5f) * side;
    float2 best = make_float2(1e38f, 0.f);
    for (int k = lane; k < count; k += 64) {
      float dx = cx - anchors[3 * k], dy = cy - anchors[3 * k + 1], dz = cz - anchors[3 * k + 2];
      float rise = dy > 0.f ? dy * .25f : dy;
      float d = dx * dx + dz * dz + rise * rise;
      if (d < best.x) best = make_float2(d, (float)k);
    }
    nearest[lane] = best;
    __syncthreads();
    for (int reach = 32; reach > 0; reach >>= 1) {
      if (lane < reach) {
        float2 other = nearest[lane + reach], mine = nearest[lane];
        if (other.x < mine.x || (other.x == mine.x && other.y < mine.y)) nearest[lane] = other;
      }
      __syncthreads();
    }
    const int anchor = (int)nearest[0].y;
    const float px = ((float)(b[0] * P.B + lx) + .5f) * P.h, py = ((float)(b[1] * P.B + ly) + .5f) * P.h,
                pz = ((float)(b[2] * P.B + lz) + .5f) * P.h;
    positions[lane] = make_float4(luminance, (px - anchors[3 * anchor]) * luminance,
                                  (py - anchors[3 * anchor + 1]) * luminance, (pz - anchors[3 * anchor + 2]) * luminance);
    colors[lane] = make_float4(rgb.x, rgb.y, rgb.z, 0.f);
    __syncthreads();
    for (int reach = 32; reach > 0; reach >>= 1) {
      if (lane < reach) {
        float4 a = positions[lane], c = positions[lane + reach], u = colors[lane], v = colors[lane + reach];
        positions[lane] = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w + c.w);
        colors[lane] = make_float4(u.x + v.x, u.y + v.y, u.z + v.z, 0.f);
      }
      __syncthreads();
    }
    if (lane < 7) {
      const float totals[7] = {positions[0].x, positions[0].y, positions[0].z, positions[0].w,
                               colors[0].x, colors[0].y, colors[0].z};
      atomicAdd(&sums[anchor * 8 + lane], totals[lane]);
    }
    __syncthreads();  // the shared sums are read before the next brick's lanes write them
  }
}

}  // namespace

void fp_launch_collect_lights(const SimParams* dP, const FpRender& R, const float* anchors, int count, float* sums,
                              int sms, cudaStream_t st) {
  k_collect_lights<<<sms * 16, 64, 0, st>>>(dP, R, anchors, count, sums);
}

void fp_launch_render(const SimParams* dP, const FpRender& R, int sms, cudaStream_t st) {
  k_render_field<<<sms * 8, RTHREADS, 0, st>>>(dP, R);
  k_render_light<<<sms * 8, RTHREADS, 0, st>>>(dP, R);
  if (R.slices) {
    int half = R.sliceW * R.sliceH;
    k_slices<<<(half + RTHREADS - 1) / RTHREADS, RTHREADS, 0, st>>>(dP, R);
  }
  int pixels = R.width * R.height;
  k_march<<<(pixels + RTHREADS - 1) / RTHREADS, RTHREADS, 0, st>>>(dP, R);
}
