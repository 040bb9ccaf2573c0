// The step's field kernels over the computing bricks: MacCormack transport of the staggered
// velocity and of the scalars with their limiters, field evolution and combustion, curl,
// forces, divergence and projection. One CTA per computing brick, grid-stride over the
// ascending list the allocation wrote, so no launch depends on a host-side count.
//
// Restates src/engine/shaders/fluid-velocity-transport.wgsl, fluid-scalar-transport.wgsl,
// fluid-field-evolution.wgsl, fluid-forces.wgsl and force-fields.wgsl. Samples read the
// neighbour bricks' cells through the brick's 27-entry record (shared memory) where the
// reference reads a texture apron that copies them; bricks without a slot read zero.
//
// Staging: for 8^3 bricks the transport kernels first copy the fields they sample, over the
// home brick and a HALO-cell rim, into shared memory ([channel][S^3], S = B + 2 HALO), with
// coalesced loads through the neighbour record. Trilinear taps inside the rim then read
// shared memory; taps past it (traces longer than the rim) take the directory path. Both
// paths compute the same sums in the same order.
#include "fp_device.cuh"
#include "fp_launch.h"

namespace {

constexpr int THREADS = 256;
constexpr int HALO = 2;
// Resident CTAs per SM the transport and force kernels are compiled and launched for (register
// cap 65536 / (256 n)): three (85 registers) beat four (64, with spills) on the B200.
#ifndef FP_TRANSPORT_CTAS
#define FP_TRANSPORT_CTAS 3
#endif

// Where the staged copy sits: its first cell and its side.
// SS, the box's side, is a compile-time constant, so staged addresses fold into immediate
// offsets of the shared-memory loads. SS = 0: nothing is staged (every read goes through the
// directory), known at compile time, so a staged kernel carries no code for the unstaged form
// and the reverse.
template <int SS>
struct Stage {
  int ox, oy, oz;
  static constexpr int S = SS, S3 = SS * SS * SS;
};
// The transport kernels' box: the brick and a HALO-cell rim when staged, else nothing.
template <bool STAGED>
using TransportStage = Stage<STAGED ? 8 + 2 * HALO : 0>;

// A field a kernel reads: the pool and, when staged, its shared copy (set exactly when the
// kernel's Stage has a side).
struct Field {
  const float* pool;
  int ch;
  const float* sm;
  bool half;  // the pool holds __half (the scalar pools in FP_PRECISION_MIXED)
};

// The staged offset of cell (x,y,z), which the caller knows lies inside the staged box.
template <int SS>
FP_DEV int stagedAt(const Stage<SS>& G, int x, int y, int z) { return ((z - G.oz) * G.S + (y - G.oy)) * G.S + (x - G.ox); }

// A cell within HALO cells of the home brick: the staged box always holds it, so no check.
template <int SS>
FP_DEV float nearCell(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& f, int c, int x, int y, int z) {
  if constexpr (SS > 0) return f.sm[c * G.S3 + stagedAt(G, x, y, z)];
  else return cellAt(P, H, f.pool, f.ch, c, x, y, z, f.half);
}

// The staged kernels' taps past the staged box (traces longer than the rim): out of line, so
// the rare path costs the kernels no instruction-cache space.
// Returned by value, so the callers' blocks stay in registers.
struct Cells8 {
  float v[8];
};
static __device__ __noinline__ Cells8 blockCellsFar(const SimParams& P, const Home& H, const Field& f, int c, int x0,
                                                    int y0, int z0) {
  Cells8 r;
#pragma unroll
  for (int j = 0; j < 8; j++) r.v[j] = cellAt(P, H, f.pool, f.ch, c, x0 + (j & 1), y0 + ((j >> 1) & 1), z0 + (j >> 2), f.half);
  return r;
}
static __device__ __noinline__ float sampleFar(const SimParams& P, const Home& H, const Field& f, int c, float px,
                                               float py, float pz) {
  return sampleCells(P, H, f.pool, f.ch, c, px, py, pz, f.half);
}

// The 2x2x2 block from corner (x0,y0,z0) of channel c into t (x fastest): from shared memory
// when `b` (the corner's staged address, channel 0) is set, else through the directory.
template <int SS>
FP_DEV void blockCells(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& f, int c, const float* b, int x0,
                       int y0, int z0, float* t) {
  if constexpr (SS > 0) {
    if (b) {
      const float* q = b + c * G.S3;
      constexpr int S = SS, S2 = SS * SS;
      t[0] = q[0]; t[1] = q[1]; t[2] = q[S]; t[3] = q[S + 1];
      t[4] = q[S2]; t[5] = q[S2 + 1]; t[6] = q[S2 + S]; t[7] = q[S2 + S + 1];
    } else {
      Cells8 r = blockCellsFar(P, H, f, c, x0, y0, z0);
#pragma unroll
      for (int j = 0; j < 8; j++) t[j] = r.v[j];
    }
  } else {
#pragma unroll
    for (int j = 0; j < 8; j++)
      t[j] = cellAt(P, H, f.pool, f.ch, c, x0 + (j & 1), y0 + ((j >> 1) & 1), z0 + (j >> 2), f.half);
  }
}
// The staged address of the block from corner (x0,y0,z0) when the whole block is staged.
template <int SS>
FP_DEV const float* stagedBlock(const Stage<SS>& G, const Field& f, int x0, int y0, int z0) {
  if constexpr (SS == 0) return nullptr;
  unsigned lx = (unsigned)(x0 - G.ox), ly = (unsigned)(y0 - G.oy), lz = (unsigned)(z0 - G.oz);
  unsigned lim = (unsigned)(G.S - 1);
  if (lx < lim && ly < lim && lz < lim) return f.sm + ((int)lz * G.S + (int)ly) * G.S + (int)lx;
  return nullptr;
}

// Trilinear sample at `pos` in cell units (fluid-sampling.wgsl:85-114).
template <int SS>
FP_DEV float fieldSample(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& f, int c, float px, float py,
                         float pz) {
  if constexpr (SS > 0) {
    float qx = px - 0.5f, qy = py - 0.5f, qz = pz - 0.5f;
    float gx = floorf(qx), gy = floorf(qy), gz = floorf(qz);
    const float* b = stagedBlock(G, f, (int)gx, (int)gy, (int)gz);
    if (b) {
      float t[8];
      blockCells(P, H, G, f, c, b, 0, 0, 0, t);
      return blend8(t, qx - gx, qy - gy, qz - gz);
    }
    return sampleFar(P, H, f, c, px, py, pz);
  } else {
    return sampleCells(P, H, f.pool, f.ch, c, px, py, pz, f.half);
  }
}

// Copy channels [0, nch) of a pool of `ch` channels over the staged box into shared memory,
// zero where no slot, with asynchronous 4-byte copies (cp.async): every thread keeps all its
// copies in flight and the caller waits once. A brick without a slot reads nothing (source
// size 0 zero-fills). A half pool is widened to FP32 on the way (plain loads: cp.async moves
// at least 4 bytes).
template <int SS>
FP_DEV void stageField(const SimParams& P, const Home& H, const Stage<SS>& G, float* sm, const float* pool, int ch,
                       bool half = false, int nch = 0) {
  constexpr int S = SS > 0 ? SS : 1, S3 = SS * SS * SS;
  if constexpr (SS == 0) return;
  if (nch <= 0) nch = ch;
  for (int i = threadIdx.x; i < S3; i += blockDim.x) {
    int lx = i % S, ly = (i / S) % S, lz = i / (S * S);
    int x = G.ox + lx, y = G.oy + ly, z = G.oz + lz;
    int s = brickSlot(P, H, x >> P.shift, y >> P.shift, z >> P.shift);
    if (half) {
      size_t base = s < 0 ? 0 : (size_t)s * ch * P.N + localCell(P, x, y, z);
      for (int c = 0; c < nch; c++) sm[c * S3 + i] = s < 0 ? 0.f : ldHalf(pool, base + (size_t)c * P.N, true);
      continue;
    }
    const float* src = s < 0 ? pool : pool + (size_t)s * ch * P.N + localCell(P, x, y, z);
    int bytes = s < 0 ? 0 : 4;
    for (int c = 0; c < nch; c++) {
      unsigned dst = (unsigned)__cvta_generic_to_shared(sm + c * S3 + i);
      const float* g = s < 0 ? pool : src + (size_t)c * P.N;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(g), "r"(bytes) : "memory");
    }
  }
}
// Wait for this thread's staged copies, then for every thread's.
FP_DEV void stageWait() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}

template <bool STAGED>
FP_DEV TransportStage<STAGED> stageOf(const SimParams& P, const Home& H) {
  TransportStage<STAGED> G;
  G.ox = H.bx * P.B - HALO;
  G.oy = H.by * P.B - HALO;
  G.oz = H.bz * P.B - HALO;
  return G;
}

// Component c of the staggered velocity at world position p: stored half a cell back along c.
template <int SS>
FP_DEV float velComp(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& v, float px, float py, float pz,
                     int c) {
  float qx = px * P.invH, qy = py * P.invH, qz = pz * P.invH;
  return fieldSample(P, H, G, v, c, c == 0 ? qx - 0.5f : qx, c == 1 ? qy - 0.5f : qy, c == 2 ? qz - 0.5f : qz);
}
// velocityAt through the directory, q in cell units.
FP_DEV float3 velocityCells(const SimParams& P, const Home& H, const Field& v, const float* q) {
  return make_float3(sampleCells(P, H, v.pool, v.ch, 0, q[0] - 0.5f, q[1], q[2], v.half),
                     sampleCells(P, H, v.pool, v.ch, 1, q[0], q[1] - 0.5f, q[2], v.half),
                     sampleCells(P, H, v.pool, v.ch, 2, q[0], q[1], q[2] - 0.5f, v.half));
}
static __device__ __noinline__ float3 velocityFar(const SimParams& P, const Home& H, const Field& v, float qx, float qy,
                                                  float qz) {
  const float q[3] = {qx, qy, qz};
  return velocityCells(P, H, v, q);
}
// velocityAt (fluid-advection.wgsl:17-21): the three staggered samples share their floors
// (per axis: unshifted, and shifted half a cell for the component stored along it) and one
// check that all three blocks are staged.
template <int SS>
FP_DEV float3 velocityAt(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& v, float px, float py,
                         float pz) {
  const float q[3] = {px * P.invH, py * P.invH, pz * P.invH};
  if constexpr (SS > 0) {
    const int o[3] = {G.ox, G.oy, G.oz};
    int i0[3], i1[3];
    float f0[3], f1[3];
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      float u0 = q[a] - 0.5f, u1 = q[a] - 1.f;
      float g0 = floorf(u0), g1 = floorf(u1);
      i0[a] = (int)g0 - o[a];
      i1[a] = (int)g1 - o[a];
      f0[a] = u0 - g0;
      f1[a] = u1 - g1;
      in = in && i1[a] >= 0 && i0[a] < G.S - 1;  // i1 <= i0 <= i1 + 1
    }
    if (in) {
      constexpr int S = SS, S2 = SS * SS;
      float t[8];
      float3 r;
      blockCells(P, H, G, v, 0, v.sm + i0[2] * S2 + i0[1] * S + i1[0], 0, 0, 0, t);
      r.x = blend8(t, f1[0], f0[1], f0[2]);
      blockCells(P, H, G, v, 1, v.sm + i0[2] * S2 + i1[1] * S + i0[0], 0, 0, 0, t);
      r.y = blend8(t, f0[0], f1[1], f0[2]);
      blockCells(P, H, G, v, 2, v.sm + i1[2] * S2 + i0[1] * S + i0[0], 0, 0, 0, t);
      r.z = blend8(t, f0[0], f0[1], f1[2]);
      return r;
    }
    return velocityFar(P, H, v, q[0], q[1], q[2]);
  } else {
    return velocityCells(P, H, v, q);
  }
}
FP_DEV float get(const float3& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// velocityOnFace (fluid-advection.wgsl:26-44): the face's own component is stored; each other
// component k is the trilinear sample at the face centre, which falls midway between two
// cells along c and along k and on the cell plane of the third axis: the mean of four cells.
template <int SS>
FP_DEV float3 velocityOnFace(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& v, int x, int y, int z,
                             int c, float3 orig) {
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (k == c) {
      r[k] = get(orig, k);
      continue;
    }
    const int cx = c == 0, cy = c == 1, cz = c == 2, kx = k == 0, ky = k == 1, kz = k == 2;
    float a = nearCell(P, H, G, v, k, x, y, z), b = nearCell(P, H, G, v, k, x + cx, y + cy, z + cz);
    float d = nearCell(P, H, G, v, k, x - kx, y - ky, z - kz),
          e = nearCell(P, H, G, v, k, x + cx - kx, y + cy - ky, z + cz - kz);
    r[k] = 0.25f * ((a + b) + (d + e));
  }
  return make_float3(r[0], r[1], r[2]);
}
// velocityAt at the centre of cell (x,y,z): each component midway between its two faces.
template <int SS>
FP_DEV float3 centreVelocity(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& v, int x, int y, int z) {
  return make_float3(0.5f * (nearCell(P, H, G, v, 0, x - 1, y, z) + nearCell(P, H, G, v, 0, x, y, z)),
                     0.5f * (nearCell(P, H, G, v, 1, x, y - 1, z) + nearCell(P, H, G, v, 1, x, y, z)),
                     0.5f * (nearCell(P, H, G, v, 2, x, y, z - 1) + nearCell(P, H, G, v, 2, x, y, z)));
}

// packDonor (fluid-advection.wgsl:79-95), 5 bits an axis; 1 << 15 asks for a retrace.
FP_DEV uint32_t packDonor(int ox, int oy, int oz) {
  int bx = ox + 16, by = oy + 16, bz = oz + 16;
  if (bx < 0 || by < 0 || bz < 0 || bx >= 32 || by >= 32 || bz >= 32) return 1u << 15;
  return (uint32_t)bx | ((uint32_t)by << 5) | ((uint32_t)bz << 10);
}

FP_DEV void cellOf(const SimParams& P, const Home& H, int c, int& x, int& y, int& z) {
  int m = P.B - 1;
  x = H.bx * P.B + (c & m);
  y = H.by * P.B + ((c >> P.shift) & m);
  z = H.bz * P.B + (c >> (2 * P.shift));
}

// ---------------------------------------------------------------------------------------
// Predictors: advectVelocityWithBounds (fluid-velocity-transport.wgsl:28-100) and
// advectScalars (fluid-scalar-transport.wgsl:38-142), fused: both read only the velocity and
// the scalars at the start of the step.
// advectVelocityWithBounds (fluid-velocity-transport.wgsl:28-100) at velocity cell (x,y,z),
// offset c of its brick's slot, on the velocity lattice P.
template <int SS>
FP_DEV void predictVelocity(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& V, size_t slot, int c, int x,
                            int y, int z) {
  const size_t N = P.N;
  // The limiter's bounds (the forward 2x2x2 block of each donor cell) are taken where the
  // correction needs them, at the donor, from the same start-of-step velocity.
  const float px = ((float)x + 0.5f) * P.h, py = ((float)y + 0.5f) * P.h, pz = ((float)z + 0.5f) * P.h;
  // solidAt at a cell centre is solidCell of that cell: centre / h + 0.25 floors to it.
  if (solidCell(P, H, x, y, z)) {
    for (int k = 0; k < 3; k++) P.velP[(slot * 3 + k) * N + c] = 0.f;
  } else {
    float3 orig = make_float3(nearCell(P, H, G, V, 0, x, y, z), nearCell(P, H, G, V, 1, x, y, z),
                              nearCell(P, H, G, V, 2, x, y, z));
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
      float face[3] = {px, py, pz};
      face[comp] += 0.5f * P.h;
      float3 fv = velocityOnFace(P, H, G, V, x, y, z, comp, orig);
      float3 vm = velocityAt(P, H, G, V, face[0] - 0.5f * P.dt * fv.x, face[1] - 0.5f * P.dt * fv.y,
                             face[2] - 0.5f * P.dt * fv.z);
      float dep[3] = {face[0] - P.dt * vm.x, face[1] - P.dt * vm.y, face[2] - P.dt * vm.z};
      float sh[3] = {dep[0], dep[1], dep[2]};
      sh[comp] -= 0.5f * P.h;
      // Divided, not multiplied by 1/h: still air lands exactly on a cell boundary here and
      // the donor cell is an integer decision the oracle repeats.
      int bx = (int)floorf(sh[0] / P.h - 0.5f), by = (int)floorf(sh[1] / P.h - 0.5f),
          bz = (int)floorf(sh[2] / P.h - 0.5f);
      P.donors[(slot * 3 + comp) * N + c] = (uint16_t)packDonor(bx - x, by - y, bz - z);
      P.velP[(slot * 3 + comp) * N + c] = velComp(P, H, G, V, dep[0], dep[1], dep[2], comp);
    }
  }
}
// advectScalars (fluid-scalar-transport.wgsl:38-142) at field cell (x,y,z), offset c of its
// brick's slot: P the field lattice, VP the velocity lattice the trace samples.
// GV: the stage of the velocity (on VP's lattice), GF: the stage of the scalars (on P's).
template <int SV, int SF>
FP_DEV void predictScalars(const SimParams& P, const SimParams& VP, const Home& H, const Stage<SV>& GV, const Field& V,
                           const Stage<SF>& GF, const Field& F, size_t slot, int c, int x, int y, int z) {
  const size_t N = P.N;
  // Scalars: a cell-centred RK2 back trace, the predictor and its donors' range.
  const float px = ((float)x + 0.5f) * P.h, py = ((float)y + 0.5f) * P.h, pz = ((float)z + 0.5f) * P.h;
  float3 cv = VP.velDiv == 1 ? centreVelocity(VP, H, GV, V, x, y, z) : velocityAt(VP, H, GV, V, px, py, pz);
  float3 vm = velocityAt(VP, H, GV, V, px - 0.5f * P.dt * cv.x, py - 0.5f * P.dt * cv.y, pz - 0.5f * P.dt * cv.z);
  float dx_ = px - P.dt * vm.x, dy_ = py - P.dt * vm.y, dz_ = pz - P.dt * vm.z;
  // The departure's trilinear block in cell units: corner `base`, fractions `fr`.
  const float dc[3] = {(float)x + (dx_ - px) * P.invH, (float)y + (dy_ - py) * P.invH,
                       (float)z + (dz_ - pz) * P.invH};
  int base[3];
  float fr[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float g = floorf(dc[a]);
    base[a] = (int)g;
    fr[a] = dc[a] - g;
  }
  const float* blk = stagedBlock(GF, F, base[0], base[1], base[2]);
  float out[4];
  float* sb = P.sb + slot * 8 * N;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    float t[8];
    blockCells(P, H, GF, F, k, blk, base[0], base[1], base[2], t);
    out[k] = blend8(t, fr[0], fr[1], fr[2]);
    if (P.maccormack) {
      // The donors' range; FP16-finite for smoke, heat and fuel, [0,1]-anchored for lifetime.
      float lo = k == 2 ? 1.f : 65504.f, hi = k == 2 ? 0.f : -65504.f;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        lo = fminf(lo, t[j]);
        hi = fmaxf(hi, t[j]);
      }
      const int row = k < 2 ? k : 5 - k;  // rows: smoke, heat, fuel, lifetime
      sb[row * N + c] = lo;
      sb[(4 + row) * N + c] = hi;
    }
  }
  if (!P.maccormack) out[2] = clamp01(out[2]);
  else if (P.lifetimeZero) out[2] = 0.f;
  // With coarse smoke the fine smoke channel carries no density
  // (fluid-scalar-transport.wgsl:127, :137).
  if (P.smokeDiv > 1) out[0] = 0.f;
  // The predictor lives within the step: FP32 in every precision, so the limiter compares
  // the corrected value with unrounded predictions.
  for (int k = 0; k < 4; k++) P.fldP[(slot * 4 + k) * N + c] = out[k];
}

// Transport kernels' forms. 0: unstaged (any grid). 1: staged, 8^3 bricks on one lattice.
// 2: staged, a velocity lattice of 8^3 cells a brick under a finer field lattice (velocity
// divisor d > 1 with 8 d field cells a brick side): the velocity is staged once over the brick
// and a HALO-cell rim on its own lattice, the scalars per cube of 8^3 field cells and a HALO rim.
constexpr int CUBE = 8;
template <int SS>
FP_DEV Stage<SS> stageAt(int ox, int oy, int oz) {
  Stage<SS> G;
  G.ox = ox;
  G.oy = oy;
  G.oz = oz;
  return G;
}
// The velocity stage of form 2: the brick on the velocity lattice VP and a HALO rim.
FP_DEV TransportStage<true> velocityStage(const SimParams& VP, const Home& H) {
  return stageAt<8 + 2 * HALO>(H.bx * VP.B - HALO, H.by * VP.B - HALO, H.bz * VP.B - HALO);
}
// velocityStage when S, else no stage.
template <bool S>
FP_DEV TransportStage<S> velocityStageIf(const SimParams& VP, const Home& H) {
  if constexpr (S) return velocityStage(VP, H);
  else return TransportStage<false>{};
}
// The cubes of 8^3 field cells of a brick of B field cells a side: cube k's first cell in the brick.
FP_DEV void cubeOrigin(int B, int k, int& ox, int& oy, int& oz) {
  const int per = B / CUBE;
  ox = (k % per) * CUBE;
  oy = ((k / per) % per) * CUBE;
  oz = k / (per * per) * CUBE;
}

template <int MODE>
FP_DEV void brick_predict(const SimParams* __restrict__ Pp, uint32_t i) {
  __shared__ int nslot[27];
  extern __shared__ float smem[];
  const SimParams& P = *Pp;
  uint32_t id = P.active[i];
  if (!homeOk(P, id)) return;  // the bounds-checked build only
  Home H = enterBrick(P, id, nslot);
  size_t slot = (size_t)nslot[13];
  if constexpr (MODE == 2) {
    const SimParams& VP = *P.vview;
    const TransportStage<true> GV = velocityStage(VP, H);
    Field V{P.vel, 3, smem};
    Field F{P.fld, 4, smem + 3 * GV.S3, P.scalarHalf != 0};
    stageField(VP, H, GV, smem, P.vel, 3);
    stageWait();
    for (int c = threadIdx.x; c < VP.N; c += blockDim.x) {
      int x, y, z;
      cellOf(VP, H, c, x, y, z);
      predictVelocity(VP, H, GV, V, slot, c, x, y, z);
    }
    const int cubes = (P.B / CUBE) * (P.B / CUBE) * (P.B / CUBE);
    for (int k = 0; k < cubes; k++) {
      int ox, oy, oz;
      cubeOrigin(P.B, k, ox, oy, oz);
      const TransportStage<true> GF =
          stageAt<8 + 2 * HALO>(H.bx * P.B + ox - HALO, H.by * P.B + oy - HALO, H.bz * P.B + oz - HALO);
      __syncthreads();  // the previous cube's stage has been read
      stageField(P, H, GF, smem + 3 * GV.S3, P.fld, 4, F.half);
      stageWait();
      for (int q = threadIdx.x; q < CUBE * CUBE * CUBE; q += blockDim.x) {
        const int lx = ox + (q & 7), ly = oy + ((q >> 3) & 7), lz = oz + (q >> 6);
        predictScalars(P, VP, H, GV, V, GF, F, slot, (lz * P.B + ly) * P.B + lx, H.bx * P.B + lx, H.by * P.B + ly,
                       H.bz * P.B + lz);
      }
    }
  } else {
    constexpr bool STAGED = MODE == 1;
    TransportStage<STAGED> G = stageOf<STAGED>(P, H);
    Field V{P.vel, 3, STAGED ? smem : nullptr};
    Field F{P.fld, 4, STAGED ? smem + 3 * G.S3 : nullptr, P.scalarHalf != 0};
    if (STAGED) {
      stageField(P, H, G, smem, P.vel, 3);
      stageField(P, H, G, smem + 3 * G.S3, P.fld, 4, F.half);
      stageWait();
    }
    if (STAGED || P.velDiv == 1) {
      for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
        int x, y, z;
        cellOf(P, H, c, x, y, z);
        predictVelocity(P, H, G, V, slot, c, x, y, z);
        predictScalars(P, P, H, G, V, G, F, slot, c, x, y, z);
      }
    } else {
      // The velocity lattice's cells, then the field lattice's.
      const SimParams& VP = *P.vview;
      for (int c = threadIdx.x; c < VP.N; c += blockDim.x) {
        int x, y, z;
        cellOf(VP, H, c, x, y, z);
        predictVelocity(VP, H, G, V, slot, c, x, y, z);
      }
      for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
        int x, y, z;
        cellOf(P, H, c, x, y, z);
        predictScalars(P, VP, H, G, V, G, F, slot, c, x, y, z);
      }
    }
  }
  __syncthreads();
}
template <int MODE>
__global__ void __launch_bounds__(THREADS, FP_TRANSPORT_CTAS) k_predict(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    brick_predict<MODE>(&P, i);
  }
}

// ---------------------------------------------------------------------------------------
// correctVelocity (fluid-velocity-transport.wgsl:104-179): bounded MacCormack correction.
// ONE: the velocity lattice is the field lattice (velocity divisor 1), known at compile time.
template <bool STAGED, bool ONE>
FP_DEV void brick_correct(const SimParams* __restrict__ Pp, uint32_t i) {
  __shared__ int nslot[27];
  extern __shared__ float smem[];
  const SimParams& P = *Pp;
  uint32_t id = P.active[i];
  if (!homeOk(P, id)) return;  // the bounds-checked build only
  Home H = enterBrick(P, id, nslot);
  TransportStage<STAGED> G = stageOf<STAGED>(P, H);
  Field V{P.vel, 3, STAGED ? smem : nullptr};
  Field Vp{P.velP, 3, STAGED ? smem + 3 * G.S3 : nullptr};
  if (STAGED) {
    stageField(P, H, G, smem, P.vel, 3);
    stageField(P, H, G, smem + 3 * G.S3, P.velP, 3);
    stageWait();
  }
  size_t slot = (size_t)nslot[13];
  const size_t N = P.N;
  for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
    int x, y, z;
    cellOf(P, H, c, x, y, z);
    float px = ((float)x + 0.5f) * P.h, py = ((float)y + 0.5f) * P.h, pz = ((float)z + 0.5f) * P.h;
    bool solid = solidCell<ONE>(P, H, x, y, z);  // solidAt at the cell centre
    float3 orig = make_float3(nearCell(P, H, G, V, 0, x, y, z), nearCell(P, H, G, V, 1, x, y, z),
                              nearCell(P, H, G, V, 2, x, y, z));
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
      float result = 0.f;
      if (!solid) {
        float predicted = nearCell(P, H, G, Vp, comp, x, y, z);
        float face[3] = {px, py, pz};
        face[comp] += 0.5f * P.h;
        uint32_t donor = P.donors[(slot * 3 + comp) * N + c];
        bool retrace = donor == (1u << 15);
        int base[3] = {x + (int)(donor & 31u) - 16, y + (int)((donor >> 5) & 31u) - 16,
                       z + (int)((donor >> 10) & 31u) - 16};
        float3 fv = make_float3(0.f, 0.f, 0.f);
        if (retrace) {
          fv = velocityOnFace(P, H, G, V, x, y, z, comp, orig);
          float3 vm = velocityAt(P, H, G, V, face[0] - 0.5f * P.dt * fv.x, face[1] - 0.5f * P.dt * fv.y,
                                 face[2] - 0.5f * P.dt * fv.z);
          float dep[3] = {face[0] - P.dt * vm.x, face[1] - P.dt * vm.y, face[2] - P.dt * vm.z};
          dep[comp] -= 0.5f * P.h;
          for (int a = 0; a < 3; a++) base[a] = (int)floorf(dep[a] / P.h - 0.5f);  // as in the predictor
        }
        // The bounds of the donor: the start-of-step component over the 2x2x2 block forward of
        // the donor cell (advectVelocityWithBounds' shared-tile min/max,
        // fluid-velocity-transport.wgsl:66-100), zero for a donor brick without a slot.
        float lo = 0.f, hi = 0.f;
        int bs = brickSlot(P, H, base[0] >> P.shift, base[1] >> P.shift, base[2] >> P.shift);
        if (bs >= 0) {
          float t[8];
          blockCells(P, H, G, V, comp, stagedBlock(G, V, base[0], base[1], base[2]), base[0], base[1], base[2], t);
          lo = 1e5f;
          hi = -1e5f;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            lo = fminf(lo, t[j]);
            hi = fmaxf(hi, t[j]);
          }
        }
        if (lo == hi && predicted == lo) {
          result = predicted;
        } else {
          if (!retrace) fv = velocityOnFace(P, H, G, V, x, y, z, comp, orig);
          float3 vm = velocityAt(P, H, G, V, face[0] + 0.5f * P.dt * fv.x, face[1] + 0.5f * P.dt * fv.y,
                                 face[2] + 0.5f * P.dt * fv.z);
          float fw[3] = {face[0] + P.dt * vm.x, face[1] + P.dt * vm.y, face[2] + P.dt * vm.z};
          fw[comp] -= 0.5f * P.h;
          float reversed = fieldSample(P, H, G, Vp, comp, fw[0] * P.invH, fw[1] * P.invH, fw[2] * P.invH);
          float corrected = predicted + 0.5f * (get(orig, comp) - reversed);
          result = (corrected < lo || corrected > hi) ? predicted : corrected;
        }
      }
      P.velC[(slot * 3 + comp) * N + c] = result;
    }
  }
  __syncthreads();
}
template <int MODE>
__global__ void __launch_bounds__(THREADS, FP_TRANSPORT_CTAS) k_correct(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    // the velocity lattice, 8^3 cells a brick in the staged forms
    brick_correct<MODE != 0, MODE == 1>(MODE == 1 ? &P : P.vview, i);
  }
}

// ---------------------------------------------------------------------------------------
// evolveFields (fluid-field-evolution.wgsl:9-84) with correctedScalars
// (fluid-scalar-transport.wgsl:144-199) and recordContent (fluid-content.wgsl:29-64).
template <int MODE>
FP_DEV void brick_evolve(const SimParams* __restrict__ Pp, uint32_t i) {
  __shared__ int nslot[27];
  __shared__ uint32_t busyAll, expandsAll;
  extern __shared__ float smem[];
  const SimParams& P = *Pp;
  uint32_t id = P.active[i];
  if (threadIdx.x == 0) {
    busyAll = 0;
    expandsAll = 0;
  }
  if (!homeOk(P, id)) return;  // the bounds-checked build only
  Home H = enterBrick(P, id, nslot);
  constexpr bool STAGED = MODE != 0;
  const SimParams& VP = MODE == 1 ? P : *P.vview;  // the velocity lattice the traces sample
  Field V{P.vel, 3, STAGED ? smem : nullptr};
  Field Fp{P.fldP, 4, STAGED ? smem + 3 * TransportStage<true>::S3 : nullptr, false};  // the predictor: FP32
  const bool half = P.scalarHalf != 0;  // the state pools
  size_t slot = (size_t)nslot[13];
  const size_t N = P.N;
  int tile = (int)(id >> 6);
  uint32_t busy = 0;
  bool expands = false;
  // One field cell (x,y,z), offset c of the brick's slot; GV stages the velocity, GF the predictor.
  auto cell = [&](const auto& GV, const auto& GF, int c, int x, int y, int z) {
      float px = ((float)x + 0.5f) * P.h, py = ((float)y + 0.5f) * P.h, pz = ((float)z + 0.5f) * P.h;
      bool solid = solidCell<MODE == 1>(P, H, x, y, z);  // solidAt at the cell centre
      float value[4] = {0.f, 0.f, 0.f, 0.f};
      float expansion = 0.f;
      bool injected = false;
      bool cvSampled = false;
      float3 cv = make_float3(0.f, 0.f, 0.f);
      if (!solid) {
        float tr[4];
        if (!P.maccormack) {
          for (int k = 0; k < 4; k++) tr[k] = nearCell(P, H, GF, Fp, k, x, y, z);
        } else {
          const float* b = P.sb + slot * 8 * N;
          float mn0 = b[0 * N + c], mn1 = b[1 * N + c], mn3 = b[2 * N + c], lmin = b[3 * N + c];
          float mx0 = b[4 * N + c], mx1 = b[5 * N + c], mx3 = b[6 * N + c], lmax = b[7 * N + c];
          if (mn0 == mx0 && mn1 == mx1 && mn3 == mx3 && lmin == lmax) {
            tr[0] = mn0;
            tr[1] = mn1;
            tr[2] = clamp01(lmin);
            tr[3] = mn3;
          } else {
            float a0 = nearCell(P, H, GF, Fp, 0, x, y, z), a1 = nearCell(P, H, GF, Fp, 1, x, y, z),
                  a2 = nearCell(P, H, GF, Fp, 2, x, y, z), a3 = nearCell(P, H, GF, Fp, 3, x, y, z);
            cv = VP.velDiv == 1 ? centreVelocity(VP, H, GV, V, x, y, z) : velocityAt(VP, H, GV, V, px, py, pz);
            cvSampled = true;
            float3 vm = velocityAt(VP, H, GV, V, px + 0.5f * P.dt * cv.x, py + 0.5f * P.dt * cv.y, pz + 0.5f * P.dt * cv.z);
            float fx = px + P.dt * vm.x, fy = py + P.dt * vm.y, fz = pz + P.dt * vm.z;
            const size_t o = slot * 4 * N + c;
            float o0 = ldHalf(P.fld, o, half), o1 = ldHalf(P.fld, o + N, half), o2 = ldHalf(P.fld, o + 2 * N, half),
                  o3 = ldHalf(P.fld, o + 3 * N, half);
            // The forward trace's trilinear block of the predictor, in cell units.
            const float fc[3] = {(float)x + (fx - px) * P.invH, (float)y + (fy - py) * P.invH,
                                 (float)z + (fz - pz) * P.invH};
            int base[3];
            float fr[3];
  #pragma unroll
            for (int a = 0; a < 3; a++) {
              float g = floorf(fc[a]);
              base[a] = (int)g;
              fr[a] = fc[a] - g;
            }
            const float* blk = stagedBlock(GF, Fp, base[0], base[1], base[2]);
            float rs[4];
  #pragma unroll
            for (int k = 0; k < 4; k++) {
              float t[8];
              blockCells(P, H, GF, Fp, k, blk, base[0], base[1], base[2], t);
              rs[k] = blend8(t, fr[0], fr[1], fr[2]);
            }
            float r0 = rs[0], r1 = rs[1], r3 = rs[3];
            float lifetime = a2;
            if (lmin != lmax || a2 != lmin) {
              float cl = a2 + 0.5f * (o2 - rs[2]);
              lifetime = (cl < lmin || cl > lmax) ? a2 : cl;
            }
            float c0 = a0 + 0.5f * (o0 - r0), c1 = a1 + 0.5f * (o1 - r1), c3 = a3 + 0.5f * (o3 - r3);
            tr[0] = (c0 < mn0 || c0 > mx0) ? a0 : c0;
            tr[1] = (c1 < mn1 || c1 > mx1) ? a1 : c1;
            tr[2] = clamp01(lifetime);
            tr[3] = (c3 < mn3 || c3 > mx3) ? a3 : c3;
          }
        }
        // With coarse smoke the fine smoke channel stages only this step's source production
        // (fluid-scalar-transport.wgsl:190-199).
        if (P.smokeDiv > 1) tr[0] = 0.f;
        float lifetime = tr[2];
        float prodS = 0.f, prodH = 0.f, injectedFuel = 0.f;
        uint2 list = tileList(P, tile, 0);
        for (uint32_t j = 0; j < list.y; j++) {
          const FpEmitter& e = P.emitters[P.tileLists[list.x + j]];
          float w = emitterWeight(e, px, py, pz);
          if (w == 0.f) continue;
          float2 var = burstVariation(e, px, py, pz, P.seedBits);
          lifetime = fmaxf(lifetime, e.flame * w * var.y);
          prodS += e.smoke * w * P.dt;
          prodH += e.heat * var.x * w * P.dt;
          injectedFuel += e.fuel * w * P.dt;
        }
        // Mesh emission at this cell (fluid-field-evolution.wgsl:33-36).
        if (const FpMeshSource* ms = meshSourceAt(P, H, x, y, z)) {
          lifetime = fmaxf(lifetime, ms->scalar[0]);
          prodS += ms->scalar[2] * P.dt;
          prodH += ms->scalar[1] * P.dt;
          injectedFuel += ms->scalar[3] * P.dt;
        }
        float remaining = 0.f, burned = 0.f;
        if (P.fuelEnabled) {
          remaining = tr[3] + injectedFuel;
          if (tr[1] + prodH >= P.ignition) {
            lifetime = fmaxf(lifetime, fminf(remaining, 1.f));
            float unburned = remaining * expf(-P.burnRate * P.dt);
            burned = remaining - unburned;
            remaining = unburned;
          }
        }
        // evaluateFlame (flame-common.wgsl:30-42)
        float before = clamp01(lifetime);
        float after = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
        if (before > 0.f) {
          const FpFlame& F = P.flame;
          after = fmaxf(0.f, before - F.dt / F.lifespan);
          f0 = F.smoke * F.lifespan * rampIntegral(F, 0, after, before);
          f1 = F.heat * F.lifespan * rampIntegral(F, 1, after, before);
          f2 = F.expansion * (F.lifespan * rampIntegral(F, 2, after, before) / F.dt);
        }
        expansion = f2 + P.flame.expansion * burned / P.dt;
        float dS = tr[0] * expf(-P.dissipation * P.dt) + (prodS + f0) * expf(-P.dissipation * P.dt * 0.5f);
        float dH = tr[1] * expf(-P.cooling * P.dt) + (prodH + f1) * expf(-P.cooling * P.dt * 0.5f);
        value[0] = fmaxf(dS, 0.f);
        value[1] = fmaxf(dH, 0.f);
        value[2] = after;
        value[3] = remaining;
        injected = prodS > 0.f || prodH > 0.f || lifetime > tr[2] || injectedFuel > 0.f;
      }
      // clearDormant (fluid-common.wgsl:8-13)
      if (!injected && value[2] == 0.f && value[0] < 0.001f && value[1] < 0.001f && value[3] < 0.001f)
        value[0] = value[1] = value[2] = value[3] = 0.f;
      for (int k = 0; k < 4; k++) stHalf(P.fldN, (slot * 4 + k) * N + c, value[k], half);
      P.expn[slot * N + c] = expansion;
      if (expansion != 0.f) expands = true;
      // holdsContent and contentSupport (fluid-content.wgsl:22-39).
      if (fmaxf(fmaxf(P.smokeDiv > 1 ? 0.f : value[0], value[2]), value[3]) > P.cutoff) {
        if (!cvSampled) cv = VP.velDiv == 1 ? centreVelocity(VP, H, GV, V, x, y, z) : velocityAt(VP, H, GV, V, px, py, pz);
        int idc[3] = {x, y, z};
        float vv[3] = {cv.x, cv.y, cv.z};
        bool low[3], high[3];
        for (int a = 0; a < 3; a++) {
          float side = (float)P.B;
          float loc = (float)(idc[a] & (P.B - 1)) + 0.5f;
          // two velocity cells of stencil (2 d field cells), and a step of motion
          float pad = fminf(side, fmaxf(2.f, 2.f * (float)P.velDiv) + fabsf(vv[a]) * P.dt / P.h);
          low[a] = loc < pad;
          high[a] = loc + pad >= side;
        }
        uint32_t row = 2u | (low[0] ? 1u : 0u) | (high[0] ? 4u : 0u);
        uint32_t plane = (row << 3u) | (low[1] ? row : 0u) | (high[1] ? (row << 6u) : 0u);
        busy |= (plane << 9u) | (low[2] ? plane : 0u) | (high[2] ? (plane << 18u) : 0u);
      }
  };
  if constexpr (MODE == 2) {
    const TransportStage<true> GV = velocityStage(VP, H);
    stageField(VP, H, GV, smem, P.vel, 3);
    const int cubes = (P.B / CUBE) * (P.B / CUBE) * (P.B / CUBE);
    for (int k = 0; k < cubes; k++) {
      int ox, oy, oz;
      cubeOrigin(P.B, k, ox, oy, oz);
      const TransportStage<true> GF =
          stageAt<8 + 2 * HALO>(H.bx * P.B + ox - HALO, H.by * P.B + oy - HALO, H.bz * P.B + oz - HALO);
      if (k > 0) __syncthreads();  // the previous cube's stage has been read
      stageField(P, H, GF, smem + 3 * GV.S3, P.fldP, 4);
      stageWait();
      for (int q = threadIdx.x; q < CUBE * CUBE * CUBE; q += blockDim.x) {
        const int lx = ox + (q & 7), ly = oy + ((q >> 3) & 7), lz = oz + (q >> 6);
        cell(GV, GF, (lz * P.B + ly) * P.B + lx, H.bx * P.B + lx, H.by * P.B + ly, H.bz * P.B + lz);
      }
    }
  } else {
    TransportStage<STAGED> G = stageOf<STAGED>(P, H);
    if (STAGED) {
      stageField(P, H, G, smem, P.vel, 3);
      stageField(P, H, G, smem + 3 * G.S3, P.fldP, 4);
      stageWait();
    }
    for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
      int x, y, z;
      cellOf(P, H, c, x, y, z);
      cell(G, G, c, x, y, z);
    }
  }
  // recordContent (fluid-content.wgsl:43-64): one update per brick.
  busy = __reduce_or_sync(0xffffffffu, busy);
  uint32_t ex = __reduce_or_sync(0xffffffffu, (uint32_t)expands);
  if ((threadIdx.x & 31) == 0) {
    if (busy) atomicOr(&busyAll, busy);
    if (ex) atomicOr(&expandsAll, 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t flags = 0;
    if (busyAll) {
      flags = FP_CONTENT | (busyAll << 3);
      uint32_t l = id & 63u;
      uint32_t bits = (1u << (l & 3u)) | (16u << ((l >> 2) & 3u)) | (256u << (l >> 4));
      atomicOr(&P.activity[(size_t)P.capacity * 64u + (id >> 6)], bits);
    }
    if (expandsAll) flags |= FP_EXPANDS;
    if (flags) P.activity[id] |= flags;
  }
  __syncthreads();
}
template <int MODE>
__global__ void __launch_bounds__(THREADS, FP_TRANSPORT_CTAS) k_evolve(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    brick_evolve<MODE>(&P, i);
  }
}

// ---------------------------------------------------------------------------------------
// computeCurl (fluid-forces.wgsl:38-75) of the corrected velocity. Staged (8^3 bricks): the
// corrected velocity over the brick and a one-cell rim, every read from shared memory.
template <bool STAGED>
FP_DEV void brick_curl(const SimParams* __restrict__ Pp, uint32_t i) {
  __shared__ int nslot[27];
  extern __shared__ float smem[];
  const SimParams& P = *Pp;
  if (!P.curlOn) return;  // the same for the whole CTA
  if (!homeOk(P, P.active[i])) return;  // the bounds-checked build only
  Home H = enterBrick(P, P.active[i], nslot);
  Stage<STAGED ? 8 + 2 : 0> G;  // staged: 8^3 bricks and a one-cell rim
  G.ox = H.bx * P.B - 1;
  G.oy = H.by * P.B - 1;
  G.oz = H.bz * P.B - 1;
  Field V{P.velC, 3, STAGED ? smem : nullptr};
  if (STAGED) {
    stageField(P, H, G, smem, P.velC, 3);
    stageWait();
  }
  size_t slot = (size_t)nslot[13];
  const size_t N = P.N;
  for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
    int x, y, z;
    cellOf(P, H, c, x, y, z);
    auto cc = [&](int qx, int qy, int qz, int comp) {
      int r[3] = {qx, qy, qz};
      r[comp] -= 1;
      return 0.5f * (nearCell(P, H, G, V, comp, qx, qy, qz) + nearCell(P, H, G, V, comp, r[0], r[1], r[2]));
    };
    float hh = 0.5f / P.h;
    float dx0 = (cc(x + 1, y, z, 1) - cc(x - 1, y, z, 1)) * hh, dx1 = (cc(x + 1, y, z, 2) - cc(x - 1, y, z, 2)) * hh;
    float dy0 = (cc(x, y + 1, z, 0) - cc(x, y - 1, z, 0)) * hh, dy1 = (cc(x, y + 1, z, 2) - cc(x, y - 1, z, 2)) * hh;
    float dz0 = (cc(x, y, z + 1, 0) - cc(x, y, z - 1, 0)) * hh, dz1 = (cc(x, y, z + 1, 1) - cc(x, y, z - 1, 1)) * hh;
    float c0 = dy1 - dz1, c1 = dz0 - dx1, c2 = dx0 - dy0;
    P.curl[(slot * 4 + 0) * N + c] = c0;
    P.curl[(slot * 4 + 1) * N + c] = c1;
    P.curl[(slot * 4 + 2) * N + c] = c2;
    P.curl[(slot * 4 + 3) * N + c] = sqrtf(c0 * c0 + c1 * c1 + c2 * c2);
  }
  __syncthreads();
}
template <bool STAGED>
__global__ void __launch_bounds__(THREADS, 6) k_curl(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    brick_curl<STAGED>(STAGED ? &P : P.vview, i);  // the velocity lattice (staged: the only one)
  }
}

// externalForces with coverage (force-fields.wgsl:312-365).
// meshCovers (force-fields.wgsl:27-47): whether mesh targets of force `index` cover velocity
// cell (x,y,z), from the coverage table.
FP_DEV bool meshCovers(const SimParams& P, const Home& H, uint32_t index, int x, int y, int z) {
  if (!P.forceCoverage) return false;
  int id = brickIdAt(P, H, x >> P.shift, y >> P.shift, z >> P.shift);
  if (id < 0) return false;
  uint32_t first = P.forceCoverage[id];
  if (first == 0xffffffffu) return false;
  const uint32_t bit = (uint32_t)localCell(P, x, y, z), words = 1u + (uint32_t)(P.N + 31) / 32u;
  const uint32_t n = P.forceCoverage[first];
  for (uint32_t e = 0; e < n; e++) {
    const uint32_t row = first + 1u + e * words;
    if (P.forceCoverage[row] == index) return ((P.forceCoverage[row + 1u + (bit >> 5)] >> (bit & 31u)) & 1u) != 0u;
  }
  return false;
}

// externalForces and coverage (force-fields.wgsl:49-103) at velocity cell (x,y,z), centre p.
FP_DEV float3 externalForces(const SimParams& P, const Home& H, int tile, int x, int y, int z, float px, float py,
                             float pz) {
  float3 result = make_float3(0.f, 0.f, 0.f);
  uint2 list = tileList(P, tile, 1);
  for (uint32_t j = 0; j < list.y; j++) {
    const uint32_t index = P.tileLists[list.x + j];
    const FpForce& f = P.forces[index];
    float weight = 1.f;
    if (f.targeted != 0.f && !(f.hasMesh == 1.f && meshCovers(P, H, index, x, y, z))) {
      float covered = 0.f;
      for (int r = 0; r < (int)f.regionCount; r++) {
        const FpRegion& g = P.regions[(int)f.regionFirst + r];
        float dx = fabsf((px - g.center[0]) / fmaxf(g.size[0], 0.03f)),
              dy = fabsf((py - g.center[1]) / fmaxf(g.size[1], 0.03f)),
              dz = fabsf((pz - g.center[2]) / fmaxf(g.size[2], 0.03f));
        float dist = g.box == 3.f ? fmaxf(dx, fmaxf(dy, dz)) : sqrtf(dx * dx + dy * dy + dz * dz);
        covered = fmaxf(covered, 1.f - smooth(0.5f, 1.f, dist));
      }
      weight = covered;
    }
    if (weight == 0.f) continue;
    float3 acc = make_float3(f.axis[0] * f.strength, f.axis[1] * f.strength, f.axis[2] * f.strength);
    if (f.kind == 1.f) {
      float qx = px * f.scale * 0.65f + P.seedF, qy = py * f.scale * 0.65f + -P.time * 0.7f,
            qz = pz * f.scale * 0.65f + P.seedF * 0.25f;
      float3 n1 = curlNoise(P, qx, qy, qz);
      float3 n2 = curlNoise(P, qx * 2.03f + 13.7f, qy * 2.03f + 5.3f, qz * 2.03f + 19.1f);
      acc = make_float3((n1.x + 0.45f * n2.x) * f.strength, (n1.y + 0.45f * n2.y) * f.strength,
                        (n1.z + 0.45f * n2.z) * f.strength);
    } else if (f.kind >= 2.f) {
      float d[3] = {px - f.center[0], py - f.center[1], pz - f.center[2]};
      float r[3] = {d[0], d[1], d[2]};
      if (f.kind == 2.f) {
        float dd = d[0] * f.axis[0] + d[1] * f.axis[1] + d[2] * f.axis[2];
        for (int a = 0; a < 3; a++) r[a] -= f.axis[a] * dd;
      }
      float rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      float distance = sqrtf(rr);
      float radius = fmaxf(f.scale, 0.01f);
      float dir[3];
      for (int a = 0; a < 3; a++) dir[a] = r[a] / fmaxf(distance, radius * 0.25f);
      float falloff = 1.f / (1.f + rr / (radius * radius));
      if (f.kind == 2.f) {
        float cr[3] = {f.axis[1] * dir[2] - f.axis[2] * dir[1], f.axis[2] * dir[0] - f.axis[0] * dir[2],
                       f.axis[0] * dir[1] - f.axis[1] * dir[0]};
        acc = make_float3((cr[0] * f.strength - dir[0] * f.inward + f.axis[0] * f.lift) * falloff,
                          (cr[1] * f.strength - dir[1] * f.inward + f.axis[1] * f.lift) * falloff,
                          (cr[2] * f.strength - dir[2] * f.inward + f.axis[2] * f.lift) * falloff);
      } else {
        acc = make_float3(dir[0] * f.strength * falloff, dir[1] * f.strength * falloff, dir[2] * f.strength * falloff);
      }
    }
    result.x += acc.x * weight;
    result.y += acc.y * weight;
    result.z += acc.z * weight;
  }
  return result;
}

// cellForce / centerForce (fluid-forces.wgsl:79-118).
// The curl is read over the force region and a one-cell rim (Gc, Fc), the evolved scalars
// over the force region (Gs, Fs): staged or through the directory.
template <bool ONE, int SC, int SS>
FP_DEV float3 cellForce(const SimParams& P, const Home& H, const Stage<SC>& Gc, const Field& Fc, const Stage<SS>& Gs,
                        const Field& Fs, int tile, int x, int y, int z) {
  if (brickSlot(P, H, x >> P.shift, y >> P.shift, z >> P.shift) < 0) return make_float3(0.f, 0.f, 0.f);
  float wx = ((float)x + 0.5f) * P.h, wy = ((float)y + 0.5f) * P.h, wz = ((float)z + 0.5f) * P.h;
  if (solidCell<ONE>(P, H, x, y, z)) return make_float3(0.f, 0.f, 0.f);  // solidAt at the centre
  // The evolved scalars of this step (the reference swaps field and corrected first); with a
  // velocity divisor d > 1 their mean over the velocity cell (velocityCellAverage).
  float heat, density;
  if (ONE || P.velDiv == 1) {
    heat = nearCell(P, H, Gs, Fs, 1, x, y, z);
    density = nearCell(P, H, Gs, Fs, 0, x, y, z);
  } else {
    heat = fieldAverage(*P.fview, H, Fs.pool, 4, 1, x, y, z, Fs.half);
    density = fieldAverage(*P.fview, H, Fs.pool, 4, 0, x, y, z, Fs.half);
  }
  // smokeVelocityAverage (smoke.wgsl:4-21): at one velocity cell per smoke spacing or less the
  // evolved coarse density sampled at the cell centre ((x + .5) d_v / d_s in smoke cells, exact),
  // else the mean of its 2x2x2 blocks of smoke cells.
  if (P.smokeDiv > 1) {
    const bool sh = P.scalarHalf != 0;
    const int ratio = (!ONE && P.velDiv > P.smokeDiv) ? P.velDiv / P.smokeDiv : 1;
    if (ratio == 1) {
      const float f = (ONE ? 1.f : (float)P.velDiv) / (float)P.smokeDiv;
      density = smokeSample(P, H, P.smkN, ((float)x + 0.5f) * f, ((float)y + 0.5f) * f, ((float)z + 0.5f) * f, sh);
    } else {
      density = 0.f;
      for (int k = 0; k < ratio; k += 2)
        for (int j = 0; j < ratio; j += 2)
          for (int q = 0; q < ratio; q += 2)
            density += smokeSample(P, H, P.smkN, (float)(x * ratio + q + 1), (float)(y * ratio + j + 1),
                                   (float)(z * ratio + k + 1), sh);
      density /= (float)max(1, (ratio / 2) * (ratio / 2) * (ratio / 2));  // ratio^3 / 8 blocks
    }
  }
  float3 conf = make_float3(0.f, 0.f, 0.f);
  if (P.vorticity != 0.f) {
    float c0 = nearCell(P, H, Gc, Fc, 0, x, y, z), c1 = nearCell(P, H, Gc, Fc, 1, x, y, z),
          c2 = nearCell(P, H, Gc, Fc, 2, x, y, z);
    float e0 = nearCell(P, H, Gc, Fc, 3, x + 1, y, z) - nearCell(P, H, Gc, Fc, 3, x - 1, y, z);
    float e1 = nearCell(P, H, Gc, Fc, 3, x, y + 1, z) - nearCell(P, H, Gc, Fc, 3, x, y - 1, z);
    float e2 = nearCell(P, H, Gc, Fc, 3, x, y, z + 1) - nearCell(P, H, Gc, Fc, 3, x, y, z - 1);
    float len = sqrtf(e0 * e0 + e1 * e1 + e2 * e2) + 0.0001f;
    float n0 = e0 / len, n1 = e1 / len, n2 = e2 / len;
    float s = P.vorticity * P.h;
    conf = make_float3((n1 * c2 - n2 * c1) * s, (n2 * c0 - n0 * c2) * s, (n0 * c1 - n1 * c0) * s);
  }
  float3 ext = externalForces(P, H, tile, x, y, z, wx, wy, wz);
  return make_float3(conf.x + ext.x, conf.y + ext.y + (P.buoyancy * heat - P.smokeWeight * density), conf.z + ext.z);
}

// sourceVelocity (fluid-forces.wgsl:122-149).
// (cx,cy,cz) is the field cell of the face position, the cell after the face on its axis.
template <bool ONE>
FP_DEV float sourceVelocity(const SimParams& P, const Home& H, int tile, float value, float fx, float fy, float fz,
                            int comp, int cx, int cy, int cz) {
  float result = value;
  uint2 list = tileList(P, tile, 0);
  for (uint32_t j = 0; j < list.y; j++) {
    const FpEmitter& e = P.emitters[P.tileLists[list.x + j]];
    if (e.response == 0.f) continue;
    float w = emitterWeight(e, fx, fy, fz);
    if (w == 0.f) continue;
    float radial = 0.f;
    if (e.outward != 0.f) {
      float d0 = fx - e.pos[0], d1 = fy - e.pos[1], d2 = fz - e.pos[2];
      float len = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      float dc = comp == 0 ? d0 : (comp == 1 ? d1 : d2);
      radial = dc / fmaxf(len, 1e-6f) * e.outward;
    }
    result = mixf(result, e.vel[comp] + radial, 1.f - expf(-e.response * w * P.dt));
  }
  // Mesh emission's velocity coupling (fluid-forces.wgsl:143-147), on the field lattice.
  const FpMeshSource* ms = meshSourceAt((ONE || P.velDiv == 1) ? P : *P.fview, H, cx, cy, cz);
  if (ms && ms->motion[3] > 0.f)
    result = mixf(result, ms->motion[comp] / ms->motion[3], 1.f - expf(-ms->motion[3] * P.dt));
  return result;
}

// applyForces (fluid-forces.wgsl:151-182): centre forces of the brick and of the cells past
// it on one axis, staged in shared memory, averaged to the faces. Staged (8^3 bricks): the
// curl over that region and a one-cell rim and the evolved smoke and heat over the region are
// copied to shared memory first.
// The side of the cubes the force kernel walks a brick in: their force tiles fit shared memory.
constexpr int FORCE_SUB = 16;

// MODE 1: 8^3 bricks on one lattice, curl and scalars staged. MODE 2: a velocity lattice of 8^3
// cells a brick under a finer field lattice: the curl staged, the scalars' means (fieldAverage)
// read through the directory. MODE 0: nothing staged.
template <int MODE>
FP_DEV void brick_forces(const SimParams* __restrict__ Pp, uint32_t i) {
  __shared__ int nslot[27];
  extern __shared__ float3 forceTile[];  // (SUB+1)^3, then the staged curl and scalars
  const SimParams& P = *Pp;
  uint32_t id = P.active[i];
  if (!homeOk(P, id)) return;  // the bounds-checked build only
  Home H = enterBrick(P, id, nslot);
  size_t slot = (size_t)nslot[13];
  const size_t N = P.N;
  int tile = (int)(id >> 6);
  // The brick in cubes of SUB cells a side (one cube up to 16^3 bricks, 8 of them in a 32^3
  // brick), each with its centre forces on the cube and one cell beyond its upper faces.
  constexpr bool ONE = MODE == 1, CSTAGED = MODE != 0;
  const int SUB = CSTAGED ? 8 : min(P.B, FORCE_SUB), E = SUB + 1, E3 = E * E * E, per = CSTAGED ? 1 : P.B / SUB;
  float* stage = reinterpret_cast<float*>(forceTile + E3);
  // Staged (8^3 bricks: E = 9): the curl over E + 2 cells a side, two scalars over E.
  Stage<CSTAGED ? 11 : 0> Gc;
  Stage<ONE ? 9 : 0> Gs;
  Gc.ox = H.bx * P.B - 1;
  Gc.oy = H.by * P.B - 1;
  Gc.oz = H.bz * P.B - 1;
  Gs.ox = H.bx * P.B;
  Gs.oy = H.by * P.B;
  Gs.oz = H.bz * P.B;
  const bool half = P.scalarHalf != 0;
  Field Fc{P.curl, 4, CSTAGED ? stage : nullptr};
  Field Fs{P.fldN, 4, ONE ? stage + 4 * Gc.S3 : nullptr, half};
  if (CSTAGED) {
    if (P.vorticity != 0.f) stageField(P, H, Gc, stage, P.curl, 4);
    if (ONE) stageField(P, H, Gs, stage + 4 * Gc.S3, P.fldN, 4, half, 2);  // smoke, heat
    stageWait();
  }
  const float decay = expf(-P.damping * P.dt);
  for (int cube = 0; cube < per * per * per; cube++) {
    const int ox = H.bx * P.B + (cube % per) * SUB, oy = H.by * P.B + ((cube / per) % per) * SUB,
              oz = H.bz * P.B + (cube / (per * per)) * SUB;
    for (int q = threadIdx.x; q < E3; q += blockDim.x) {
      int lx = q % E, ly = (q / E) % E, lz = q / (E * E);
      if ((lx == SUB) + (ly == SUB) + (lz == SUB) >= 2) continue;
      forceTile[q] = cellForce<ONE>(P, H, Gc, Fc, Gs, Fs, tile, ox + lx, oy + ly, oz + lz);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < SUB * SUB * SUB; k += blockDim.x) {
      const int lx = k % SUB, ly = (k / SUB) % SUB, lz = k / (SUB * SUB);
      const int x = ox + lx, y = oy + ly, z = oz + lz;
      const int c = (((z & (P.B - 1)) * P.B) + (y & (P.B - 1))) * P.B + (x & (P.B - 1));
      int t = (lz * E + ly) * E + lx;
      float3 F0 = forceTile[t];
      float f[3] = {0.5f * (F0.x + forceTile[t + 1].x), 0.5f * (F0.y + forceTile[t + E].y),
                    0.5f * (F0.z + forceTile[t + E * E].z)};
      float px = ((float)x + 0.5f) * P.h, py = ((float)y + 0.5f) * P.h, pz = ((float)z + 0.5f) * P.h;
      float out[3];
      for (int a = 0; a < 3; a++) {
        float v = P.velC[(slot * 3 + a) * N + c] * decay + P.dt * f[a];
        float face[3] = {px, py, pz};
        face[a] += 0.5f * P.h;
        // the face's field cell: (x + 1) d on its axis, x d + d/2 on the others (x + 1, x for d = 1)
        const int d = ONE ? 1 : P.velDiv, o = d >> 1;
        out[a] = sourceVelocity<ONE>(P, H, tile, v, face[0], face[1], face[2], a, a == 0 ? (x + 1) * d : x * d + o,
                                        a == 1 ? (y + 1) * d : y * d + o, a == 2 ? (z + 1) * d : z * d + o);
      }
      // enforceFaces (fluid-forces.wgsl:15-31)
      // solidAt at a cell centre is solidCell of that cell: centre / h + 0.25 floors to it.
      if (solidCell<ONE>(P, H, x, y, z)) {
        out[0] = out[1] = out[2] = 0.f;
      } else {
        if (solidCell<ONE>(P, H, x + 1, y, z)) out[0] = 0.f;
        if (solidCell<ONE>(P, H, x, y + 1, z)) out[1] = 0.f;
        if (solidCell<ONE>(P, H, x, y, z + 1)) out[2] = 0.f;
      }
      for (int a = 0; a < 3; a++) P.velF[(slot * 3 + a) * N + c] = out[a];
    }
    __syncthreads();  // the tile is read before the next cube's forces overwrite it
  }
}
template <int MODE>
__global__ void __launch_bounds__(THREADS, FP_TRANSPORT_CTAS) k_forces(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    brick_forces<MODE>(MODE == 1 ? &P : P.vview, i);  // the velocity lattice
  }
}
// Shared memory of the staged force kernel: the (B+1)^3 force tile, the curl over (B+3)^3,
// two scalar channels over (B+1)^3.
constexpr size_t FORCE_STAGED_BYTES = 729 * sizeof(float3) + (4 * 1331 + 2 * 729) * sizeof(float);
constexpr size_t FORCE_CURL_STAGED_BYTES = 729 * sizeof(float3) + 4 * 1331 * sizeof(float);  // MODE 2

// pressureUnknown (fluid-forces.wgsl:210-226): the cell's brick and those of its negative
// neighbours compute.
FP_DEV bool pressureUnknown(const SimParams& P, const Home& H, int x, int y, int z) {
  int sh = P.shift;
  int lx = (x - 1) >> sh, ly = (y - 1) >> sh, lz = (z - 1) >> sh, hx = x >> sh, hy = y >> sh, hz = z >> sh;
  if (P.ground) ly = max(ly, 0);
  for (int bz = lz; bz <= hz; bz++)
    for (int by = ly; by <= hy; by++)
      for (int bx = lx; bx <= hx; bx++)
        if (brickSlot(P, H, bx, by, bz) < 0) return false;
  return true;
}

// pressureUnknown of every cell of the home brick and of the layer past its upper faces, as a
// table built once per brick: a cell's answer depends only on its brick (offset 0 or 1 from the
// home on each axis) and on which axes its brick-local coordinate is 0 (then the brick below on
// that axis must compute too). Bit ((oz*2 + oy)*2 + ox)*8 + (fz*2 + fy)*2 + fx; the ground's
// rule as pressureUnknown's (bricks below y = 0 are not asked). Every thread of the CTA calls it.
FP_DEV uint64_t unknownTable(const SimParams& P, const Home& H, uint32_t* words) {
  const int t = threadIdx.x;
  if (t < 64) {
    const int ox = (t >> 3) & 1, oy = (t >> 4) & 1, oz = t >> 5, fx = t & 1, fy = (t >> 1) & 1, fz = (t >> 2) & 1;
    bool u = true;
    for (int dz = oz - fz; dz <= oz; dz++)
      for (int dy = oy - fy; dy <= oy; dy++)
        for (int dx = ox - fx; dx <= ox; dx++) {
          if (P.ground && H.by + dy < 0) continue;
          if (H.nslot[nbrIndex(dx, dy, dz)] < 0) u = false;
        }
    const uint32_t b = __ballot_sync(0xffffffffu, u);
    if ((t & 31) == 0) words[t >> 5] = b;
  }
  __syncthreads();
  return (uint64_t)words[0] | ((uint64_t)words[1] << 32);
}
// pressureUnknown of cell (x,y,z) of the home brick or of the layer past its upper faces.
FP_DEV bool unknownIn(uint64_t table, const SimParams& P, const Home& H, int x, int y, int z) {
  const int m = P.B - 1;
  const int o = (((z >> P.shift) - H.bz) * 2 + ((y >> P.shift) - H.by)) * 2 + ((x >> P.shift) - H.bx);
  const int f = (((z & m) == 0) * 2 + ((y & m) == 0)) * 2 + ((x & m) == 0);
  return ((table >> (o * 8 + f)) & 1ull) != 0ull;
}

// computeDivergence (fluid-forces.wgsl:184-203) and the finest level's first Jacobi
// iterate from zero (initializePressure, pressure.wgsl:485-505), fused: the iterate needs
// only the cell's own right-hand side.
// ONE: one lattice (velocity divisor 1) known at compile time.
template <bool ONE>
FP_DEV void brick_divergence(const SimParams* __restrict__ Pp, uint32_t i, int pSel) {
  __shared__ int nslot[27];
  __shared__ uint32_t unknownWords[2];
  const SimParams& P = *Pp;
  float* pOut = P.p0[pSel];
  if (!homeOk(P, P.active[i])) return;  // the bounds-checked build only
  Home H = enterBrick(P, P.active[i], nslot);
  const uint64_t unknowns = unknownTable(P, H, unknownWords);
  size_t slot = (size_t)nslot[13];
  const size_t N = P.N;
  for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
    int x, y, z;
    cellOf(P, H, c, x, y, z);
    float d = (P.velF[(slot * 3 + 0) * N + c] - cellAt(P, H, P.velF, 3, 0, x - 1, y, z)) / P.h +
              (P.velF[(slot * 3 + 1) * N + c] - cellAt(P, H, P.velF, 3, 1, x, y - 1, z)) / P.h +
              (P.velF[(slot * 3 + 2) * N + c] - cellAt(P, H, P.velF, 3, 2, x, y, z - 1)) / P.h;
    // The expansion rate is on the field lattice: its mean over the velocity cell
    // (velocityCellAverage, fluid-forces.wgsl:202).
    const float ex =
        (ONE || P.velDiv == 1) ? P.expn[slot * N + c] : fieldAverage(*P.fview, H, P.expn, 1, 0, x, y, z, false);
    float rhs = P.h * P.h * (d - ex);
    P.div[slot * N + c] = rhs;
    uint8_t t = P.topo[0][slot * N + c];
    float first = 0.f;
    if (!(t & FP_STORED_SOLID) && unknownIn(unknowns, P, H, x, y, z)) {
      float diag = (float)((t >> 0) & 1) + (float)((t >> 1) & 1) + ((float)((t >> 2) & 1) + (float)((t >> 3) & 1)) +
                   ((float)((t >> 4) & 1) + (float)((t >> 5) & 1));
      first = mixf(0.f, (0.f - rhs) / fmaxf(diag, 1e-12f), 0.8f);
    }
    pOut[slot * N + c] = first;
  }
  __syncthreads();
}
template <bool ONE>
__global__ void __launch_bounds__(THREADS, 6) k_divergence(FpBatch bt, int pSel) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    brick_divergence<ONE>(ONE ? &P : P.vview, i, pSel);  // the velocity lattice
  }
}

// project (fluid-forces.wgsl:228-262) into the velocity pool of the next step.
template <bool ONE>
FP_DEV void brick_project(const SimParams* __restrict__ Pp, uint32_t i, int pSel) {
  __shared__ int nslot[27];
  __shared__ uint32_t unknownWords[2];
  const SimParams& P = *Pp;
  const float* p = P.p0[pSel];
  if (!homeOk(P, P.active[i])) return;  // the bounds-checked build only
  Home H = enterBrick(P, P.active[i], nslot);
  const uint64_t unknowns = unknownTable(P, H, unknownWords);
  size_t slot = (size_t)nslot[13];
  const size_t N = P.N;
  for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
    int x, y, z;
    cellOf(P, H, c, x, y, z);
    float res[3] = {0.f, 0.f, 0.f};
    if (!solidCell<ONE>(P, H, x, y, z)) {  // solidAt at the cell centre
      float cp = p[slot * N + c];
      bool pu = unknownIn(unknowns, P, H, x, y, z);
      for (int a = 0; a < 3; a++) {
        int n[3] = {x, y, z};
        n[a] += 1;
        float v = P.velF[(slot * 3 + a) * N + c];
        if (solidCell<ONE>(P, H, n[0], n[1], n[2])) {
          res[a] = 0.f;
        } else if (!pu && !unknownIn(unknowns, P, H, n[0], n[1], n[2])) {
          res[a] = 0.f;
        } else {
          float pn = cellAt(P, H, p, 1, 0, n[0], n[1], n[2]);
          res[a] = v - (pn - cp) / P.h;
        }
      }
    }
    for (int a = 0; a < 3; a++) P.velP[(slot * 3 + a) * N + c] = res[a];
  }
  __syncthreads();
}
template <bool ONE>
__global__ void __launch_bounds__(THREADS) k_project(FpBatch bt, int pSel) {
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    brick_project<ONE>(ONE ? &P : P.vview, i, pSel);  // the velocity lattice
  }
}

// buildNoise (curl-noise.wgsl:34-45) once: analytic curl of hashed value noise, rounded to
// half precision as the reference's rgba16float table holds it.
__device__ float nhash(int px, int py, int pz) {
  uint32_t v0 = ((uint32_t)px & 15u) * 1664525u + 1013904223u, v1 = ((uint32_t)py & 15u) * 1664525u + 1013904223u,
           v2 = ((uint32_t)pz & 15u) * 1664525u + 1013904223u;
  v0 += v1 * v2;
  v1 += v2 * v0;
  v2 += v0 * v1;
  v0 ^= v0 >> 16u;
  v1 ^= v1 >> 16u;
  v2 ^= v2 >> 16u;
  v0 += v1 * v2;
  v1 += v2 * v0;
  v2 += v0 * v1;
  return (float)(v0 >> 8u) / 16777216.f;
}
__device__ float3 noiseGradient(float px, float py, float pz) {
  float p[3] = {px, py, pz}, f[3], s[3], ds[3];
  int i[3];
  for (int a = 0; a < 3; a++) {
    i[a] = (int)floorf(p[a]);
    f[a] = p[a] - floorf(p[a]);
    s[a] = f[a] * f[a] * f[a] * (f[a] * (f[a] * 6.f - 15.f) + 10.f);
    ds[a] = 30.f * f[a] * f[a] * (f[a] - 1.f) * (f[a] - 1.f);
  }
  float a = nhash(i[0], i[1], i[2]), b = nhash(i[0] + 1, i[1], i[2]), c = nhash(i[0], i[1] + 1, i[2]),
        d = nhash(i[0] + 1, i[1] + 1, i[2]), e = nhash(i[0], i[1], i[2] + 1), f1 = nhash(i[0] + 1, i[1], i[2] + 1),
        g = nhash(i[0], i[1] + 1, i[2] + 1), h = nhash(i[0] + 1, i[1] + 1, i[2] + 1);
  return make_float3(mixf(mixf(b - a, d - c, s[1]), mixf(f1 - e, h - g, s[1]), s[2]) * ds[0],
                     mixf(mixf(c - a, d - b, s[0]), mixf(g - e, h - f1, s[0]), s[2]) * ds[1],
                     mixf(mixf(e - a, f1 - b, s[0]), mixf(g - c, h - d, s[0]), s[1]) * ds[2]);
}
__global__ void k_noise(float4* __restrict__ out) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 64 * 64 * 64) return;
  int x = idx & 63, y = (idx >> 6) & 63, z = idx >> 12;
  float px = ((float)x + 0.5f) / 64.f * 16.f, py = ((float)y + 0.5f) / 64.f * 16.f, pz = ((float)z + 0.5f) / 64.f * 16.f;
  float3 dx = noiseGradient(px, py, pz), dy = noiseGradient(px + 7.1f, py + 3.7f, pz + 11.3f),
         dz = noiseGradient(px + 5.2f, py + 7.9f, pz + 9.5f);
  float cx = dz.y - dy.z, cy = dx.z - dz.x, cz = dy.x - dx.y;
  out[idx] = make_float4(__half2float(__float2half_rn(cx)), __half2float(__float2half_rn(cy)),
                         __half2float(__float2half_rn(cz)), 0.f);
}

// The projected velocity's divergence: over the cells that are pressure unknowns, not solid,
// with every neighbour an unknown or solid, the sum of squares of h x div u = sum over axes of
// the face differences, and of the cell's three face velocities. FP64 sums per simulation.
__global__ void __launch_bounds__(THREADS) k_post_divergence(FpBatch bt) {
  __shared__ int nslot[27];
  __shared__ double scratch[32];
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = *workSim(bt, FP_WORK_ACTIVE, item, i).vview;  // the velocity lattice
    if (!homeOk(P, P.active[i])) continue;  // the bounds-checked build only
    Home H = enterBrick(P, P.active[i], nslot);
    const size_t slot = (size_t)nslot[13], N = P.N;
    double d2 = 0.0, v2 = 0.0;
    for (int c = threadIdx.x; c < P.N; c += blockDim.x) {
      int x, y, z;
      cellOf(P, H, c, x, y, z);
      auto solid = [&](int qx, int qy, int qz) {
        return solidCell(P, H, qx, qy, qz);  // solidAt at the cell centre
      };
      if (solid(x, y, z) || !pressureUnknown(P, H, x, y, z)) continue;
      bool interior = true;
      const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
      for (int k = 0; k < 6 && interior; k++) {
        int qx = x + off[k][0], qy = y + off[k][1], qz = z + off[k][2];
        interior = solid(qx, qy, qz) || pressureUnknown(P, H, qx, qy, qz);
      }
      if (!interior) continue;
      float u0 = P.velP[(slot * 3 + 0) * N + c], u1 = P.velP[(slot * 3 + 1) * N + c],
            u2 = P.velP[(slot * 3 + 2) * N + c];
      // What the projection drives to zero: h (div u - expansion), the expansion rate the cell's
      // mean on the field lattice as computeDivergence subtracts it (fluid-forces.wgsl:184-203).
      const float ex = P.velDiv == 1 ? P.expn[slot * N + c] : fieldAverage(*P.fview, H, P.expn, 1, 0, x, y, z, false);
      float d = (u0 - cellAt(P, H, P.velP, 3, 0, x - 1, y, z)) + (u1 - cellAt(P, H, P.velP, 3, 1, x, y - 1, z)) +
                (u2 - cellAt(P, H, P.velP, 3, 2, x, y, z - 1)) - P.h * ex;
      d2 += (double)d * (double)d;
      v2 += (double)u0 * u0 + (double)u1 * u1 + (double)u2 * u2;
    }
    d2 = blockSum(d2, scratch);
    v2 = blockSum(v2, scratch);
    if (threadIdx.x == 0) {
      atomicAdd(&P.solver->div2, d2);
      atomicAdd(&P.solver->vel2, v2);
      P.solver->measured = 1;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Coarse smoke (smoke_divisor d > 1, smoke.wgsl): a CTA of 64 threads per computing brick,
// a thread per coarse cell. Positions are world positions of coarse cell centres; velocities
// are the start-of-step velocity, sampled through the directory.
constexpr int SMOKE_THREADS = 64;

struct SmokeCell {
  int q[3];
  float p[3];
};
FP_DEV SmokeCell smokeCellOf(const SimParams& P, const Home& H, int c) {
  const int sh = P.smokeShift, SB = 1 << sh;
  const float sp = P.h * (float)P.smokeDiv;  // voxelSize x d: a power of two, exact
  SmokeCell s;
  s.q[0] = H.bx * SB + (c & (SB - 1));
  s.q[1] = H.by * SB + ((c >> sh) & (SB - 1));
  s.q[2] = H.bz * SB + (c >> (2 * sh));
  for (int a = 0; a < 3; a++) s.p[a] = ((float)s.q[a] + 0.5f) * sp;
  return s;
}
// The coarse smoke field of a brick of 8^3 smoke cells staged with a HALO rim (SmokeStage, on
// the smoke lattice; `on` false: nothing staged). smokeCellS / smokeSampleS read the stage where
// it holds the cell and the directory elsewhere: the same values as smokeCell / smokeSample.
struct SmokeStage {
  int ox, oy, oz;
  bool on;
  const float* st;
  static constexpr int S = 8 + 2 * HALO, S3 = S * S * S;
};
FP_DEV SmokeStage stageSmoke(const SimParams& P, const Home& H, bool on, float* sm, const float* pool, bool half) {
  SmokeStage G;
  G.on = on;
  G.st = sm;
  G.ox = H.bx * 8 - HALO;
  G.oy = H.by * 8 - HALO;
  G.oz = H.bz * 8 - HALO;
  if (!on) return G;
  const int sh = P.smokeShift, m = (1 << sh) - 1;
  for (int i = threadIdx.x; i < SmokeStage::S3; i += blockDim.x) {
    const int x = G.ox + i % SmokeStage::S, y = G.oy + (i / SmokeStage::S) % SmokeStage::S,
              z = G.oz + i / (SmokeStage::S * SmokeStage::S);
    const int s = brickSlot(P, H, x >> sh, y >> sh, z >> sh);
    sm[i] = s < 0 ? 0.f : ldHalf(pool, (size_t)s * P.smokeCells + ((((z & m) << sh) | (y & m)) << sh | (x & m)), half);
  }
  return G;
}
FP_DEV float smokeCellS(const SimParams& P, const Home& H, const SmokeStage& G, const float* pool, int x, int y, int z,
                        bool half) {
  if (G.on) {
    const unsigned lx = (unsigned)(x - G.ox), ly = (unsigned)(y - G.oy), lz = (unsigned)(z - G.oz);
    if (lx < (unsigned)SmokeStage::S && ly < (unsigned)SmokeStage::S && lz < (unsigned)SmokeStage::S)
      return G.st[((int)lz * SmokeStage::S + (int)ly) * SmokeStage::S + (int)lx];
  }
  return smokeCell(P, H, pool, x, y, z, half);
}
FP_DEV float smokeSampleS(const SimParams& P, const Home& H, const SmokeStage& G, const float* pool, float px, float py,
                          float pz, bool half) {
  float qx = px - 0.5f, qy = py - 0.5f, qz = pz - 0.5f;
  float gx = floorf(qx), gy = floorf(qy), gz = floorf(qz);
  int x0 = (int)gx, y0 = (int)gy, z0 = (int)gz;
  float t[8];
#pragma unroll
  for (int j = 0; j < 8; j++) t[j] = smokeCellS(P, H, G, pool, x0 + (j & 1), y0 + ((j >> 1) & 1), z0 + (j >> 2), half);
  return blend8(t, qx - gx, qy - gy, qz - gz);
}

// traceBack / traceForward (fluid-advection.wgsl:67-75) from `p` with centre velocity `cv`.
// G and V: the velocity and its stage (on the velocity lattice), or no stage.
template <int SS>
FP_DEV float3 smokeTrace(const SimParams& P, const Home& H, const Stage<SS>& G, const Field& V, const float* p, float3 cv,
                         float sign) {
  float3 vm = velocityAt(*P.vview, H, G, V, p[0] + sign * 0.5f * P.dt * cv.x, p[1] + sign * 0.5f * P.dt * cv.y,
                         p[2] + sign * 0.5f * P.dt * cv.z);
  return make_float3(p[0] + sign * P.dt * vm.x, p[1] + sign * P.dt * vm.y, p[2] + sign * P.dt * vm.z);
}

// advectSmoke (smoke.wgsl:101-124): the predictor at the back-traced departure and, for
// MacCormack, the donors' range (smokeDonorBounds :63-77: min from 1e30, max from 0).
// VSTAGED: the velocity lattice has 8^3 cells a brick and the smoke grid 8^3 or more: the
// velocity is staged once per brick over the brick and a HALO rim (256 threads a CTA); else
// every velocity sample reads through the directory (64 threads a CTA).
template <bool VSTAGED>
__global__ void __launch_bounds__(VSTAGED ? 256 : SMOKE_THREADS, VSTAGED ? 3 : 8) k_smoke_advect(FpBatch bt) {
  __shared__ int nslot[27];
  extern __shared__ float smem[];
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    if (P.smokeDiv == 1) continue;  // the same for the whole CTA
    if (!homeOk(P, P.active[i])) continue;  // the bounds-checked build only
    Home H = enterBrick(P, P.active[i], nslot);
    const size_t slot = (size_t)nslot[13], SN = (size_t)P.smokeCells;
    const float sp = P.h * (float)P.smokeDiv, invSp = 1.f / sp;
    const bool half = P.scalarHalf != 0;
    const TransportStage<VSTAGED> G = velocityStageIf<VSTAGED>(*P.vview, H);
    Field V{P.vel, 3, VSTAGED ? smem : nullptr};
    SmokeStage GS = stageSmoke(P, H, VSTAGED && P.smokeShift == 3, smem + 3 * G.S3, P.smk, half);
    if (VSTAGED) {
      stageField(*P.vview, H, G, smem, P.vel, 3);
      stageWait();
    }
    for (int c = threadIdx.x; c < P.smokeCells; c += blockDim.x) {
      SmokeCell s = smokeCellOf(P, H, c);
      float density = 0.f;
      if (!solidAt(P, H, s.p[0], s.p[1], s.p[2])) {
        float3 cv = velocityAt(*P.vview, H, G, V, s.p[0], s.p[1], s.p[2]);
        float3 dep = smokeTrace(P, H, G, V, s.p, cv, -1.f);
        density = smokeSampleS(P, H, GS, P.smk, dep.x * invSp, dep.y * invSp, dep.z * invSp, half);
        if (P.maccormack) {
          // The donor block is an integer decision: divided, as the oracle does.
          int bx = (int)floorf(dep.x / sp - 0.5f), by = (int)floorf(dep.y / sp - 0.5f), bz = (int)floorf(dep.z / sp - 0.5f);
          float lo = 1e30f, hi = 0.f;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            float v = smokeCellS(P, H, GS, P.smk, bx + (k & 1), by + ((k >> 1) & 1), bz + (k >> 2), half);
            lo = fminf(lo, v);
            hi = fmaxf(hi, v);
          }
          P.smkB[(slot * 2 + 0) * SN + c] = lo;
          P.smkB[(slot * 2 + 1) * SN + c] = hi;
        }
      }
      P.smkP[slot * SN + c] = density;
    }
    __syncthreads();
  }
}

// contentSupport (fluid-content.wgsl:29-39) on the smoke grid: pads in smoke cells, two at least.
FP_DEV uint32_t smokeSupport(const SimParams& P, const int* q, float3 v) {
  const int SB = 1 << P.smokeShift;
  const float sp = P.h * (float)P.smokeDiv, side = (float)SB;
  const float vv[3] = {v.x, v.y, v.z};
  bool low[3], high[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float loc = (float)(q[a] & (SB - 1)) + 0.5f;
    float pad = fminf(side, fmaxf(2.f, 2.f * ((P.h * (float)P.velDiv) / sp)) + fabsf(vv[a]) * P.dt / sp);
    low[a] = loc < pad;
    high[a] = loc + pad >= side;
  }
  uint32_t row = 2u | (low[0] ? 1u : 0u) | (high[0] ? 4u : 0u);
  uint32_t plane = (row << 3u) | (low[1] ? row : 0u) | (high[1] ? (row << 6u) : 0u);
  return (plane << 9u) | (low[2] ? plane : 0u) | (high[2] ? (plane << 18u) : 0u);
}

// evolveSmoke (smoke.wgsl:126-178): the bounded MacCormack correction, decay, the volume
// average of the evolved fine cells' source production (smokeProduction :23-38: the mean of
// each 2x2x2 block, a trilinear sample at its shared corner), dormant clearing, content flags.
template <bool VSTAGED>
__global__ void __launch_bounds__(VSTAGED ? 256 : SMOKE_THREADS, VSTAGED ? 3 : 8) k_smoke_evolve(FpBatch bt) {
  __shared__ int nslot[27];
  __shared__ uint32_t busyAll;
  extern __shared__ float smem[];
  uint32_t total = workTotal(bt, FP_WORK_ACTIVE);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_ACTIVE, item, i);
    if (P.smokeDiv == 1) continue;  // the same for the whole CTA
    const uint32_t id = P.active[i];
    if (threadIdx.x == 0) busyAll = 0;
    if (!homeOk(P, id)) continue;  // the bounds-checked build only
    Home H = enterBrick(P, id, nslot);
    const size_t slot = (size_t)nslot[13], SN = (size_t)P.smokeCells;
    const int d = P.smokeDiv, blocks = d / 2;
    const float sp = P.h * (float)d, invSp = 1.f / sp, volume = (float)(d * d * d / 8);
    const bool half = P.scalarHalf != 0;
    const TransportStage<VSTAGED> G = velocityStageIf<VSTAGED>(*P.vview, H);
    Field V{P.vel, 3, VSTAGED ? smem : nullptr};
    SmokeStage GS = stageSmoke(P, H, VSTAGED && P.smokeShift == 3, smem + 3 * G.S3, P.smkP, false);
    if (VSTAGED) {
      stageField(*P.vview, H, G, smem, P.vel, 3);
      stageWait();
    }
    uint32_t busy = 0;
    for (int c = threadIdx.x; c < P.smokeCells; c += blockDim.x) {
      SmokeCell s = smokeCellOf(P, H, c);
      float density = 0.f;
      if (!solidAt(P, H, s.p[0], s.p[1], s.p[2])) {
        float3 cv = velocityAt(*P.vview, H, G, V, s.p[0], s.p[1], s.p[2]);
        const float predictor = P.smkP[slot * SN + c];
        float bounded = predictor;
        if (P.maccormack) {
          const float lo = P.smkB[(slot * 2 + 0) * SN + c], hi = P.smkB[(slot * 2 + 1) * SN + c];
          if (lo != hi || predictor != lo) {
            const float original = ldHalf(P.smk, slot * SN + c, half);
            float3 fwd = smokeTrace(P, H, G, V, s.p, cv, 1.f);
            float reversed = smokeSampleS(P, H, GS, P.smkP, fwd.x * invSp, fwd.y * invSp, fwd.z * invSp, false);
            float corrected = predictor + 0.5f * (original - reversed);
            bounded = (corrected < lo || corrected > hi) ? predictor : corrected;
          }
        }
        float produced[4] = {0.f, 0.f, 0.f, 0.f};
        for (int bz = 0; bz < blocks; bz++)
          for (int by = 0; by < blocks; by++)
            for (int bx = 0; bx < blocks; bx++) {
              const float fx = (float)(s.q[0] * d + 2 * bx + 1), fy = (float)(s.q[1] * d + 2 * by + 1),
                          fz = (float)(s.q[2] * d + 2 * bz + 1);
              // sampleCells at the shared corner of a 2x2x2 block of the brick's own field cells
              // (fractions exactly one half): read from the slot directly.
              const int x0 = (int)fx - 1, y0 = (int)fy - 1, z0 = (int)fz - 1;
#pragma unroll
              for (int k = 0; k < 4; k++) {
                float t[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                  t[j] = ldHalf(P.fldN, (slot * 4 + k) * (size_t)P.N + localCell(P, x0 + (j & 1), y0 + ((j >> 1) & 1), z0 + (j >> 2)),
                                half);
                produced[k] += blend8(t, 0.5f, 0.5f, 0.5f);
              }
            }
#pragma unroll
        for (int k = 0; k < 4; k++) produced[k] /= volume;
        density = fmaxf(0.f, bounded * expf(-P.dissipation * P.dt) + produced[0]);
        if (produced[0] == 0.f && produced[2] == 0.f && fmaxf(density, fmaxf(produced[1], produced[3])) < 0.001f)
          density = 0.f;
        if (density > P.cutoff) busy |= smokeSupport(P, s.q, cv);
      }
      stHalf(P.smkN, slot * SN + c, density, half);
    }
    // recordContent (fluid-content.wgsl:43-64)
    busy = __reduce_or_sync(0xffffffffu, busy);
    if ((threadIdx.x & 31) == 0 && busy) atomicOr(&busyAll, busy);
    __syncthreads();
    if (threadIdx.x == 0 && busyAll) {
      uint32_t l = id & 63u;
      uint32_t bits = (1u << (l & 3u)) | (16u << ((l >> 2) & 3u)) | (256u << (l >> 4));
      atomicOr(&P.activity[(size_t)P.capacity * 64u + (id >> 6)], bits);
      P.activity[id] |= FP_CONTENT | (busyAll << 3);
    }
    __syncthreads();
  }
}

}  // namespace

// Staged kernels for 8^3 bricks: `channels` staged fields over (8 + 2 HALO)^3 cells.
static size_t stagedBytes(int channels) {
  const int S = 8 + 2 * HALO;
  return (size_t)channels * S * S * S * sizeof(float);
}
// The velocity lattice 8^3 a brick and the smoke grid 8^3 or finer: the staged forms.
static bool smokeStaged(int B, int vd, int sd) { return B == CUBE * vd && B / sd >= CUBE; }
void fp_launch_smoke_advect(const FpBatch& bt, int B, int vd, int sd, int sms, cudaStream_t st) {
  if (smokeStaged(B, vd, sd))
    k_smoke_advect<true><<<sms * 3, 256, stagedBytes(4), st>>>(bt);
  else
    k_smoke_advect<false><<<sms * 16, SMOKE_THREADS, 0, st>>>(bt);
}
void fp_launch_smoke_evolve(const FpBatch& bt, int B, int vd, int sd, int sms, cudaStream_t st) {
  if (smokeStaged(B, vd, sd))
    k_smoke_evolve<true><<<sms * 3, 256, stagedBytes(4), st>>>(bt);
  else
    k_smoke_evolve<false><<<sms * 16, SMOKE_THREADS, 0, st>>>(bt);
}


// Shared-memory limits of the step kernels, set once before any launch (and so before any
// stream capture of one).
void fp_step_configure(int B) {
  cudaFuncSetAttribute(k_predict<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stagedBytes(7));
  cudaFuncSetAttribute(k_predict<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stagedBytes(7));
  cudaFuncSetAttribute(k_correct<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stagedBytes(6));
  cudaFuncSetAttribute(k_correct<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stagedBytes(6));
  cudaFuncSetAttribute(k_evolve<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stagedBytes(7));
  cudaFuncSetAttribute(k_evolve<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stagedBytes(7));
  const size_t side = (size_t)(B < FORCE_SUB ? B : FORCE_SUB) + 1, smem = side * side * side * sizeof(float3);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_forces<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// The transport kernels' form for bricks of B field cells and velocity divisor vd.
static int transportMode(int B, int vd) { return (B == 8 && vd == 1) ? 1 : ((vd > 1 && B == CUBE * vd) ? 2 : 0); }
void fp_launch_predict(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st) {
  const int mode = transportMode(B, vd);
  if (mode == 1)
    k_predict<1><<<sms * FP_TRANSPORT_CTAS, THREADS, stagedBytes(7), st>>>(bt);
  else if (mode == 2)
    k_predict<2><<<sms * FP_TRANSPORT_CTAS, THREADS, stagedBytes(7), st>>>(bt);
  else
    k_predict<0><<<sms * FP_TRANSPORT_CTAS, THREADS, 0, st>>>(bt);
}
void fp_launch_correct(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st) {
  const int mode = transportMode(B, vd);
  if (mode == 1)
    k_correct<1><<<sms * FP_TRANSPORT_CTAS, THREADS, stagedBytes(6), st>>>(bt);
  else if (mode == 2)
    k_correct<2><<<sms * FP_TRANSPORT_CTAS, THREADS, stagedBytes(6), st>>>(bt);
  else
    k_correct<0><<<sms * FP_TRANSPORT_CTAS, THREADS, 0, st>>>(bt);
}
void fp_launch_evolve(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st) {
  const int mode = transportMode(B, vd);
  if (mode == 1)
    k_evolve<1><<<sms * FP_TRANSPORT_CTAS, THREADS, stagedBytes(7), st>>>(bt);
  else if (mode == 2)
    k_evolve<2><<<sms * FP_TRANSPORT_CTAS, THREADS, stagedBytes(7), st>>>(bt);
  else
    k_evolve<0><<<sms * FP_TRANSPORT_CTAS, THREADS, 0, st>>>(bt);
}
void fp_launch_curl(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st) {
  if (B == 8 && vd == 1)  // staged: 8^3 bricks, one lattice
    k_curl<true><<<sms * 6, THREADS, 3 * 10 * 10 * 10 * sizeof(float), st>>>(bt);
  else
    k_curl<false><<<sms * 6, THREADS, 0, st>>>(bt);
}
void fp_launch_forces(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st) {
  const int mode = transportMode(B, vd);
  if (mode == 1) {  // staged: 8^3 bricks, one lattice
    k_forces<1><<<sms * FP_TRANSPORT_CTAS, THREADS, FORCE_STAGED_BYTES, st>>>(bt);
    return;
  }
  if (mode == 2) {  // the curl staged on a velocity lattice of 8^3 cells a brick
    k_forces<2><<<sms * FP_TRANSPORT_CTAS, THREADS, FORCE_CURL_STAGED_BYTES, st>>>(bt);
    return;
  }
  const size_t side = (size_t)(B < FORCE_SUB ? B : FORCE_SUB) + 1, smem = side * side * side * sizeof(float3);
  k_forces<0><<<sms * FP_TRANSPORT_CTAS, THREADS, smem, st>>>(bt);
}
void fp_launch_divergence(const FpBatch& bt, int pSel, int vd, int sms, cudaStream_t st) {
  if (vd == 1)
    k_divergence<true><<<sms * 6, THREADS, 0, st>>>(bt, pSel);
  else
    k_divergence<false><<<sms * 6, THREADS, 0, st>>>(bt, pSel);
}
void fp_launch_project(const FpBatch& bt, int pSel, int vd, int sms, cudaStream_t st) {
  if (vd == 1)
    k_project<true><<<sms * 4, THREADS, 0, st>>>(bt, pSel);
  else
    k_project<false><<<sms * 4, THREADS, 0, st>>>(bt, pSel);
}
void fp_launch_noise(float4* noise, cudaStream_t st) { k_noise<<<64 * 64 * 64 / 256, 256, 0, st>>>(noise); }
void fp_launch_post_divergence(const FpBatch& bt, int sms, cudaStream_t st) {
  k_post_divergence<<<sms * 4, THREADS, 0, st>>>(bt);
}
