// Mesh colliders and mesh emitters on the GPU: the host-side passes of the reference that turn
// a triangle mesh into the frame's inputs.
//
//   fp_mesh_voxelize  Collider.meshMask (src/library/handles.ts:299-325) and
//                     MeshCollider.voxelize (src/library/MeshCollider.ts:85-167): every triangle
//                     rasterised into the columns of a box of lattice cells (a CTA a triangle,
//                     threads over its columns), the +z crossings counted, placed and sorted per
//                     column, the winding along each column setting the occupancy bits.
//   fp_mesh_splat     MeshSourceRasterizer.prepare (src/engine/MeshSourceRasterizer.ts:64-167):
//                     samples splatted trilinearly into a per-emitter coverage hash, coverage
//                     capped at 1 folded into a cell hash of the summed rates, compacted to
//                     records.
//
// The reference computes in JavaScript doubles; so does this file, with no multiply-add
// contraction (built with -fmad=false), so the voxelisation's edge tests, the decisions that set
// the bits, match the reference's bit for bit. Scratch is allocated per call: these run when a
// mesh moves or an emitter's samples change, not every step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/firepro.h"
#include "fp_error.h"

namespace {

// ---------------------------------------------------------------------------------------
// Voxelisation

struct Box {
  int nx, ny, nz;
  double m[16];     // toBox: world -> the voxelizer's box (column-major)
  double half[2];   // domain x / 2, domain z / 2
  double cell[3];   // domain / resolution, as the reference divides it
};

// A point through a column-major 4x4 with the perspective divide (a homogeneous transform,
// as three.js's Vector3.applyMatrix4 evaluates it: each row summed left to right).
__host__ __device__ inline void transformPoint(const double* e, double x, double y, double z, double* out) {
  double w = 1.0 / (e[3] * x + e[7] * y + e[11] * z + e[15]);
  out[0] = (e[0] * x + e[4] * y + e[8] * z + e[12]) * w;
  out[1] = (e[1] * x + e[5] * y + e[9] * z + e[13]) * w;
  out[2] = (e[2] * x + e[6] * y + e[10] * z + e[14]) * w;
}

// edge (MeshCollider.ts:123-124): twice the signed area of (a, b, (x, y)).
__device__ inline double edgeFn(const double* a, const double* b, double x, double y) {
  return (a[0] - x) * (b[1] - y) - (a[1] - y) * (b[0] - x);
}
// ownsEdge (MeshCollider.ts:125): the top-left rule for a sample exactly on an edge.
__device__ inline bool ownsEdge(const double* a, const double* b) { return b[1] > a[1] || (b[1] == a[1] && b[0] < a[0]); }

struct Crossing {
  double z;
  int sign;
  int pad;
};

// One triangle's box coordinates (MeshCollider.ts:111-121): corners through toBox, then into
// cell units with x and z from the box's centre line.
__device__ inline void corner(const Box& B, const float* pos, const uint32_t* idx, uint32_t k, double* out) {
  uint32_t v = idx ? idx[k] : k;
  double p[3];
  transformPoint(B.m, (double)pos[3 * v], (double)pos[3 * v + 1], (double)pos[3 * v + 2], p);
  out[0] = (p[0] + B.half[0]) / B.cell[0];
  out[1] = p[1] / B.cell[1];
  out[2] = (p[2] + B.half[1]) / B.cell[2];
}

// PASS 0 counts crossings per column; PASS 1 writes them at the column's offset.
template <int PASS>
__global__ void k_vox_raster(Box B, const float* __restrict__ pos, const uint32_t* __restrict__ idx, uint32_t tris,
                             uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                             uint32_t* __restrict__ fill, Crossing* __restrict__ out) {
  for (uint32_t t = blockIdx.x; t < tris; t += gridDim.x) {
    double a[3], b[3], c[3];
    corner(B, pos, idx, 3 * t, a);
    corner(B, pos, idx, 3 * t + 1, b);
    corner(B, pos, idx, 3 * t + 2, c);
    double area = edgeFn(a, b, c[0], c[1]);
    if (area == 0.0) continue;  // the same for the whole CTA
    const int sign = area > 0.0 ? 1 : -1;
    if (area < 0.0) {
      for (int k = 0; k < 3; k++) {
        double s = b[k];
        b[k] = c[k];
        c[k] = s;
      }
      area = -area;
    }
    const double mnx = fmin(fmin(a[0], b[0]), c[0]), mxx = fmax(fmax(a[0], b[0]), c[0]);
    const double mny = fmin(fmin(a[1], b[1]), c[1]), mxy = fmax(fmax(a[1], b[1]), c[1]);
    // Clamped in FP64 before the conversion, so a corner far outside the box converts safely.
    const long x0 = (long)fmax(0.0, ceil(mnx - 0.5)), x1 = (long)fmin((double)(B.nx - 1), floor(mxx - 0.5));
    const long y0 = (long)fmax(0.0, ceil(mny - 0.5)), y1 = (long)fmin((double)(B.ny - 1), floor(mxy - 0.5));
    if (x1 < x0 || y1 < y0) continue;
    const long w = x1 - x0 + 1, n = w * (y1 - y0 + 1);
    for (long q = threadIdx.x; q < n; q += blockDim.x) {
      const long x = x0 + q % w, y = y0 + q / w;
      const double px = (double)x + 0.5, py = (double)y + 0.5;
      const double v0 = edgeFn(b, c, px, py), v1 = edgeFn(c, a, px, py), v2 = edgeFn(a, b, px, py);
      if (v0 < 0.0 || (v0 == 0.0 && !ownsEdge(b, c))) continue;
      if (v1 < 0.0 || (v1 == 0.0 && !ownsEdge(c, a))) continue;
      if (v2 < 0.0 || (v2 == 0.0 && !ownsEdge(a, b))) continue;
      const long col = y * B.nx + x;
      if (PASS == 0) {
        atomicAdd(&counts[col], 1u);
      } else {
        uint32_t at = offsets[col] + atomicAdd(&fill[col], 1u);
        out[at].z = (v0 * a[2] + v1 * b[2] + v2 * c[2]) / area;
        out[at].sign = sign;
      }
    }
  }
}

// Exclusive offsets of the column counts, in one CTA.
__global__ void __launch_bounds__(1024) k_vox_offsets(const uint32_t* __restrict__ counts, uint32_t n,
                                                      uint32_t* __restrict__ offsets, uint32_t* __restrict__ total) {
  __shared__ uint32_t part[1024];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < n; base += 1024) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < n ? counts[i] : 0u;
    part[threadIdx.x] = v;
    __syncthreads();
    for (unsigned off = 1; off < 1024; off <<= 1) {
      uint32_t add = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
      __syncthreads();
      part[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < n) offsets[i] = carry + part[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += part[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// Per column (MeshCollider.ts:155-163): its crossings sorted by depth, then the winding at each
// cell centre z + 0.5; a nonzero winding sets the cell's bit.
__global__ void k_vox_columns(Box B, const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                              Crossing* __restrict__ cr, uint32_t* __restrict__ words) {
  const long columns = (long)B.nx * B.ny;
  for (long col = blockIdx.x * (long)blockDim.x + threadIdx.x; col < columns; col += (long)gridDim.x * blockDim.x) {
    const uint32_t n = counts[col];
    if (n == 0) continue;
    Crossing* c = cr + offsets[col];
    for (uint32_t i = 1; i < n; i++) {  // insertion sort: a column holds a few crossings
      Crossing v = c[i];
      uint32_t j = i;
      while (j > 0 && c[j - 1].z > v.z) {
        c[j] = c[j - 1];
        j--;
      }
      c[j] = v;
    }
    int winding = 0;
    uint32_t cursor = 0;
    for (int z = 0; z < B.nz; z++) {
      while (cursor < n && c[cursor].z <= (double)z + 0.5) winding += c[cursor++].sign;
      if (winding != 0) {
        const uint64_t cell = (uint64_t)z * (uint64_t)columns + (uint64_t)col;
        atomicOr(&words[cell >> 5], 1u << (cell & 31));
      }
    }
  }
}

// Matrix4.multiply (a x b, column-major), each entry summed left to right.
void mul4(const double* a, const double* b, double* out) {
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++)
      out[c * 4 + r] = a[r] * b[c * 4] + a[4 + r] * b[c * 4 + 1] + a[8 + r] * b[c * 4 + 2] + a[12 + r] * b[c * 4 + 3];
}

struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

int deviceError(const char* what, cudaError_t e) {
  return fp_set_error(e == cudaErrorMemoryAllocation ? FP_ENOMEM : FP_EDEVICE,
                      std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------
// Surface splat

constexpr uint64_t EMPTY = ~0ull;
constexpr int COORD_BITS = 21;  // cells within 2^20 of the origin on every axis
constexpr int64_t COORD_LIMIT = (int64_t)1 << (COORD_BITS - 1);

__host__ __device__ inline uint64_t cellKey(int64_t x, int64_t y, int64_t z) {
  const uint64_t m = ((uint64_t)1 << COORD_BITS) - 1;
  return ((uint64_t)(x + COORD_LIMIT) & m) | (((uint64_t)(y + COORD_LIMIT) & m) << COORD_BITS) |
         (((uint64_t)(z + COORD_LIMIT) & m) << (2 * COORD_BITS));
}
__device__ inline uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}
// The slot of `key` in an open-addressed table of `cap` (a power of two) keys; inserted when
// absent. The table is sized at least twice the keys it can receive, so a probe ends.
__device__ inline uint32_t slotOf(unsigned long long* keys, uint32_t cap, uint64_t key) {
  uint32_t s = (uint32_t)(mix64(key) & (cap - 1));
  for (uint32_t probe = 0; probe < cap; probe++) {
    unsigned long long prev = atomicCAS(&keys[s], (unsigned long long)EMPTY, (unsigned long long)key);
    if (prev == EMPTY || prev == key) return s;
    s = (s + 1) & (cap - 1);
  }
  return cap;  // full: unreachable with the sizing above
}

__device__ inline void atomicMaxDouble(double* addr, double v) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long old = *a;
  while (__longlong_as_double((long long)old) < v) {
    unsigned long long prev = atomicCAS(a, old, (unsigned long long)__double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}

struct SplatSource {
  const double* samples;
  const double* weights;
  uint32_t count;
  double area, flame, heat, smoke, fuel, vel[3], response;
};

// One emitter's coverage (MeshSourceRasterizer.ts:106-128): 8 cells a sample.
__global__ void k_splat_cover(SplatSource S, double sp0, double sp1, double sp2, double meanFace,
                              unsigned long long* keys, double* cover, uint32_t cap, int* overflow) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S.count; i += gridDim.x * blockDim.x) {
    const double g[3] = {S.samples[3 * i] / sp0 - 0.5, S.samples[3 * i + 1] / sp1 - 0.5, S.samples[3 * i + 2] / sp2 - 0.5};
    double base[3], f[3];
    for (int a = 0; a < 3; a++) {
      base[a] = floor(g[a]);
      f[a] = g[a] - base[a];
    }
    for (int k = 0; k < 8; k++) {
      const int x = k & 1, y = (k >> 1) & 1, z = k >> 2;
      const double cx = base[0] + x, cy = base[1] + y, cz = base[2] + z;
      if (fabs(cx) >= (double)COORD_LIMIT || fabs(cy) >= (double)COORD_LIMIT || fabs(cz) >= (double)COORD_LIMIT) {
        atomicExch(overflow, 1);
        continue;
      }
      const double tri = (x ? f[0] : 1.0 - f[0]) * (y ? f[1] : 1.0 - f[1]) * (z ? f[2] : 1.0 - f[2]);
      const double value = (S.weights[i] * S.area * tri) / meanFace;
      uint32_t s = slotOf(keys, cap, cellKey((int64_t)cx, (int64_t)cy, (int64_t)cz));
      if (s < cap) atomicAdd(&cover[s], value);
    }
  }
}

// The emitter's covered cells into the cell table (MeshSourceRasterizer.ts:130-155): coverage
// capped at 1 scales the emitter's rates; cells sum them, the flame takes the maximum.
// cells: 8 doubles a slot (flame, heat, smoke, fuel, motion xyz, response).
__global__ void k_splat_fold(SplatSource S, const unsigned long long* __restrict__ ckeys, const double* __restrict__ cover,
                             uint32_t ccap, unsigned long long* keys, double* cells, uint32_t cap) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ccap; i += gridDim.x * blockDim.x) {
    if (ckeys[i] == EMPTY) continue;
    const double mask = fmin(1.0, cover[i]);
    if (mask <= 0.0) continue;
    uint32_t s = slotOf(keys, cap, ckeys[i]);
    if (s >= cap) continue;
    double* c = cells + (size_t)s * 8;
    atomicMaxDouble(&c[0], S.flame * mask);
    atomicAdd(&c[1], S.heat * mask);
    atomicAdd(&c[2], S.smoke * mask);
    atomicAdd(&c[3], S.fuel * mask);
    const double response = S.response * mask;
    atomicAdd(&c[4], S.vel[0] * response);
    atomicAdd(&c[5], S.vel[1] * response);
    atomicAdd(&c[6], S.vel[2] * response);
    atomicAdd(&c[7], response);
  }
}

__global__ void k_splat_compact(const unsigned long long* __restrict__ keys, const double* __restrict__ cells, uint32_t cap,
                                fp_mesh_source* out, uint32_t* count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    if (k == EMPTY) continue;
    const uint64_t m = ((uint64_t)1 << COORD_BITS) - 1;
    fp_mesh_source r;
    r.cell[0] = (int32_t)((int64_t)(k & m) - COORD_LIMIT);
    r.cell[1] = (int32_t)((int64_t)((k >> COORD_BITS) & m) - COORD_LIMIT);
    r.cell[2] = (int32_t)((int64_t)((k >> (2 * COORD_BITS)) & m) - COORD_LIMIT);
    r.cell[3] = 0;
    const double* c = cells + (size_t)i * 8;
    for (int j = 0; j < 4; j++) r.scalar[j] = (float)c[j];
    for (int j = 0; j < 4; j++) r.motion[j] = (float)c[4 + j];
    out[atomicAdd(count, 1u)] = r;
  }
}

uint32_t pow2AtLeast(uint64_t n) {
  uint64_t c = 1024;
  while (c < n) c <<= 1;
  return (uint32_t)std::min<uint64_t>(c, 1u << 31);
}

}  // namespace

extern "C" int fp_mesh_voxelize(int device, const fp_mesh* mesh, const double world[16], double spacing, int32_t lo[3],
                                int32_t dims[3], uint32_t* words, uint32_t* word_count) {
  if (!mesh || !world || !lo || !dims || !word_count || !mesh->positions || mesh->vertex_count == 0)
    return fp_set_error(FP_EINVAL, "fp_mesh_voxelize needs a mesh with positions, a transform and outputs.");
  const uint32_t count = mesh->indices ? mesh->index_count : mesh->vertex_count;
  if (!count || count % 3) return fp_set_error(FP_EINVAL, "Mesh collider geometry must contain complete triangles.");
  if (!(spacing > 0.0) || !std::isfinite(spacing)) return fp_set_error(FP_EINVAL, "spacing must be a positive number.");
  for (int k = 0; k < 16; k++)
    if (!std::isfinite(world[k])) return fp_set_error(FP_EINVAL, "the transform must be finite.");
  // The geometry's bounding box over every vertex, placed by the transform's eight corners
  // (Box3.applyMatrix4), then one cell of margin (handles.ts:306-313).
  double bmin[3] = {INFINITY, INFINITY, INFINITY}, bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t v = 0; v < mesh->vertex_count; v++)
    for (int a = 0; a < 3; a++) {
      double p = (double)mesh->positions[3 * v + a];
      if (!std::isfinite(p)) return fp_set_error(FP_EINVAL, "Mesh collider contains nonfinite positions.");
      bmin[a] = std::min(bmin[a], p);
      bmax[a] = std::max(bmax[a], p);
    }
  if (mesh->indices)
    for (uint32_t i = 0; i < count; i++)
      if (mesh->indices[i] >= mesh->vertex_count)
        return fp_set_error(FP_EINVAL, "Mesh collider contains an invalid triangle index.");
  double wmin[3] = {INFINITY, INFINITY, INFINITY}, wmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int k = 0; k < 8; k++) {
    double p[3];
    transformPoint(world, (k & 1) ? bmax[0] : bmin[0], (k & 2) ? bmax[1] : bmin[1], (k & 4) ? bmax[2] : bmin[2], p);
    for (int a = 0; a < 3; a++) {
      wmin[a] = std::min(wmin[a], p[a]);
      wmax[a] = std::max(wmax[a], p[a]);
    }
  }
  long size[3];
  for (int a = 0; a < 3; a++) {
    double l = std::floor(wmin[a] / spacing) - 1.0, h = std::ceil(wmax[a] / spacing) + 1.0;
    if (!(std::fabs(l) < 1e9 && std::fabs(h) < 1e9)) return fp_set_error(FP_EINVAL, "the mesh lies too far from the origin.");
    lo[a] = (int32_t)l;
    size[a] = (long)(h - l);
    dims[a] = (int32_t)size[a];
  }
  const uint64_t cells = (uint64_t)size[0] * size[1] * size[2];
  if (cells > ((uint64_t)1 << 32)) return fp_set_error(FP_ELIMIT, "the mesh collider's box exceeds 2^32 cells.");
  const uint32_t need = (uint32_t)((cells + 31) / 32);
  const uint32_t have = *word_count;
  *word_count = need;
  if (!words || have < need) return FP_OK;  // the sizes only
  // toBox (handles.ts:315-322): the translation that centres the box in x and z and puts its
  // floor at y = 0, times the transform; then the voxelizer's cell size (MeshCollider.ts:109).
  Box B;
  B.nx = (int)size[0];
  B.ny = (int)size[1];
  B.nz = (int)size[2];
  double T[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  T[12] = -((double)lo[0] + (double)size[0] / 2.0) * spacing;
  T[13] = -(double)lo[1] * spacing;
  T[14] = -((double)lo[2] + (double)size[2] / 2.0) * spacing;
  mul4(T, world, B.m);
  double domain[3];
  for (int a = 0; a < 3; a++) {
    domain[a] = (double)size[a] * spacing;
    B.cell[a] = domain[a] / (double)size[a];
  }
  B.half[0] = domain[0] / 2.0;
  B.half[1] = domain[2] / 2.0;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return deviceError("cudaSetDevice", e);
  Scratch S;
  const uint64_t columns = (uint64_t)B.nx * B.ny;
  const uint32_t tris = count / 3;
  float* pos = S.get<float>((size_t)mesh->vertex_count * 3);
  uint32_t* idx = mesh->indices ? S.get<uint32_t>(count) : nullptr;
  uint32_t* counts = S.get<uint32_t>(columns);
  uint32_t* offsets = S.get<uint32_t>(columns);
  uint32_t* fill = S.get<uint32_t>(columns);
  uint32_t* total = S.get<uint32_t>(1);
  uint32_t* bits = S.get<uint32_t>(need);
  if (!pos || (mesh->indices && !idx) || !counts || !offsets || !fill || !total || !bits)
    return fp_set_error(FP_ENOMEM, "out of device memory for the voxelization");
  cudaMemcpy(pos, mesh->positions, (size_t)mesh->vertex_count * 12, cudaMemcpyHostToDevice);
  if (idx) cudaMemcpy(idx, mesh->indices, (size_t)count * 4, cudaMemcpyHostToDevice);
  cudaMemset(counts, 0, columns * 4);
  cudaMemset(fill, 0, columns * 4);
  cudaMemset(bits, 0, (size_t)need * 4);
  const int grid = (int)std::min<uint32_t>(tris, 148u * 16u);
  k_vox_raster<0><<<grid, 128>>>(B, pos, idx, tris, counts, nullptr, nullptr, nullptr);
  k_vox_offsets<<<1, 1024>>>(counts, (uint32_t)columns, offsets, total);
  uint32_t crossings = 0;
  if ((e = cudaMemcpy(&crossings, total, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) return deviceError("voxelize", e);
  Crossing* cr = S.get<Crossing>(crossings);
  if (!cr) return fp_set_error(FP_ENOMEM, "out of device memory for the voxelization");
  k_vox_raster<1><<<grid, 128>>>(B, pos, idx, tris, nullptr, offsets, fill, cr);
  k_vox_columns<<<(int)std::min<uint64_t>((columns + 255) / 256, 148 * 8), 256>>>(B, counts, offsets, cr, bits);
  if ((e = cudaMemcpy(words, bits, (size_t)need * 4, cudaMemcpyDeviceToHost)) != cudaSuccess) return deviceError("voxelize", e);
  return FP_OK;
}

extern "C" int fp_mesh_splat(int device, const fp_mesh_emitter* emitters, uint32_t emitter_count, double spacing,
                             fp_mesh_source* records, uint32_t* count) {
  if (!count || (emitter_count && !emitters)) return fp_set_error(FP_EINVAL, "fp_mesh_splat needs emitters and a count.");
  if (!(spacing > 0.0) || !std::isfinite(spacing)) return fp_set_error(FP_EINVAL, "spacing must be a positive number.");
  // The reference's checks (MeshSourceRasterizer.ts:95-101), before any work.
  uint64_t visits = 0, samples = 0;
  for (uint32_t k = 0; k < emitter_count; k++) {
    const fp_mesh_emitter& m = emitters[k];
    if ((m.sample_count && (!m.samples || !m.weights)) || !(m.surface_area > 0))
      return fp_set_error(FP_EINVAL, "Mesh sources require surface samples and a positive surface area.");
    visits += (uint64_t)m.sample_count * 8;
    if (visits > 2000000) return fp_set_error(FP_EINVAL, "Mesh source sampling exceeds two million cell visits.");
    samples = std::max<uint64_t>(samples, m.sample_count);
  }
  samples = std::max<uint64_t>(samples, 1);
  const uint32_t capacity = *count;
  if (emitter_count == 0) {
    *count = 0;
    return FP_OK;
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return deviceError("cudaSetDevice", e);
  Scratch S;
  const uint32_t ccap = pow2AtLeast(samples * 8 * 2), cap = pow2AtLeast(visits * 2);
  unsigned long long* ckeys = S.get<unsigned long long>(ccap);
  double* cover = S.get<double>(ccap);
  unsigned long long* keys = S.get<unsigned long long>(cap);
  double* cells = S.get<double>((size_t)cap * 8);
  double* dev = S.get<double>(samples * 4);
  int* overflow = S.get<int>(1);
  uint32_t* n = S.get<uint32_t>(1);
  fp_mesh_source* out = S.get<fp_mesh_source>(cap);
  if (!ckeys || !cover || !keys || !cells || !dev || !overflow || !n || !out)
    return fp_set_error(FP_ENOMEM, "out of device memory for the splat");
  cudaMemset(keys, 0xff, (size_t)cap * 8);
  cudaMemset(cells, 0, (size_t)cap * 64);
  cudaMemset(overflow, 0, 4);
  cudaMemset(n, 0, 4);
  // meanFaceArea (MeshSourceRasterizer.ts:102-103) of a cubic lattice.
  const double meanFace = (spacing * spacing + spacing * spacing + spacing * spacing) / 3.0;
  for (uint32_t k = 0; k < emitter_count; k++) {
    const fp_mesh_emitter& m = emitters[k];
    if (m.sample_count == 0) continue;
    cudaMemcpy(dev, m.samples, (size_t)m.sample_count * 24, cudaMemcpyHostToDevice);
    cudaMemcpy(dev + 3 * (size_t)samples, m.weights, (size_t)m.sample_count * 8, cudaMemcpyHostToDevice);
    SplatSource src{dev, dev + 3 * (size_t)samples, m.sample_count, m.surface_area, m.flame, m.heat_rate, m.smoke_rate,
                    m.fuel_rate, {m.velocity[0], m.velocity[1], m.velocity[2]}, m.velocity_response};
    cudaMemset(ckeys, 0xff, (size_t)ccap * 8);
    cudaMemset(cover, 0, (size_t)ccap * 8);
    k_splat_cover<<<std::max(1u, std::min(148u * 8u, (m.sample_count + 255) / 256)), 256>>>(
        src, spacing, spacing, spacing, meanFace, ckeys, cover, ccap, overflow);
    k_splat_fold<<<std::min(148u * 8u, (ccap + 255) / 256), 256>>>(src, ckeys, cover, ccap, keys, cells, cap);
  }
  k_splat_compact<<<std::min(148u * 8u, (cap + 255) / 256), 256>>>(keys, cells, cap, out, n);
  uint32_t got = 0;
  int over = 0;
  if ((e = cudaMemcpy(&got, n, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) return deviceError("splat", e);
  cudaMemcpy(&over, overflow, 4, cudaMemcpyDeviceToHost);
  if (over) return fp_set_error(FP_ELIMIT, "a mesh source sample lies more than 2^20 cells from the origin.");
  *count = got;
  if (!records || capacity < got) return records ? fp_set_error(FP_ELIMIT, "the records do not fit: " + std::to_string(got) + " needed.") : FP_OK;
  std::vector<fp_mesh_source> host(got);
  if (got && (e = cudaMemcpy(host.data(), out, (size_t)got * sizeof(fp_mesh_source), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return deviceError("splat", e);
  std::sort(host.begin(), host.end(), [](const fp_mesh_source& a, const fp_mesh_source& b) {
    if (a.cell[0] != b.cell[0]) return a.cell[0] < b.cell[0];
    if (a.cell[1] != b.cell[1]) return a.cell[1] < b.cell[1];
    return a.cell[2] < b.cell[2];
  });
  if (got) std::memcpy(records, host.data(), (size_t)got * sizeof(fp_mesh_source));
  return FP_OK;
}
