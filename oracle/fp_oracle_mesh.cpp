// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// The oracle of the mesh passes: Collider.meshMask (src/library/handles.ts:299-325) with
// MeshCollider.voxelize (src/library/MeshCollider.ts:85-167), and MeshSourceRasterizer.prepare
// (src/engine/MeshSourceRasterizer.ts:64-167), restated in FP64 in the reference's own order:
// crossings collected column by column in triangle order and sorted, coverage summed sample by
// sample into an ordered map, emitters folded in order. Built without contraction
// (-ffp-contract=off), as the reference's JavaScript numbers round.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "../include/firepro.h"

namespace {

void applyMatrix4(const double* e, double x, double y, double z, double* out) {
  double w = 1.0 / (e[3] * x + e[7] * y + e[11] * z + e[15]);
  out[0] = (e[0] * x + e[4] * y + e[8] * z + e[12]) * w;
  out[1] = (e[1] * x + e[5] * y + e[9] * z + e[13]) * w;
  out[2] = (e[2] * x + e[6] * y + e[10] * z + e[14]) * w;
}

void multiply(const double* a, const double* b, double* te) {
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++)
      te[c * 4 + r] = a[r] * b[c * 4] + a[4 + r] * b[c * 4 + 1] + a[8 + r] * b[c * 4 + 2] + a[12 + r] * b[c * 4 + 3];
}

double edge(const double* a, const double* b, double x, double y) { return (a[0] - x) * (b[1] - y) - (a[1] - y) * (b[0] - x); }
bool ownsEdge(const double* a, const double* b) { return b[1] > a[1] || (b[1] == a[1] && b[0] < a[0]); }

}  // namespace

extern "C" {

// lo, dims and the occupancy bits (x fastest) of the mesh under `world`; returns the words
// written, or -1 when `capacity` is short.
int64_t or_mesh_voxelize(const float* positions, uint32_t vertexCount, const uint32_t* indices, uint32_t indexCount,
                         const double* world, double spacing, int32_t* lo, int32_t* dims, uint32_t* words,
                         uint64_t capacity) {
  const uint32_t count = indices ? indexCount : vertexCount;
  // handles.ts:306-313: the bounding box of every vertex, through the transform's corners.
  double bmin[3] = {INFINITY, INFINITY, INFINITY}, bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t v = 0; v < vertexCount; v++)
    for (int a = 0; a < 3; a++) {
      bmin[a] = std::min(bmin[a], (double)positions[3 * v + a]);
      bmax[a] = std::max(bmax[a], (double)positions[3 * v + a]);
    }
  double wmin[3] = {INFINITY, INFINITY, INFINITY}, wmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int k = 0; k < 8; k++) {
    double p[3];
    applyMatrix4(world, (k & 1) ? bmax[0] : bmin[0], (k & 2) ? bmax[1] : bmin[1], (k & 4) ? bmax[2] : bmin[2], p);
    for (int a = 0; a < 3; a++) {
      wmin[a] = std::min(wmin[a], p[a]);
      wmax[a] = std::max(wmax[a], p[a]);
    }
  }
  double l[3], size[3];
  for (int a = 0; a < 3; a++) {
    l[a] = std::floor(wmin[a] / spacing) - 1;
    size[a] = std::ceil(wmax[a] / spacing) + 1 - l[a];
    lo[a] = (int32_t)l[a];
    dims[a] = (int32_t)size[a];
  }
  double T[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  T[12] = -(l[0] + size[0] / 2) * spacing;
  T[13] = -l[1] * spacing;
  T[14] = -(l[2] + size[2] / 2) * spacing;
  double toBox[16];
  multiply(T, world, toBox);
  // MeshCollider.voxelize
  const int nx = (int)size[0], ny = (int)size[1], nz = (int)size[2];
  double domain[3], cell[3];
  for (int a = 0; a < 3; a++) {
    domain[a] = size[a] * spacing;
    cell[a] = domain[a] / size[a];
  }
  std::vector<double> v((size_t)count * 3);
  for (uint32_t k = 0; k < count; k++) {
    uint32_t vi = indices ? indices[k] : k;
    double p[3];
    applyMatrix4(toBox, positions[3 * vi], positions[3 * vi + 1], positions[3 * vi + 2], p);
    v[3 * k] = (p[0] + domain[0] / 2) / cell[0];
    v[3 * k + 1] = p[1] / cell[1];
    v[3 * k + 2] = (p[2] + domain[2] / 2) / cell[2];
  }
  std::vector<std::vector<std::pair<double, int>>> columns((size_t)nx * ny);
  for (size_t off = 0; off + 9 <= v.size(); off += 9) {
    double a[3], b[3], c[3];
    std::memcpy(a, &v[off], 24);
    std::memcpy(b, &v[off + 3], 24);
    std::memcpy(c, &v[off + 6], 24);
    double area = edge(a, b, c[0], c[1]);
    if (area == 0) continue;
    int sign = area > 0 ? 1 : -1;
    if (area < 0) {
      std::swap(b, c);
      area = -area;
    }
    double x0 = std::max(0.0, std::ceil(std::min({a[0], b[0], c[0]}) - 0.5));
    double x1 = std::min((double)(nx - 1), std::floor(std::max({a[0], b[0], c[0]}) - 0.5));
    double y0 = std::max(0.0, std::ceil(std::min({a[1], b[1], c[1]}) - 0.5));
    double y1 = std::min((double)(ny - 1), std::floor(std::max({a[1], b[1], c[1]}) - 0.5));
    for (double y = y0; y <= y1; y++)
      for (double x = x0; x <= x1; x++) {
        double values[3] = {edge(b, c, x + 0.5, y + 0.5), edge(c, a, x + 0.5, y + 0.5), edge(a, b, x + 0.5, y + 0.5)};
        const double* from[3] = {b, c, a};
        const double* to[3] = {c, a, b};
        bool out = false;
        for (int i = 0; i < 3; i++) out = out || values[i] < 0 || (values[i] == 0 && !ownsEdge(from[i], to[i]));
        if (out) continue;
        columns[(size_t)y * nx + (size_t)x].push_back({(values[0] * a[2] + values[1] * b[2] + values[2] * c[2]) / area, sign});
      }
  }
  const uint64_t cells = (uint64_t)nx * ny * nz, need = (cells + 31) / 32;
  if (!words || capacity < need) return -1;
  std::memset(words, 0, need * 4);
  for (size_t col = 0; col < columns.size(); col++) {
    auto& cr = columns[col];
    std::stable_sort(cr.begin(), cr.end(), [](const std::pair<double, int>& p, const std::pair<double, int>& q) {
      return p.first < q.first;
    });
    int winding = 0;
    size_t cursor = 0;
    for (int z = 0; z < nz; z++) {
      while (cursor < cr.size() && cr[cursor].first <= z + 0.5) winding += cr[cursor++].second;
      if (winding != 0) {
        uint64_t bit = (uint64_t)z * nx * ny + col;
        words[bit >> 5] |= 1u << (bit & 31);
      }
    }
  }
  return (int64_t)need;
}

// MeshSourceRasterizer.prepare: the records, ascending by (x, y, z); returns the count, or -1
// when `capacity` is short.
int64_t or_mesh_splat(const fp_mesh_emitter* emitters, uint32_t count, double spacing, fp_mesh_source* records,
                      uint64_t capacity) {
  struct Cell {
    double flame = 0, heat = 0, smoke = 0, fuel = 0, mx = 0, my = 0, mz = 0, response = 0;
  };
  std::map<std::tuple<int64_t, int64_t, int64_t>, Cell> cells;
  const double meanFace = (spacing * spacing + spacing * spacing + spacing * spacing) / 3;
  for (uint32_t k = 0; k < count; k++) {
    const fp_mesh_emitter& s = emitters[k];
    std::map<std::tuple<int64_t, int64_t, int64_t>, double> coverage;
    for (uint32_t i = 0; i < s.sample_count; i++) {
      double g[3], base[3], f[3];
      for (int a = 0; a < 3; a++) {
        g[a] = s.samples[3 * i + a] / spacing - 0.5;
        base[a] = std::floor(g[a]);
        f[a] = g[a] - base[a];
      }
      for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
          for (int x = 0; x < 2; x++) {
            double tri = (x ? f[0] : 1 - f[0]) * (y ? f[1] : 1 - f[1]) * (z ? f[2] : 1 - f[2]);
            double value = (s.weights[i] * s.surface_area * tri) / meanFace;
            coverage[{(int64_t)(base[0] + x), (int64_t)(base[1] + y), (int64_t)(base[2] + z)}] += value;
          }
    }
    for (auto& kv : coverage) {
      double mask = std::min(1.0, kv.second);
      if (mask <= 0) continue;
      Cell& c = cells[kv.first];
      c.flame = std::max(c.flame, s.flame * mask);
      c.heat += s.heat_rate * mask;
      c.smoke += s.smoke_rate * mask;
      c.fuel += s.fuel_rate * mask;
      double response = s.velocity_response * mask;
      c.mx += s.velocity[0] * response;
      c.my += s.velocity[1] * response;
      c.mz += s.velocity[2] * response;
      c.response += response;
    }
  }
  if (!records || capacity < cells.size()) return cells.size() ? -1 : 0;
  size_t r = 0;
  for (auto& kv : cells) {
    fp_mesh_source& o = records[r++];
    o.cell[0] = (int32_t)std::get<0>(kv.first);
    o.cell[1] = (int32_t)std::get<1>(kv.first);
    o.cell[2] = (int32_t)std::get<2>(kv.first);
    o.cell[3] = 0;
    const Cell& c = kv.second;
    o.scalar[0] = (float)c.flame;
    o.scalar[1] = (float)c.heat;
    o.scalar[2] = (float)c.smoke;
    o.scalar[3] = (float)c.fuel;
    o.motion[0] = (float)c.mx;
    o.motion[1] = (float)c.my;
    o.motion[2] = (float)c.mz;
    o.motion[3] = (float)c.response;
  }
  return (int64_t)cells.size();
}

}  // extern "C"
