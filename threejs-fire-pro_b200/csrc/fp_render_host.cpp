// Host side of the volume render (fp_render.cu): the blackbody table, the render box and
// Engine::render.
#include <algorithm>
#include <array>
#include <map>
#include <cmath>
#include <cstring>
#include <vector>

#include "fp_engine.hpp"
#include "fp_render.h"

// blackbodyTable (src/engine/blackbody.ts:1-97): Planck radiance integrated against the
// multi-lobe CIE 1931 observer fit of Wyman, Sloan and Shirley (JCGT 2013, Table 1) at 5 nm
// from 360 nm, converted to linear sRGB, each entry peak-normalised with its log2 radiance
// relative to 1800 K; 500 K to 10000 K.
static const double kLobes[3][3][4] = {
    {{0.362, 442, 0.0624, 0.0374}, {1.056, 599.8, 0.0264, 0.0323}, {-0.065, 501.1, 0.049, 0.0382}},
    {{0.821, 568.8, 0.0213, 0.0247}, {0.286, 530.9, 0.0613, 0.0322}, {0, 0, 0, 0}},
    {{1.217, 437, 0.0845, 0.0278}, {0.681, 459, 0.0385, 0.0725}, {0, 0, 0, 0}}};
static const int kLobeCount[3] = {3, 2, 2};

static void blackbodyRGB(double kelvin, double rgb[3]) {
  const double h = 6.62607015e-34, c = 299792458.0, k = 1.380649e-23;
  double xyz[3] = {0, 0, 0};
  for (int i = 0; i < 95; i++) {
    double wavelength = 360.0 + i * 5.0;
    double w = wavelength * 1e-9;
    double radiance = 2.0 * h * c * c / (std::pow(w, 5) * std::expm1(h * c / (w * k * kelvin))) * 5e-9;
    for (int ch = 0; ch < 3; ch++) {
      double s = 0.0;
      for (int l = 0; l < kLobeCount[ch]; l++) {
        const double* L = kLobes[ch][l];
        double d = (wavelength - L[1]) * (wavelength < L[1] ? L[2] : L[3]);
        s += L[0] * std::exp(-0.5 * d * d);
      }
      xyz[ch] += s * radiance;
    }
  }
  rgb[0] = std::max(0.0, 3.2406 * xyz[0] - 1.5372 * xyz[1] - 0.4986 * xyz[2]);
  rgb[1] = std::max(0.0, -0.9689 * xyz[0] + 1.8758 * xyz[1] + 0.0415 * xyz[2]);
  rgb[2] = std::max(0.0, 0.0557 * xyz[0] - 0.204 * xyz[1] + 1.057 * xyz[2]);
}

void fp_blackbody_table(float* out4) {
  double ref[3];
  blackbodyRGB(1800.0, ref);
  double refPeak = std::max(ref[0], std::max(ref[1], ref[2]));
  for (int i = 0; i < FP_BLACKBODY_SIZE; i++) {
    double kelvin = 500.0 + (10000.0 - 500.0) * i / (FP_BLACKBODY_SIZE - 1);
    double rgb[3];
    blackbodyRGB(kelvin, rgb);
    double peak = std::max(rgb[0], std::max(rgb[1], rgb[2]));
    if (peak <= 0) {
      out4[i * 4 + 0] = out4[i * 4 + 1] = out4[i * 4 + 2] = 0.f;
      out4[i * 4 + 3] = -32.f;
      continue;
    }
    for (int ch = 0; ch < 3; ch++) out4[i * 4 + ch] = (float)(rgb[ch] / peak);
    out4[i * 4 + 3] = (float)std::max(-32.0, std::log2(peak / refPeak));
  }
}

namespace fp {

// TileDirectory.clusters (TileDirectory.ts:189-237): the tiles grouped by touch (faces, edges or
// corners), in creation order, each group boxed; boxes that overlap merge until none do, and
// the surviving boxes are numbered in the order of their first group.
void Engine::buildClusters() {
  const auto& slots = dir_.slots();
  std::vector<int> order;
  for (size_t s = 0; s < slots.size(); s++)
    if (slots[s].alive) order.push_back((int)s);
  std::sort(order.begin(), order.end(), [&](int a, int b) { return slots[a].seq < slots[b].seq; });
  std::vector<int> group(slots.size(), -1);
  std::vector<std::array<int, 6>> boxes;
  std::vector<int> stack;
  for (int first : order) {
    if (group[first] >= 0) continue;
    const int index = (int)boxes.size();
    const TileDirectory::Tile& f = slots[first];
    std::array<int, 6> box = {f.x, f.y, f.z, f.x, f.y, f.z};
    group[first] = index;
    stack.assign(1, first);
    while (!stack.empty()) {
      const TileDirectory::Tile& t = slots[stack.back()];
      stack.pop_back();
      const int c[3] = {t.x, t.y, t.z};
      for (int a = 0; a < 3; a++) {
        box[a] = std::min(box[a], c[a]);
        box[3 + a] = std::max(box[3 + a], c[a]);
      }
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            int n = dir_.slotAt(t.x + dx, t.y + dy, t.z + dz);
            if (n >= 0 && group[n] < 0) {
              group[n] = index;
              stack.push_back(n);
            }
          }
    }
    boxes.push_back(box);
  }
  std::vector<int> into(boxes.size());
  for (size_t i = 0; i < into.size(); i++) into[i] = (int)i;
  auto root = [&](int i) {
    while (into[i] != i) i = into[i] = into[into[i]];
    return i;
  };
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
  clusterBoxes_.clear();
  for (size_t i = 0; i < boxes.size(); i++)
    if (root((int)i) == (int)i) {
      renumbered[i] = (int)(clusterBoxes_.size() / 6);
      clusterBoxes_.insert(clusterBoxes_.end(), boxes[i].begin(), boxes[i].end());
    }
  clusterOf_.assign(slots.size(), -1);
  for (size_t s = 0; s < slots.size(); s++)
    if (group[s] >= 0) clusterOf_[s] = renumbered[root(group[s])];
}

// updateBoxes (FluidSimulation.ts:916-957): what the render draws in each cluster of tiles, the
// bricks with content at the latest measurement and the sources' bricks (each in the cluster of
// its centre's tile), grown by two bricks and kept within the cluster's tiles; clusters with none
// of these get no box. Boxes in cluster order.
void Engine::updateRenderBox() {
  const int TB = 4, MARGIN = 2;
  std::map<int, std::array<int, 6>> found;
  auto include = [&](const int* l, const int* u) {
    int c[3];
    for (int a = 0; a < 3; a++) c[a] = (int)std::floor(((double)l[a] + (double)u[a]) / 2.0);
    if (ground_) c[1] = std::max(0, c[1]);
    auto div = [](int n) { return (int)std::floor((double)n / 4.0); };
    int slot = dir_.slotAt(div(c[0]), div(c[1]), div(c[2]));
    if (slot < 0 || slot >= (int)clusterOf_.size() || clusterOf_[slot] < 0) return;
    auto it = found.find(clusterOf_[slot]);
    if (it == found.end()) {
      found[clusterOf_[slot]] = {l[0], l[1], l[2], u[0], u[1], u[2]};
      return;
    }
    for (int a = 0; a < 3; a++) {
      it->second[a] = std::min(it->second[a], l[a]);
      it->second[3 + a] = std::max(it->second[3 + a], u[a]);
    }
  };
  for (auto& ct : contentTiles_) {
    int t[3] = {ct.first.x, ct.first.y, ct.first.z}, l[3], u[3];
    bool ok = true;
    for (int a = 0; a < 3; a++) {
      uint32_t used = (ct.second >> (a * 4)) & 15u;
      if (!used) ok = false;
      if (!used) break;
      l[a] = t[a] * TB + __builtin_ctz(used);
      u[a] = t[a] * TB + (31 - __builtin_clz(used));
    }
    if (ok) include(l, u);
  }
  for (size_t s = 0; s + 6 <= sourceBoxes_.size(); s += 6) include(&sourceBoxes_[s], &sourceBoxes_[s + 3]);
  renderBoxes_.clear();
  for (auto& kv : found) {
    const int* tiles = &clusterBoxes_[(size_t)kv.first * 6];
    for (int a = 0; a < 3; a++) renderBoxes_.push_back(std::max(kv.second[a] - MARGIN, tiles[a] * TB));
    for (int a = 0; a < 3; a++) renderBoxes_.push_back(std::min(kv.second[3 + a] + MARGIN, (tiles[3 + a] + 1) * TB - 1));
  }
}

// The blackbody table and the parameters a render pass reads: the latest state and the
// directory (device, on the simulation's stream).
int Engine::renderInputs() {
  int rc;
  if (!lut_.ptr) {
    std::vector<float> table(FP_BLACKBODY_SIZE * 4);
    fp_blackbody_table(table.data());
    if (!alloc(lut_, table.size() * 4, false)) return FP_ENOMEM;
    if ((rc = check(cudaMemcpy(lut_.ptr, table.data(), table.size() * 4, cudaMemcpyHostToDevice), "render"))) return rc;
  }
  if (!renderParams_.ptr && !alloc(renderParams_, sizeof(SimParams), false)) return FP_ENOMEM;
  if (!renderParamsH_ && (rc = check(cudaMallocHost(&renderParamsH_, sizeof(SimParams)), "cudaMallocHost"))) return rc;
  // The parameters the render reads: the latest state and the directory.
  cudaStreamSynchronize(stream());  // the previous render's parameters were read
  SimParams& P = *renderParamsH_;
  std::memset(&P, 0, sizeof(P));
  P.B = B_;
  P.shift = shift_;
  P.N = N_;
  P.W = W_;
  P.h = h_;
  P.invH = 1.f / h_;
  P.capacity = capacity_;
  P.slots = slots_;
  P.bounds = (FpBounds*)bounds_.ptr;
  P.tileRec = (const int4*)tileRecD_.ptr;
  P.tileNbr = (const int*)tileNbrD_.ptr;
  P.hash = (const int4*)hashD_.ptr;
  P.hashMask = (uint32_t)hash_.size() - 1;
  P.entries = (int*)entries_.ptr;
  P.records = (int*)records_.ptr;
  P.active = (uint32_t*)active_.ptr;
  P.counters = (FpCounters*)counters_.ptr;
  P.fld = (float*)fld_[fldIdx_[0]].ptr;
  P.scalarHalf = precision_ == FP_PRECISION_MIXED ? 1 : 0;
  P.smokeDiv = smokeDiv_;  // the coarse smoke grid, when there is one
  P.smokeShift = sshift_;
  P.smokeCells = SN_;
  P.smk = (float*)smoke_[smokeIdx_[0]].ptr;
  P.velDiv = vd_;  // the field lattice's view only: the render reads no velocity
  P.solidSpan = 1;
  P.fshift = shift_;
  P.fineH = h_;
  P.fview = P.vview = (const SimParams*)renderParams_.ptr;
  if ((rc = check(cudaMemcpyAsync(renderParams_.ptr, &P, sizeof(P), cudaMemcpyHostToDevice, stream()), "render")))
    return rc;
  return FP_OK;
}

// The optical model's settings (fire-emission.wgsl's uniforms).
static void optics(FpRender& R, const fp_render_settings& rs) {
  std::memcpy(R.optical, rs.optical, sizeof(R.optical));
  std::memcpy(R.light, rs.light, sizeof(R.light));
  std::memcpy(R.smoke, rs.smoke, sizeof(R.smoke));
  std::memcpy(R.fire, rs.fire, sizeof(R.fire));
  std::memcpy(R.sceneLight, rs.scene_light, sizeof(R.sceneLight));
  std::memcpy(R.ambient, rs.ambient_light, sizeof(R.ambient));
  R.flameOpacity = rs.flame_opacity;
}

int Engine::render(const fp_camera& cam, const fp_render_settings& rs, float* image, float* host) {
  if (cam.width == 0 || cam.height == 0 || cam.width > 16384 || cam.height > 16384)
    return fail(FP_EINVAL, "render: width and height must be from 1 to 16384.");
  if (rs.lighting_divisor != 1 && rs.lighting_divisor != 2 && rs.lighting_divisor != 4)
    return fail(FP_EINVAL, "rendering.lightingDivisor must be 1, 2 or 4.");
  if (rs.ray_steps < 8 || rs.ray_steps > 1024) return fail(FP_EINVAL, "rendering.raySteps must be from 8 to 1024.");
  if (rs.shadow_samples < 1 || rs.shadow_samples > 256) return fail(FP_EINVAL, "shadow samples must be from 1 to 256.");
  if (rs.filter < 0 || rs.filter > 2) return fail(FP_EINVAL, "rendering.filter must be 0, 1 or 2.");
  if (cam.half_resolution > 1) return fail(FP_EINVAL, "render: half_resolution must be 0 or 1.");
  int rc = consume();
  if (rc) return rc;
  const int divShift = rs.lighting_divisor == 1 ? 0 : (rs.lighting_divisor == 2 ? 1 : 2);
  const int lightShift = shift_ - divShift, L = 1 << lightShift, blocks = (B_ / 8) * (B_ / 8) * (B_ / 8);
  size_t pixels = (size_t)cam.width * cam.height;
  // Pools sized for every slot; the table and the parameters once.
  bool ok = (renderField_.bytes >= (size_t)slots_ * 4 * N_ * 4 || grow(renderField_, (size_t)slots_ * 4 * N_ * 4, 0)) &&
            (lighting_.bytes >= (size_t)slots_ * 4 * L * L * L * 4 ||
             grow(lighting_, (size_t)slots_ * 4 * L * L * L * 4, 0)) &&
            (occupancy_.bytes >= (size_t)slots_ * blocks || grow(occupancy_, (size_t)slots_ * blocks, 0)) &&
            (smokeDiv_ == 1 || renderSmoke_.bytes >= (size_t)slots_ * SN_ * 4 ||
             grow(renderSmoke_, (size_t)slots_ * SN_ * 4, 0)) &&
            (renderParams_.ptr || alloc(renderParams_, sizeof(SimParams), false));
  if (!ok) return FP_ENOMEM;
  float* out = image;
  if (host) {
    if (image_.bytes < pixels * 16 && !alloc(image_, pixels * 16, false)) return FP_ENOMEM;
    out = (float*)image_.ptr;
  }
  if ((rc = renderInputs())) return rc;
  // The scene's depth and the half-resolution slices.
  const float* depth = nullptr;
  if (cam.scene_depth) {
    if (sceneDepth_.bytes < pixels * 4 && !alloc(sceneDepth_, pixels * 4, false)) return FP_ENOMEM;
    if ((rc = check(cudaMemcpyAsync(sceneDepth_.ptr, cam.scene_depth, pixels * 4, cudaMemcpyHostToDevice, stream()),
                    "render")))
      return rc;
    depth = (const float*)sceneDepth_.ptr;
  }
  const int sliceW = std::max(1, (int)((cam.width + 1) / 2)), sliceH = std::max(1, (int)((cam.height + 1) / 2));
  const size_t sliceBytes = (size_t)sliceW * sliceH * FP_SLICES * 16;
  if (cam.half_resolution && slices_.bytes < sliceBytes && !alloc(slices_, sliceBytes, false)) return FP_ENOMEM;
  FpRender R;
  std::memset(&R, 0, sizeof(R));
  std::memcpy(R.ivp, cam.inverse_view_projection, sizeof(R.ivp));
  R.width = (int)cam.width;
  R.height = (int)cam.height;
  R.time = cam.time;
  optics(R, rs);
  R.shadowSamples = (int)rs.shadow_samples;
  R.raySteps = (int)rs.ray_steps;
  R.filter = rs.filter;
  R.lightShift = lightShift;
  // The boxes of the latest step (none before the first).
  R.boxCount = steps_ > 0 ? (int)(renderBoxes_.size() / 6) : 0;
  if (R.boxCount > 0) {
    const size_t bytes = renderBoxes_.size() * 4;
    if (renderBoxesD_.bytes < bytes && !alloc(renderBoxesD_, std::max<size_t>(bytes, 64 * 24), false)) return FP_ENOMEM;
    if ((rc = check(cudaMemcpyAsync(renderBoxesD_.ptr, renderBoxes_.data(), bytes, cudaMemcpyHostToDevice, stream()),
                    "render")))
      return rc;
  }
  R.boxes = (const int*)renderBoxesD_.ptr;
  R.depth = depth;
  R.slices = cam.half_resolution ? (float*)slices_.ptr : nullptr;
  R.sliceW = sliceW;
  R.sliceH = sliceH;
  R.renderField = (float*)renderField_.ptr;
  R.renderSmoke = (float*)renderSmoke_.ptr;
  R.lighting = (float*)lighting_.ptr;
  R.occupancy = (uint8_t*)occupancy_.ptr;
  R.lut = (const float4*)lut_.ptr;
  R.image = out;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, owner_->device());
  fp_launch_render((const SimParams*)renderParams_.ptr, R, sms, stream());
  if ((rc = check(cudaGetLastError(), "render launch"))) return rc;
  if (host) {
    if ((rc = check(cudaMemcpyAsync(host, out, pixels * 16, cudaMemcpyDeviceToHost, stream()), "render"))) return rc;
    return check(cudaStreamSynchronize(stream()), "render");
  }
  return FP_OK;
}

int Engine::collectLights(const fp_render_settings& rs, const float* anchors, uint32_t count, float* sums) {
  if (count > 65536) return fail(FP_EINVAL, "scene lights: at most 65536 anchors.");
  int rc = consume();
  if (rc) return rc;
  if (count == 0) return FP_OK;
  if ((rc = renderInputs())) return rc;
  const size_t abytes = (size_t)count * 3 * 4, sbytes = (size_t)count * 8 * 4;
  if ((anchors_.bytes < abytes && !grow(anchors_, abytes, 0)) || (lightSums_.bytes < sbytes && !grow(lightSums_, sbytes, 0)))
    return FP_ENOMEM;
  if ((rc = check(cudaMemcpyAsync(anchors_.ptr, anchors, abytes, cudaMemcpyHostToDevice, stream()), "scene lights")) ||
      (rc = check(cudaMemsetAsync(lightSums_.ptr, 0, sbytes, stream()), "scene lights")))
    return rc;
  FpRender R;
  std::memset(&R, 0, sizeof(R));
  optics(R, rs);
  R.lut = (const float4*)lut_.ptr;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, owner_->device());
  fp_launch_collect_lights((const SimParams*)renderParams_.ptr, R, (const float*)anchors_.ptr, (int)count,
                           (float*)lightSums_.ptr, sms, stream());
  if ((rc = check(cudaGetLastError(), "scene lights launch"))) return rc;
  if ((rc = check(cudaMemcpyAsync(sums, lightSums_.ptr, sbytes, cudaMemcpyDeviceToHost, stream()), "scene lights")))
    return rc;
  return check(cudaStreamSynchronize(stream()), "scene lights");
}

}  // namespace fp
