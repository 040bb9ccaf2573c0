// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// Shared helpers of the CPU oracle: small vector types, precision rounding that restates
// the reference's half-precision storage, and the noise functions. Only tests/, bench.py's
// CPU-baseline leg and __graft_entry__.smoke() may load the oracle.
//
// Parity unpinned: the reference (TypeScript + WGSL) ships no tests, no golden vectors and
// no CPU path, and cannot run here, so this restatement is pinned only by reading.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

template <class R>
struct V3 {
  R v[3];
  R& operator[](int i) { return v[i]; }
  const R& operator[](int i) const { return v[i]; }
};
struct I3 {
  int v[3];
  int& operator[](int i) { return v[i]; }
  const int& operator[](int i) const { return v[i]; }
  bool operator==(const I3& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};

template <class R> inline V3<R> v3(R a, R b, R c) { return V3<R>{{a, b, c}}; }
inline I3 i3(int a, int b, int c) { return I3{{a, b, c}}; }

// Storage precision of one pool class.
enum Store { STORE_EXACT = 0, STORE_F16 = 1, STORE_BF16 = 2 };

// Round-to-nearest-even to IEEE binary16, returned as a double (WGSL `f16(x)`, an
// rgba16float/r16float store). Overflow saturates to infinity like a hardware store.
inline double round_f16(double x) {
  if (!std::isfinite(x) || x == 0.0) return x;
  double a = std::fabs(x);
  if (a >= 65520.0) return std::copysign(INFINITY, x);
  int e;
  std::frexp(a, &e);               // a = m * 2^e, m in [0.5, 1)
  int exp2 = e - 1;                // a in [2^exp2, 2^(exp2+1))
  if (exp2 < -14) exp2 = -14;      // subnormal spacing 2^-24
  double ulp = std::ldexp(1.0, exp2 - 10);
  double q = a / ulp;              // exact: power-of-two scaling
  double r = std::nearbyint(q);    // ties to even (default rounding mode)
  return std::copysign(r * ulp, x);
}

// Round-to-nearest-even to bfloat16 (8 mantissa bits), from the float value.
inline double round_bf16(double xd) {
  float x = (float)xd;
  if (!std::isfinite(x)) return x;
  uint32_t u;
  std::memcpy(&u, &x, 4);
  uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  u &= 0xffff0000u;
  float y;
  std::memcpy(&y, &u, 4);
  return y;
}

template <class R>
inline R store_round(R x, int mode) {
  if (mode == STORE_F16) return (R)round_f16((double)x);
  if (mode == STORE_BF16) return (R)round_bf16((double)x);
  return x;
}

// `truncateHalf` (src/engine/shaders/fluid-common.wgsl:109-114): round toward zero to half
// precision, as Apple GPUs store half floats. Applied only in the reference's half mode.
inline double truncate_half(double xd) {
  float x = (float)xd;
  if (std::fabs(x) < 6.103515625e-5f) {
    return std::trunc(x * 16777216.0f) / 16777216.0f;
  }
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u &= 0xffffe000u;
  float y;
  std::memcpy(&y, &u, 4);
  return y;
}

template <class R> inline R mixr(R a, R b, R t) { return a * (R(1) - t) + b * t; }
template <class R> inline R clampr(R x, R lo, R hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class R> inline R smoothstep(R e0, R e1, R x) {
  R t = clampr((x - e0) / (e1 - e0), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
template <class R> inline R fractr(R x) { return x - std::floor(x); }
inline int floori(double x) { return (int)std::floor(x); }

// `hash` (src/engine/shaders/curl-noise.wgsl:1-11): the lattice hash of the curl noise.
inline double noise_hash(int px, int py, int pz) {
  uint32_t v[3] = {((uint32_t)px & 15u) * 1664525u + 1013904223u,
                   ((uint32_t)py & 15u) * 1664525u + 1013904223u,
                   ((uint32_t)pz & 15u) * 1664525u + 1013904223u};
  v[0] += v[1] * v[2];
  v[1] += v[2] * v[0];
  v[2] += v[0] * v[1];
  for (int i = 0; i < 3; i++) v[i] ^= v[i] >> 16u;
  v[0] += v[1] * v[2];
  v[1] += v[2] * v[0];
  v[2] += v[0] * v[1];
  return (double)(float)(v[0] >> 8u) / 16777216.0;
}

// `noiseGradient` (curl-noise.wgsl:13-31) in the caller's real type.
template <class R>
inline V3<R> noise_gradient(V3<R> p) {
  int i[3];
  R f[3], s[3], ds[3];
  for (int a = 0; a < 3; a++) {
    i[a] = (int)std::floor(p[a]);
    f[a] = p[a] - std::floor(p[a]);
    s[a] = f[a] * f[a] * f[a] * (f[a] * (f[a] * R(6) - R(15)) + R(10));
    ds[a] = R(30) * f[a] * f[a] * (f[a] - R(1)) * (f[a] - R(1));
  }
  R a = (R)noise_hash(i[0], i[1], i[2]);
  R b = (R)noise_hash(i[0] + 1, i[1], i[2]);
  R c = (R)noise_hash(i[0], i[1] + 1, i[2]);
  R d = (R)noise_hash(i[0] + 1, i[1] + 1, i[2]);
  R e = (R)noise_hash(i[0], i[1], i[2] + 1);
  R f1 = (R)noise_hash(i[0] + 1, i[1], i[2] + 1);
  R g = (R)noise_hash(i[0], i[1] + 1, i[2] + 1);
  R h = (R)noise_hash(i[0] + 1, i[1] + 1, i[2] + 1);
  V3<R> r;
  r[0] = mixr(mixr(b - a, d - c, s[1]), mixr(f1 - e, h - g, s[1]), s[2]) * ds[0];
  r[1] = mixr(mixr(c - a, d - b, s[0]), mixr(g - e, h - f1, s[0]), s[2]) * ds[1];
  r[2] = mixr(mixr(e - a, f1 - b, s[0]), mixr(g - c, h - d, s[0]), s[1]) * ds[2];
  return r;
}

// `burstGradient` (src/engine/shaders/fluid-sources.wgsl:41-49).
template <class R>
inline R burst_gradient(int cx, int cy, int cz, R ox, R oy, R oz, uint32_t seedBits) {
  uint32_t h = (uint32_t)cx * 374761393u + (uint32_t)cy * 668265263u + (uint32_t)cz * 2246822519u +
               seedBits * 3266489917u;
  h = (h ^ (h >> 13u)) * 1274126177u;
  h = (h ^ (h >> 16u)) & 15u;
  R a = h < 8u ? ox : oy;
  R b = h < 4u ? oy : ((h == 12u || h == 14u) ? ox : oz);
  return ((h & 1u) == 0u ? a : -a) + ((h & 2u) == 0u ? b : -b);
}

// `burstPerlin` (fluid-sources.wgsl:51-66).
template <class R>
inline R burst_perlin(V3<R> p, uint32_t seedBits) {
  int c[3];
  R f[3], s[3];
  for (int a = 0; a < 3; a++) {
    c[a] = (int)std::floor(p[a]);
    f[a] = p[a] - std::floor(p[a]);
    s[a] = f[a] * f[a] * f[a] * (f[a] * (f[a] * R(6) - R(15)) + R(10));
  }
  auto g = [&](int dx, int dy, int dz) {
    return burst_gradient<R>(c[0] + dx, c[1] + dy, c[2] + dz, f[0] - dx, f[1] - dy, f[2] - dz, seedBits);
  };
  R a = g(0, 0, 0), b = g(1, 0, 0), cc = g(0, 1, 0), d = g(1, 1, 0);
  R e = g(0, 0, 1), gg = g(1, 0, 1), h = g(0, 1, 1), j = g(1, 1, 1);
  return mixr(mixr(mixr(a, b, s[0]), mixr(cc, d, s[0]), s[1]), mixr(mixr(e, gg, s[0]), mixr(h, j, s[0]), s[1]),
              s[2]);
}

// `burstPattern` (fluid-sources.wgsl:68-71).
template <class R>
inline R burst_pattern(V3<R> p, uint32_t seedBits) {
  V3<R> q = v3<R>(p[0] * R(2) + R(5.2), p[1] * R(2) + R(9.7), p[2] * R(2) + R(3.1));
  R n = (burst_perlin(p, seedBits) + R(0.35) * burst_perlin(q, seedBits)) / R(1.35);
  return clampr(R(0.5) + R(0.5) * n, R(0), R(1));
}

}  // namespace orc
