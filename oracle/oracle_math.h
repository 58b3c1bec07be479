// Oracle (test infrastructure only): scalar CPU restatement of the reference
// frame's shader arithmetic.  Nothing in the product links this code; tests,
// the smoke check and the CPU-baseline leg of bench.py load it as the checker.
//
// Arithmetic contract (shared with the CUDA kernels, which restate the same
// expressions independently): binary32 IEEE round-to-nearest, no contraction
// (built with -ffp-contract=off), expressions evaluated left to right exactly
// as written in the WGSL, elementary functions from detmath.h.
#pragma once

#include <stdint.h>

#include "../appearance_b200/csrc/detmath.h"

namespace orc {

using dm::sqr;

struct V2 { float x, y; };
struct V3 { float x, y, z; };

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 v3s(float s) { return V3{s, s, s}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(V3 a) { return dm::sqrt_(dot(a, a)); }
inline V3 normalize(V3 a) { return a / length(a); }
inline float distance(V3 a, V3 b) { return length(a - b); }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 vabs(V3 a) { return {dm::fabs_(a.x), dm::fabs_(a.y), dm::fabs_(a.z)}; }
inline V3 vmax(V3 a, V3 b) { return {dm::fmax(a.x, b.x), dm::fmax(a.y, b.y), dm::fmax(a.z, b.z)}; }
inline V3 vmin(V3 a, V3 b) { return {dm::fmin(a.x, b.x), dm::fmin(a.y, b.y), dm::fmin(a.z, b.z)}; }
inline V3 vsqrt(V3 a) { return {dm::sqrt_(a.x), dm::sqrt_(a.y), dm::sqrt_(a.z)}; }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V3 mix3(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
// reflect(e1, e2) = e1 - 2 * dot(e2, e1) * e2
inline V3 reflect(V3 i, V3 n) { return i - (2.0f * dot(n, i)) * n; }
inline float luma(V3 c) { return dot(c, v3(0.2126f, 0.7152f, 0.0722f)); }

// Column-major 3x3 (columns c0, c1, c2), as WGSL mat3x3.
struct M3 { V3 c0, c1, c2; };
inline V3 mul(const M3& m, V3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
inline V3 mul_t(const M3& m, V3 v) { return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }
inline M3 zero_m3() { return M3{v3s(0), v3s(0), v3s(0)}; }

// jcgt 2017 "Building an Orthonormal Basis, Revisited" (math.wgsl:71-86).
inline M3 onb(V3 n) {
  V3 t1, t2;
  if (n.z < 0.0f) {
    float a = 1.0f / (1.0f - n.z);
    float b = n.x * n.y * a;
    t1 = v3(1.0f - n.x * n.x * a, -b, n.x);
    t2 = v3(b, n.y * n.y * a - 1.0f, -n.y);
  } else {
    float a = 1.0f / (1.0f + n.z);
    float b = -n.x * n.y * a;
    t1 = v3(1.0f - n.x * n.x * a, b, -n.x);
    t2 = v3(b, 1.0f - n.y * n.y * a, -n.y);
  }
  return M3{t1, t2, n};
}

// ---- random.wgsl:10-68 ----
inline uint32_t pcg_hash(uint32_t x) {
  uint32_t state = x * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
inline float rnd(uint32_t& s) {
  s = pcg_hash(s);
  return (float)s / 4294967296.0f;  // f32(0xFFFFFFFF) rounds to 2^32
}
inline uint32_t xor_shift(uint32_t st) {
  uint32_t s = st ^ (st << 13);
  s ^= s >> 17;
  s ^= s << 5;
  return s;
}
inline uint32_t hash_combine(uint32_t x, uint32_t y) {
  const uint32_t M = 1664525u, C = 1013904223u;
  uint32_t seed = (x * M + y + C) * M;
  seed ^= (seed >> 11u);
  seed ^= (seed << 7u) & 0x9d2c5680u;
  seed ^= (seed << 15u) & 0xefc60000u;
  seed ^= (seed >> 18u);
  return seed;
}

// ---- packing.wgsl:12-76 ----
inline uint32_t rgb9e5_pack(V3 rgb) {
  const float max_val = dm::bits2f(0x477F8000u);
  const float min_val = dm::bits2f(0x37800000u);
  V3 c = v3(dm::clamp(rgb.x, 0.0f, max_val), dm::clamp(rgb.y, 0.0f, max_val),
            dm::clamp(rgb.z, 0.0f, max_val));
  float max_channel = dm::fmax(dm::fmax(min_val, c.x), dm::fmax(c.y, c.z));
  float bias = dm::bits2f((dm::f2bits(max_channel) + 0x07804000u) & 0x7F800000u);
  uint32_t r = dm::f2bits(c.x + bias), g = dm::f2bits(c.y + bias), b = dm::f2bits(c.z + bias);
  uint32_t e = (dm::f2bits(bias) << 4u) + 0x10000000u;
  return e | (b << 18) | (g << 9) | (r & 0x1FFu);
}
inline V3 rgb9e5_unpack(uint32_t d) {
  float sc = dm::ldexp_(1.0f, (int)(d >> 27) - 24);
  return v3((float)(d & 0x1FFu) * sc, (float)((d >> 9) & 0x1FFu) * sc, (float)((d >> 18) & 0x1FFu) * sc);
}
inline uint32_t oct30_pack(V3 dir) {
  float den = dm::fabs_(dir.x) + dm::fabs_(dir.y) + dm::fabs_(dir.z);
  float rx = dir.x / den, ry = dir.y / den;
  if (dir.z < 0.0f) {
    float sx = rx >= 0.0f ? 1.0f : -1.0f;
    float sy = ry >= 0.0f ? 1.0f : -1.0f;
    float nx = (1.0f - dm::fabs_(ry)) * sx;
    float ny = (1.0f - dm::fabs_(rx)) * sy;
    rx = nx;
    ry = ny;
  }
  rx = rx * 0.5f + 0.5f;
  ry = ry * 0.5f + 0.5f;
  return (dm::f2u(dm::rint_(ry * 32767.0f)) << 15) | dm::f2u(dm::rint_(rx * 32767.0f));
}
inline V3 oct30_unpack(uint32_t p) {
  float ex = (float)(p & 0x7fffu) / 32767.0f;
  float ey = (float)((p >> 15) & 0x7fffu) / 32767.0f;
  ex = ex * 2.0f - 1.0f;
  ey = ey * 2.0f - 1.0f;
  V3 n = v3(ex, ey, 1.0f - dm::fabs_(ex) - dm::fabs_(ey));
  float t = dm::saturate(-n.z);
  n.x = n.x + (n.x >= 0.0f ? -t : t);
  n.y = n.y + (n.y >= 0.0f ? -t : t);
  return normalize(n);
}

}  // namespace orc
