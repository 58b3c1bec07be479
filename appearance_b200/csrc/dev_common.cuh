// Device-side vector algebra, packing formats and RNG of the frame.
//
// Arithmetic contract: the kernels are compiled with -fmad=false and IEEE
// division / square root, every vector expression is evaluated left to right
// as in the reference WGSL, and transcendental functions come from detmath.h.
// Under that contract a kernel's result is a deterministic function of its
// inputs, independent of thread scheduling.
#pragma once

#include <stdint.h>

#include "detmath.h"

namespace ap {

#define APD __device__ __forceinline__

APD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
APD float3 f3s(float s) { return make_float3(s, s, s); }
APD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
APD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
APD float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
APD float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
APD float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
APD float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
APD float3 operator/(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
APD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
APD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
APD float len(float3 a) { return dm::sqrt_(dot(a, a)); }
APD float3 normalize(float3 a) { return a / len(a); }
APD float dist(float3 a, float3 b) { return len(a - b); }
APD float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
APD float3 vabs(float3 a) { return f3(dm::fabs_(a.x), dm::fabs_(a.y), dm::fabs_(a.z)); }
APD float3 vmax(float3 a, float3 b) { return f3(dm::fmax(a.x, b.x), dm::fmax(a.y, b.y), dm::fmax(a.z, b.z)); }
APD float3 vsqrt(float3 a) { return f3(dm::sqrt_(a.x), dm::sqrt_(a.y), dm::sqrt_(a.z)); }
APD float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
APD float3 mix3(float3 a, float3 b, float t) { return a * (1.0f - t) + b * t; }
APD float3 reflect(float3 i, float3 n) { return i - (2.0f * dot(n, i)) * n; }
APD float luma(float3 c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }
APD float sqr(float x) { return x * x; }

// Exclusive prefix of `flag` over the block's threads in thread order, and
// the block's total.  Every thread of the block calls it, once per kernel
// (blockDim.x a multiple of 32, at most 1024).
APD uint32_t block_prefix(bool flag, uint32_t* total) {
  __shared__ uint32_t s_warp[32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) s_warp[warp] = (uint32_t)__popc(b);
  __syncthreads();
  uint32_t off = 0, tot = 0;
  for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) {
    const uint32_t c = s_warp[w];
    off += w < warp ? c : 0u;
    tot += c;
  }
  *total = tot;
  return off + (uint32_t)__popc(b & ((1u << lane) - 1u));
}

// Column-major 3x3: columns c0, c1, c2.
struct Mat3 {
  float3 c0, c1, c2;
};
APD float3 mul(const Mat3& m, float3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
APD float3 mul_t(const Mat3& m, float3 v) { return f3(dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)); }

// Orthonormal basis around n (Duff et al., JCGT 6(1) 2017), columns (t1, t2, n).
APD Mat3 onb(float3 n) {
  float3 t1, t2;
  if (n.z < 0.0f) {
    float a = 1.0f / (1.0f - n.z);
    float b = n.x * n.y * a;
    t1 = f3(1.0f - n.x * n.x * a, -b, n.x);
    t2 = f3(b, n.y * n.y * a - 1.0f, -n.y);
  } else {
    float a = 1.0f / (1.0f + n.z);
    float b = -n.x * n.y * a;
    t1 = f3(1.0f - n.x * n.x * a, b, -n.x);
    t2 = f3(b, 1.0f - n.y * n.y * a, -n.y);
  }
  Mat3 m;
  m.c0 = t1;
  m.c1 = t2;
  m.c2 = n;
  return m;
}

// ---- PCG hash stream (Jarzynski & Olano, JCGT 9(3) 2020), as random.wgsl ----
APD uint32_t pcg_hash(uint32_t x) {
  uint32_t state = x * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
APD float rnd(uint32_t& s) {
  s = pcg_hash(s);
  return __uint2float_rn(s) / 4294967296.0f;
}
APD uint32_t xor_shift(uint32_t st) {
  uint32_t s = st ^ (st << 13);
  s ^= s >> 17;
  s ^= s << 5;
  return s;
}
APD uint32_t hash_combine(uint32_t x, uint32_t y) {
  uint32_t seed = (x * 1664525u + y + 1013904223u) * 1664525u;
  seed ^= (seed >> 11u);
  seed ^= (seed << 7u) & 0x9d2c5680u;
  seed ^= (seed << 15u) & 0xefc60000u;
  seed ^= (seed >> 18u);
  return seed;
}

// ---- shared-exponent RGB (9:9:9:5) and 2x15-bit octahedral unit vectors ----
APD uint32_t pack_rgb9e5(float3 rgb) {
  const float max_val = __uint_as_float(0x477F8000u);
  const float min_val = __uint_as_float(0x37800000u);
  float r = dm::clamp(rgb.x, 0.0f, max_val), g = dm::clamp(rgb.y, 0.0f, max_val),
        b = dm::clamp(rgb.z, 0.0f, max_val);
  float mc = dm::fmax(dm::fmax(min_val, r), dm::fmax(g, b));
  float bias = __uint_as_float((__float_as_uint(mc) + 0x07804000u) & 0x7F800000u);
  uint32_t ri = __float_as_uint(r + bias), gi = __float_as_uint(g + bias), bi = __float_as_uint(b + bias);
  uint32_t e = (__float_as_uint(bias) << 4u) + 0x10000000u;
  return e | (bi << 18) | (gi << 9) | (ri & 0x1FFu);
}
APD float3 unpack_rgb9e5(uint32_t d) {
  float sc = __uint_as_float((uint32_t)((int)(d >> 27) - 24 + 127) << 23);
  return f3(__uint2float_rn(d & 0x1FFu) * sc, __uint2float_rn((d >> 9) & 0x1FFu) * sc,
            __uint2float_rn((d >> 18) & 0x1FFu) * sc);
}
APD uint32_t pack_oct30(float3 dir) {
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
  return (dm::f2u(rintf(ry * 32767.0f)) << 15) | dm::f2u(rintf(rx * 32767.0f));
}
APD float3 unpack_oct30(uint32_t p) {
  float ex = __uint2float_rn(p & 0x7fffu) / 32767.0f;
  float ey = __uint2float_rn((p >> 15) & 0x7fffu) / 32767.0f;
  ex = ex * 2.0f - 1.0f;
  ey = ey * 2.0f - 1.0f;
  float3 n = f3(ex, ey, 1.0f - dm::fabs_(ex) - dm::fabs_(ey));
  float t = dm::saturate(-n.z);
  n.x = n.x + (n.x >= 0.0f ? -t : t);
  n.y = n.y + (n.y >= 0.0f ? -t : t);
  return normalize(n);
}

}  // namespace ap
