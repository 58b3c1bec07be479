// Deterministic binary32 elementary functions shared by the CUDA kernels and
// the CPU oracle.
//
// Every function is a fixed sequence of IEEE-754 round-to-nearest multiplies,
// adds, divides and square roots (no fused multiply-add, no hardware
// approximations), so a host build with -ffp-contract=off and a device build
// with -fmad=false return identical bits for identical inputs.  The method is
// Cody-Waite argument reduction followed by a polynomial on the reduced range
// (W. J. Cody, W. Waite, "Software Manual for the Elementary Functions",
// Prentice-Hall 1980).  The coefficients are least-squares fits made by
// gen_detmath.py next to this file; accuracy is a few ulp on the ranges the
// frame uses (tests/test_detmath.py checks it against float64 references).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define DM_HD __host__ __device__ __forceinline__
#else
#define DM_HD inline
#include <math.h>
#include <string.h>
#endif

namespace dm {

DM_HD uint32_t f2bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}

DM_HD float bits2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

constexpr float PI = 3.14159265358979323846f;
constexpr float TWO_PI = 6.28318530717958647692f;
constexpr float HALF_PI = 1.57079632679489661923f;
constexpr float INV_PI = 0.318309886183790671538f;
constexpr float F32_MAX = 3.40282347e+38f;

// min/max/clamp with one fixed rule on every platform: a NaN operand yields
// the other operand, and ties (including -0 vs +0) return the first operand.
DM_HD float fmin(float a, float b) { return (b < a || a != a) ? b : a; }
DM_HD float fmax(float a, float b) { return (b > a || a != a) ? b : a; }
DM_HD float clamp(float x, float lo, float hi) { return fmin(fmax(x, lo), hi); }
DM_HD float saturate(float x) { return clamp(x, 0.0f, 1.0f); }
DM_HD float sqr(float x) { return x * x; }

DM_HD float fabs_(float x) { return bits2f(f2bits(x) & 0x7fffffffu); }

DM_HD float floor_(float x) { return floorf(x); }
DM_HD float ceil_(float x) { return ceilf(x); }
// Round half to even (the default IEEE rounding mode on both targets).
DM_HD float rint_(float x) { return rintf(x); }
DM_HD float fract(float x) { return x - floor_(x); }
DM_HD float sqrt_(float x) { return sqrtf(x); }

// float -> u32, truncating; NaN and negatives give 0, overflow saturates.
DM_HD uint32_t f2u(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)x;
}
// float -> i32, truncating; NaN gives 0, overflow saturates.
DM_HD int32_t f2i(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int32_t)x;
}

// x * 2^n for integer n in [-252, 254] without overflow of the scale factor.
DM_HD float ldexp_(float x, int n) {
  while (n > 127) { x = x * 1.70141183e+38f; n -= 127; }
  while (n < -126) { x = x * 1.17549435e-38f; n += 126; }
  return x * bits2f((uint32_t)(n + 127) << 23);
}

// ---- sin / cos -------------------------------------------------------------
// Reduction by pi/2 split in three parts (the first with few mantissa bits so
// k * PIO2_1 is exact for |k| < 2^13), then odd/even polynomials on |r|<=pi/4.
DM_HD void sincos_(float x, float* s, float* c) {
  const float PIO2_1 = 1.570312500e+00f;
  const float PIO2_2 = 4.837512970e-04f;
  const float PIO2_3 = 7.549790126e-08f;
  const float TWO_OVER_PI = 0.636619772367581343076f;
  if (x != x || fabs_(x) == bits2f(0x7f800000u)) {
    *s = x - x;
    *c = x - x;
    return;
  }
  float k = rint_(x * TWO_OVER_PI);
  float r = x - k * PIO2_1;
  r = r - k * PIO2_2;
  r = r - k * PIO2_3;
  float z = r * r;
  float ps = -1.984017581e-04f + z * 2.725872264e-06f;
  ps = 8.333331905e-03f + z * ps;
  ps = -1.666666716e-01f + z * ps;
  float sr = r + (r * z) * ps;
  float pc = 2.480067451e-05f + z * -2.730829465e-07f;
  pc = -1.388888806e-03f + z * pc;
  pc = 4.166666791e-02f + z * pc;
  float cr = (1.0f - 0.5f * z) + (z * z) * pc;
  int q = (int)f2i(k) & 3;
  float so, co;
  if (q == 0) { so = sr; co = cr; }
  else if (q == 1) { so = cr; co = -sr; }
  else if (q == 2) { so = -sr; co = -cr; }
  else { so = -cr; co = sr; }
  *s = so;
  *c = co;
}
DM_HD float sin_(float x) { float s, c; sincos_(x, &s, &c); return s; }
DM_HD float cos_(float x) { float s, c; sincos_(x, &s, &c); return c; }

// ---- exp -------------------------------------------------------------------
DM_HD float exp_(float x) {
  if (x != x) return x;
  if (x > 88.7228317f) return bits2f(0x7f800000u);
  if (x < -103.972084f) return 0.0f;
  const float LOG2E = 1.44269504088896340736f;
  const float LN2_1 = 6.933593750e-01f;
  const float LN2_2 = -2.121944417e-04f;
  float k = rint_(x * LOG2E);
  float r = x - k * LN2_1;
  r = r - k * LN2_2;
  float p = 1.393319690e-03f + r * 1.975042542e-04f;
  p = 8.333520964e-03f + r * p;
  p = 4.166647047e-02f + r * p;
  p = 1.666666567e-01f + r * p;
  p = 5.000000000e-01f + r * p;
  float e = 1.0f + (r + (r * r) * p);
  return ldexp_(e, (int)f2i(k));
}

// ---- log -------------------------------------------------------------------
DM_HD float log_(float x) {
  if (x != x) return x;
  if (x < 0.0f) return bits2f(0x7fc00000u);
  if (x == 0.0f) return -bits2f(0x7f800000u);
  if (x == bits2f(0x7f800000u)) return x;
  int e = 0;
  if (x < 1.17549435e-38f) { x = x * 8388608.0f; e = -23; }
  uint32_t u = f2bits(x);
  e += (int)((u >> 23) & 0xff) - 127;
  float m = bits2f((u & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = 2.855234146e-01f + z * 2.329930216e-01f;
  p = 4.000010192e-01f + z * p;
  p = 6.666666865e-01f + z * p;
  float lm = (s + s) + (s * z) * p;
  float fe = (float)e;
  const float LN2_1 = 6.933593750e-01f;
  const float LN2_2 = -2.121944417e-04f;
  return fe * LN2_1 + (fe * LN2_2 + lm);
}

// pow for the cases the frame needs: x >= 0 (WGSL leaves x < 0 undefined; it
// returns NaN here).
DM_HD float pow_(float x, float y) {
  if (x != x || y != y) return x + y;
  if (x < 0.0f) return bits2f(0x7fc00000u);
  if (y == 0.0f) return 1.0f;
  if (x == 0.0f) return y > 0.0f ? 0.0f : bits2f(0x7f800000u);
  if (x == 1.0f) return 1.0f;
  return exp_(y * log_(x));
}

// x^128 for x >= 0 as seven squarings: the a-trous normal weight's exponent
// (PHI_NORMAL = 128, svgf_atrous.wgsl) is a power of two.
DM_HD float pow128(float x) {
  x = x * x;
  x = x * x;
  x = x * x;
  x = x * x;
  x = x * x;
  x = x * x;
  return x * x;
}

// ---- atan2 -----------------------------------------------------------------
DM_HD float atan_unit(float t) {  // t in [0, 1]
  const float TAN_PI_8 = 0.414213562373095048802f;
  float base = 0.0f;
  if (t > TAN_PI_8) {
    t = (t - 1.0f) / (t + 1.0f);
    base = 0.785398163397448309616f;
  }
  float z = t * t;
  float p = -8.644333482e-02f + z * 5.091862008e-02f;
  p = 1.107451767e-01f + z * p;
  p = -1.428436488e-01f + z * p;
  p = 1.999998242e-01f + z * p;
  p = -3.333333433e-01f + z * p;
  return base + (t + (t * z) * p);
}

DM_HD float atan2_(float y, float x) {
  if (x != x || y != y) return x + y;
  float ax = fabs_(x), ay = fabs_(y);
  bool ysign = (f2bits(y) >> 31) != 0;
  bool xsign = (f2bits(x) >> 31) != 0;
  float a;
  if (ax == 0.0f && ay == 0.0f) {
    a = xsign ? PI : 0.0f;
  } else if (ay <= ax) {
    a = atan_unit(ay / ax);
    if (xsign) a = PI - a;
  } else {
    a = HALF_PI - atan_unit(ax / ay);
    if (xsign) a = PI - a;
  }
  return ysign ? -a : a;
}

// ---- acos ------------------------------------------------------------------
DM_HD float asin_poly(float t) {  // t in [0, 0.5]
  float z = t * t;
  float p = 1.733718626e-02f + z * 3.341230750e-02f;
  p = 3.105505556e-02f + z * p;
  p = 4.460413754e-02f + z * p;
  p = 7.500075549e-02f + z * p;
  p = 1.666666716e-01f + z * p;
  return t + (t * z) * p;
}

DM_HD float acos_(float x) {
  if (x != x) return x;
  if (x > 1.0f || x < -1.0f) return bits2f(0x7fc00000u);
  if (fabs_(x) <= 0.5f) return HALF_PI - asin_poly(x < 0.0f ? -x : x) * (x < 0.0f ? -1.0f : 1.0f);
  if (x > 0.0f) {
    float s = sqrt_((1.0f - x) * 0.5f);
    return 2.0f * asin_poly(s);
  }
  float s = sqrt_((1.0f + x) * 0.5f);
  return PI - 2.0f * asin_poly(s);
}

}  // namespace dm
