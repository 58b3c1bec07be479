// Software ray traversal of the compressed 8-wide BVH (scene_layout.h) and the
// watertight ray/triangle test, for sm_100a (no RT cores).
//
// Node layout and quantisation follow the compressed-wide-BVH idea of
// H. Ylitie, T. Karras, S. Laine, "Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs", HPG 2017: one 80-byte node holds 8 child
// boxes quantised to 8 bits per plane relative to a per-node origin and
// power-of-two scale, read with five 128-bit loads.  Traversal is nearest-child-
// first with the other hit children pushed with their entry distance and
// culled on pop.  The triangle test is Woop/Benthin/Wald (JCGT 2013) in the same
// operation order as the CPU oracle, so closest-hit results are bit-identical:
// the closest hit is the minimum of (t, global triangle id) over all triangles
// that pass the test, which no traversal order can change.
#pragma once

#include "dev_common.cuh"
#include "scene_layout.h"

namespace ap {

constexpr int kTraversalStack = 96;
constexpr uint32_t kNoHit = 0xFFFFFFFFu;

struct Hit {
  float t, u, v;
  uint32_t tri;  // global triangle id or kNoHit
};

struct RayPre {
  float3 o, d;
  int kx, ky, kz;
  float sx, sy, sz;
  float3 inv;          // box-test reciprocal direction (0 where the component is 0)
  uint32_t zero_axes;  // bit k < 3: direction component k is +-0; bit 3: some component is below 2^-64
  uint32_t neg_axes;   // bit k: direction component k is negative (the far plane is entered first)
};

APD float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

APD RayPre ray_pre(float3 o, float3 d) {
  RayPre r;
  r.o = o;
  r.d = d;
  float ax = dm::fabs_(d.x), ay = dm::fabs_(d.y), az = dm::fabs_(d.z);
  int kz = 0;
  float m = ax;
  if (ay > m) { kz = 1; m = ay; }
  if (az > m) { kz = 2; }
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  if (comp(d, kz) < 0.0f) { int t = kx; kx = ky; ky = t; }
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  float dz = comp(d, kz);
  r.sx = comp(d, kx) / dz;
  r.sy = comp(d, ky) / dz;
  r.sz = 1.0f / dz;
  r.zero_axes = (d.x == 0.0f ? 1u : 0u) | (d.y == 0.0f ? 2u : 0u) | (d.z == 0.0f ? 4u : 0u);
  // bit 3: a component below 2^-64 in magnitude (zero included), for which
  // the box test takes its exact form
  const float kTiny = 5.42101086e-20f;  // 2^-64
  if (!(ax >= kTiny && ay >= kTiny && az >= kTiny)) r.zero_axes |= 8u;
  r.inv = f3(d.x == 0.0f ? 0.0f : 1.0f / d.x, d.y == 0.0f ? 0.0f : 1.0f / d.y, d.z == 0.0f ? 0.0f : 1.0f / d.z);
  r.neg_axes = (r.inv.x < 0.0f ? 1u : 0u) | (r.inv.y < 0.0f ? 2u : 0u) | (r.inv.z < 0.0f ? 4u : 0u);
  return r;
}

// Watertight inside test and barycentrics in binary32 (Woop, Benthin, Wald,
// JCGT 2013), distance t in double from the original vertices; same
// expressions as the oracle (intersect_tri).
APD bool intersect_tri(const RayPre& r, float3 v0, float3 v1, float3 v2, float tmin, float tmax,
                       float& t, float& u, float& v) {
  float3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
  float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
  float Ax = comp(A, r.kx) - r.sx * Akz, Ay = comp(A, r.ky) - r.sy * Akz;
  float Bx = comp(B, r.kx) - r.sx * Bkz, By = comp(B, r.ky) - r.sy * Bkz;
  float Cx = comp(C, r.kx) - r.sx * Ckz, Cy = comp(C, r.ky) - r.sy * Ckz;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = U + V + W;
  if (det == 0.0f) return false;
  // distance along the ray in double precision from the original vertices, only
  // for candidates that passed the inside test (one or two per ray)
  double e1x = (double)v1.x - v0.x, e1y = (double)v1.y - v0.y, e1z = (double)v1.z - v0.z;
  double e2x = (double)v2.x - v0.x, e2y = (double)v2.y - v0.y, e2z = (double)v2.z - v0.z;
  double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
  double wx = (double)v0.x - r.o.x, wy = (double)v0.y - r.o.y, wz = (double)v0.z - r.o.z;
  double td = (nx * wx + ny * wy + nz * wz) / (nx * r.d.x + ny * r.d.y + nz * r.d.z);
  if (!(td >= (double)tmin)) return false;
  float tt = (float)td;
  if (!(tt <= tmax)) return false;
  float rcp = 1.0f / det;
  t = tt;
  u = V * rcp;
  v = W * rcp;
  return true;
}

// Child boxes of one node: conservativeness.
//
// A slab value is computed as fma(q, s/d, (p - o)/d) with the power-of-two
// scale s exact.  Its error is at most 3 ulp of |(p - o)/d| (the rounding of
// p - o, of the product and of the fma, which can cancel against q*s/d) plus a
// relative error of 1/d itself.  The watertight inside test may accept a hit
// point outside the exact triangle by a few ulp of the vertex distances from
// the origin.  Each slab is therefore widened by 2^-19 of (|p - o| + node
// extent)/|d| and each interval by a relative 2^-21, so no child that holds a
// triangle accepted inside [tmin, tmax] is culled.  The widening e is folded
// into the per-node offsets once, fma(q, s/d, b - e) and fma(q, s/d, b + e)
// with b = (p - o)/d: the one extra rounding (of b -+ e) is half an ulp of
// |b| + e, far inside the 2^-19 margin, which is 16 ulp of |b| alone.  For a
// zero direction component the slab is all of t when the origin lies inside
// the child's bounds decoded as p + q*s (rounded to nearest, which never
// shrinks the conservatively quantised box), and empty otherwise.
//
// Two forms of that test.  The exact form (NodeFrame, child_entry) decodes
// each plane byte as the float q.  The fast form (NodeFrameQ,
// child_entry_q), taken by rays whose direction components are all at least
// 2^-64 in magnitude (ray_pre sets bit 3 of zero_axes otherwise), decodes it
// with one byte permute as Q = 1 + q 2^-15 (q under the exponent of 1.0 at
// mantissa bits 15..8) and computes the slab as fma(Q, A, c) with A = 2^15 a,
// a = s/d (exact: a power-of-two multiple, finite for |1/d| <= 2^64 and any
// node scale below 2^49), and c = (b -+ e) - A, since Q A = A + q a exactly
// inside the fma.  The rounding of c adds at most half an ulp of
// |b| + e + 2^15 |a|: 2^-24 |b|, inside the 2^-19 margin, plus 2^-9 |a|, which
// a further widening of 2^-8 |a| (1/256 of a quantum) covers.  The fast form
// also folds the interval ends' relative 2^-21 widening into the per-node
// slack: every slab value is at most |b| + 255 |a| (+ e) in magnitude, so a
// slack of 1.5 * 2^-19 (|b| + 255 |a|) lowers each near slab (raises each far
// one) by more than 2^-21 of its value on top of the 2^-19 margin, and the
// entry and exit need no per-child widening (checked against exact plane
// distances over random nodes and rays: the margin left is at least the exact
// form's 2^-19 slack plus its 2^-21 interval widening).  It pairs the near and
// far planes in packed fp32 fmas (fma.rn.f32x2, the same rounding per lane as a
// scalar fma).  Boxes of either form hold every triangle the test accepts, so
// both give the same hits.
struct NodeFrame {
  float px, py, pz, sxs, sys, szs;  // origin and scales of the quantisation grid
  float ax, ay, az;                 // slab = fma(q, a, b -+ e) per axis
  float blx, bly, blz, bhx, bhy, bhz;  // b - e (near planes), b + e (far planes)
};

APD NodeFrame node_frame(const uint4 w0, const RayPre& r) {
  NodeFrame f;
  f.px = __uint_as_float(w0.x);
  f.py = __uint_as_float(w0.y);
  f.pz = __uint_as_float(w0.z);
  f.sxs = __uint_as_float((w0.w & 0xffu) << 23);
  f.sys = __uint_as_float(((w0.w >> 8) & 0xffu) << 23);
  f.szs = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
  f.ax = f.sxs * r.inv.x;
  f.ay = f.sys * r.inv.y;
  f.az = f.szs * r.inv.z;
  const float bx = (f.px - r.o.x) * r.inv.x;
  const float by = (f.py - r.o.y) * r.inv.y;
  const float bz = (f.pz - r.o.z) * r.inv.z;
  const float kSlack = 1.9073486e-06f;  // 2^-19
  const float ex = (fabsf(bx) + 255.0f * fabsf(f.ax)) * kSlack;
  const float ey = (fabsf(by) + 255.0f * fabsf(f.ay)) * kSlack;
  const float ez = (fabsf(bz) + 255.0f * fabsf(f.az)) * kSlack;
  f.blx = bx - ex;
  f.bhx = bx + ex;
  f.bly = by - ey;
  f.bhy = by + ey;
  f.blz = bz - ez;
  f.bhz = bz + ez;
  return f;
}

// The fast form's per-node terms, paired for the packed fmas: (A_x, A_y) and
// (A_z, A_z) multiply (near x, near y), (far x, far y) and (near z, far z).
struct NodeFrameQ {
  float2 axy, azz;
  float2 cn_xy, cf_xy, c_z;  // c of the near x/y planes, the far x/y planes, near and far z
};

APD NodeFrameQ node_frame_q(const uint4 w0, const RayPre& r) {
  NodeFrameQ f;
  const float ax = __uint_as_float((w0.w & 0xffu) << 23) * r.inv.x;
  const float ay = __uint_as_float(((w0.w >> 8) & 0xffu) << 23) * r.inv.y;
  const float az = __uint_as_float(((w0.w >> 16) & 0xffu) << 23) * r.inv.z;
  const float bx = (__uint_as_float(w0.x) - r.o.x) * r.inv.x;
  const float by = (__uint_as_float(w0.y) - r.o.y) * r.inv.y;
  const float bz = (__uint_as_float(w0.z) - r.o.z) * r.inv.z;
  const float kSlack = 2.86102295e-06f;                 // 1.5 * 2^-19 of |b|
  const float kSlackA = 255.0f * 2.86102295e-06f + 0.00390625f;  // 1.5 * 2^-19 of the extent + 2^-8 of a quantum
  const float ex = fmaf(fabsf(ax), kSlackA, fabsf(bx) * kSlack);
  const float ey = fmaf(fabsf(ay), kSlackA, fabsf(by) * kSlack);
  const float ez = fmaf(fabsf(az), kSlackA, fabsf(bz) * kSlack);
  const float Ax = ax * 32768.0f, Ay = ay * 32768.0f, Az = az * 32768.0f;
  f.axy = make_float2(Ax, Ay);
  f.azz = make_float2(Az, Az);
  f.cn_xy = make_float2((bx - ex) - Ax, (by - ey) - Ay);
  f.cf_xy = make_float2((bx + ex) - Ax, (by + ey) - Ay);
  f.c_z = make_float2((bz - ez) - Az, (bz + ez) - Az);
  return f;
}

constexpr float kGrow = 1.0f + 4.8e-7f;  // relative 2^-21

// Byte k of `word` as a float.  Exact: the byte is placed under the exponent
// of 2^23 (0x4B000000) with one byte permute, and 2^23 + b - 2^23 = b exactly;
// this keeps the 48 conversions of a node off the conversion pipe.
APD float byte_at(uint32_t word, int k) {
  return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7440u | (uint32_t)k)) - 8388608.0f;
}

// Byte k of `word` as 1 + byte * 2^-15 (0x3F80bb00), one byte permute.
APD float byte_q15(uint32_t word, int k) {
  return __uint_as_float(__byte_perm(word, 0x3F800000u, 0x7604u | ((uint32_t)k << 4)));
}

// Packed fp32 fma (sm_100): a * b + c per lane, each rounded as fmaf.
APD float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

// A node's quantised child planes ordered by the ray's octant: per axis the
// words (children 0-3, 4-7) of the plane the ray enters first (near) and the
// one it leaves by (far).  With a negative direction component the larger
// coordinate is reached first, so lo and hi swap; then near <= far holds per
// child without a min/max (fma(q, a, b) is monotonic in q), and the values
// are the ones min/max would pick.  Zero components (inv = 0) keep lo/hi.
struct NodePlanes {
  uint32_t nx[2], fx[2], ny[2], fy[2], nz[2], fz[2];
};

APD NodePlanes node_planes(const uint4 w2, const uint4 w3, const uint4 w4, uint32_t neg) {
  NodePlanes p;
  const bool sx = neg & 1u, sy = neg & 2u, sz = neg & 4u;
  p.nx[0] = sx ? w3.z : w2.x;
  p.nx[1] = sx ? w3.w : w2.y;
  p.fx[0] = sx ? w2.x : w3.z;
  p.fx[1] = sx ? w2.y : w3.w;
  p.ny[0] = sy ? w4.x : w2.z;
  p.ny[1] = sy ? w4.y : w2.w;
  p.fy[0] = sy ? w2.z : w4.x;
  p.fy[1] = sy ? w2.w : w4.y;
  p.nz[0] = sz ? w4.z : w3.x;
  p.nz[1] = sz ? w4.w : w3.y;
  p.fz[0] = sz ? w3.x : w4.z;
  p.fz[1] = sz ? w3.y : w4.w;
  return p;
}

// Interval widening by a relative 2^-21 toward +-inf: x + |x| 2^-21 equals
// x * (1 + 2^-21) for x >= 0 and x * (1 - 2^-21) for x < 0, in one fma.
constexpr float kRelGrow = 4.76837158e-07f;  // 2^-21
APD float grow_up(float x) { return fmaf(fabsf(x), kRelGrow, x); }
APD float grow_down(float x) { return fmaf(-fabsf(x), kRelGrow, x); }

// Entry distance from the six slab values, or +inf when the box is missed
// inside [tmin, tmax]; tmax_grown = tmax * kGrow.
APD float slab_entry(float lx, float hx, float ly, float hy, float lz, float hz, float tmin, float tmax_grown) {
  const float tn = grow_down(fmaxf(fmaxf(lx, ly), fmaxf(lz, tmin)));
  const float tf = grow_up(fminf(fminf(hx, hy), hz));
  return (tn <= tf && tn <= tmax_grown) ? tn : __uint_as_float(0x7f800000u);
}

// Entry distance of child i (a compile-time index after unrolling), exact
// form, with the zero-direction-component test.
APD float child_entry(const NodeFrame& f, const NodePlanes& pl, const RayPre& r, int i, float tmin,
                      float tmax_grown) {
  const int k = i & 3, h = i >> 2;
  float lx = fmaf(byte_at(pl.nx[h], k), f.ax, f.blx), hx = fmaf(byte_at(pl.fx[h], k), f.ax, f.bhx);
  float ly = fmaf(byte_at(pl.ny[h], k), f.ay, f.bly), hy = fmaf(byte_at(pl.fy[h], k), f.ay, f.bhy);
  float lz = fmaf(byte_at(pl.nz[h], k), f.az, f.blz), hz = fmaf(byte_at(pl.fz[h], k), f.az, f.bhz);
  const float inf = __uint_as_float(0x7f800000u);
  if (r.zero_axes & 1u) {
    bool in = r.o.x >= f.px + byte_at(pl.nx[h], k) * f.sxs && r.o.x <= f.px + byte_at(pl.fx[h], k) * f.sxs;
    lx = in ? -inf : inf;
    hx = in ? inf : -inf;
  }
  if (r.zero_axes & 2u) {
    bool in = r.o.y >= f.py + byte_at(pl.ny[h], k) * f.sys && r.o.y <= f.py + byte_at(pl.fy[h], k) * f.sys;
    ly = in ? -inf : inf;
    hy = in ? inf : -inf;
  }
  if (r.zero_axes & 4u) {
    bool in = r.o.z >= f.pz + byte_at(pl.nz[h], k) * f.szs && r.o.z <= f.pz + byte_at(pl.fz[h], k) * f.szs;
    lz = in ? -inf : inf;
    hz = in ? inf : -inf;
  }
  return slab_entry(lx, hx, ly, hy, lz, hz, tmin, tmax_grown);
}

// Entry distance of child i, fast form (no zero or tiny direction component;
// the interval widening is in the slack).
APD float child_entry_q(const NodeFrameQ& f, const NodePlanes& pl, int i, float tmin, float tmax_grown) {
  const int k = i & 3, h = i >> 2;
  const float2 n = fma2(make_float2(byte_q15(pl.nx[h], k), byte_q15(pl.ny[h], k)), f.axy, f.cn_xy);
  const float2 x = fma2(make_float2(byte_q15(pl.fx[h], k), byte_q15(pl.fy[h], k)), f.axy, f.cf_xy);
  const float2 z = fma2(make_float2(byte_q15(pl.nz[h], k), byte_q15(pl.fz[h], k)), f.azz, f.c_z);
  const float tn = fmaxf(fmaxf(n.x, n.y), fmaxf(z.x, tmin));
  const float tf = fminf(fminf(x.x, x.y), z.y);
  return (tn <= tf && tn <= tmax_grown) ? tn : __uint_as_float(0x7f800000u);
}

// Entry distances of a node's 8 children (+inf where missed), the form picked
// once per node.
APD void child_entries(const uint4 w0, const uint4 w2, const uint4 w3, const uint4 w4, const RayPre& r, float tmin,
                       float tmax_grown, float tns[8]) {
  const NodePlanes pl = node_planes(w2, w3, w4, r.neg_axes);
  if (r.zero_axes) {
    const NodeFrame f = node_frame(w0, r);
#pragma unroll
    for (int i = 0; i < 8; ++i) tns[i] = child_entry(f, pl, r, i, tmin, tmax_grown);
  } else {
    const NodeFrameQ f = node_frame_q(w0, r);
#pragma unroll
    for (int i = 0; i < 8; ++i) tns[i] = child_entry_q(f, pl, i, tmin, tmax_grown);
  }
}

APD uint32_t meta_of(const uint4 w1, int i) { return ((i < 4 ? w1.z : w1.w) >> (8 * (i & 3))) & 0xffu; }

// Visit counters of one ray (instrumented builds of the traversal kernels).
struct Visits {
  uint32_t nodes = 0, tris = 0;
};

// Resumable traversal of one ray.  Closest hit: the nearest hit inner child is
// visited next and the others are pushed with their entry distance, culled on
// pop; any hit: stops at the first accepted triangle.  The traversal stack
// holds at most BvhStats::max_stack entries (checked at build).
//
// One step is either one node (8 child boxes) or one triangle: the triangles
// of a node's leaf children (at most 24, stored contiguously from the node's
// triangle base) become a pending bit mask that the following steps test one
// at a time, before the next node.  Short, uniform steps keep the lanes of a
// warp on the same path more of the time than testing all of a node's
// triangles at once.
struct Trav {
  RayPre r;
  Hit hit;          // closest: best so far (hit.t doubles as tmax); any: hit.tri != kNoHit when occluded
  float tmax;       // any-hit query range
  uint32_t node;
  float node_t;     // entry distance of `node` (closest hit)
  uint32_t tri_base, tri_mask;  // pending triangles: tri_base + bit index
  int sp;
  bool have;        // `node` is the next node to visit
};

APD void trav_init(Trav& t, float3 o, float3 d, float tmax) {
  t.r = ray_pre(o, d);
  t.hit.t = tmax;
  t.hit.u = 0.0f;
  t.hit.v = 0.0f;
  t.hit.tri = kNoHit;
  t.tmax = tmax;
  t.node = 0;
  t.node_t = 0.0f;
  t.tri_base = 0;
  t.tri_mask = 0;
  t.sp = 0;
  t.have = true;
}

// Runs up to `budget` steps; returns true when the ray is finished.  kUnroll
// unrolls the 8 child tests.
// The scene S is a DevScene or any view with the same `nodes` and `tris`
// (the only fields the traversal reads), such as BvhView.
struct BvhView {
  const uint4* nodes;
  const float4* tris;
};

template <bool kAny, bool kCount, bool kUnroll = false, class S>
APD bool trav_step(const S& s, Trav& t, uint2* stack, int budget, Visits* vc) {
  for (int step = 0; step < budget; ++step) {
    if (t.tri_mask) {
      const int j = __ffs(t.tri_mask) - 1;
      t.tri_mask &= t.tri_mask - 1;
      if (kCount) vc->tris++;
      const float4* tp = s.tris + 3 * (size_t)(t.tri_base + j);
      const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
      float th, u, v;
      const float lim = kAny ? t.tmax : t.hit.t;
      if (intersect_tri(t.r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z), 0.0f, lim, th, u, v)) {
        const uint32_t gid = __float_as_uint(a.w);
        if (kAny) {
          t.hit.tri = gid;
          return true;
        }
        if (th < t.hit.t || gid < t.hit.tri) {  // th <= hit.t here: strictly closer or a tie
          t.hit.t = th;
          t.hit.u = u;
          t.hit.v = v;
          t.hit.tri = gid;
        }
      }
      continue;
    }
    if (t.have && !kAny && t.node_t > t.hit.t * kGrow) t.have = false;  // culled by a hit found since
    if (!t.have) {
      bool got = false;
      while (t.sp > 0) {
        uint2 e = stack[--t.sp];
        if (kAny || __uint_as_float(e.y) <= t.hit.t * kGrow) {
          t.node = e.x;
          got = true;
          break;
        }
      }
      if (!got) return true;
    }
    t.have = false;
    if (kCount) vc->nodes++;
    const uint4* np = s.nodes + 5 * (size_t)t.node;
    const uint4 w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
    const float range_grown = (kAny ? t.tmax : t.hit.t) * kGrow;
    uint32_t tri_mask = 0;
    float best_t = __uint_as_float(0x7f800000u);
    uint32_t best_node = 0;
    float tns[8];
    child_entries(w0, w2, w3, w4, t.r, 0.0f, range_grown, tns);
#pragma unroll(kUnroll ? 8 : 1)
    for (int i = 0; i < 8; ++i) {
      const uint32_t meta = meta_of(w1, i);
      if (meta == 0u) continue;
      const float tn = tns[i];
      if (!(tn < __uint_as_float(0x7f800000u))) continue;
      if (meta & 0xe0u) {
        tri_mask |= (meta >> 5) << (meta & 0x1fu);  // unary count at the leaf's offset
      } else {
        const uint32_t child = w1.x + (meta & 7u);
        if (tn < best_t) {  // nearest child next (any hit too: occluders near the origin are found sooner)
          if (t.have && t.sp < kTraversalStack) stack[t.sp++] = make_uint2(best_node, __float_as_uint(best_t));
          best_t = tn;
          best_node = child;
          t.have = true;
        } else if (t.sp < kTraversalStack) {
          stack[t.sp++] = make_uint2(child, __float_as_uint(tn));
        }
      }
    }
    t.node = best_node;
    t.node_t = best_t;
    t.tri_base = w1.y;
    t.tri_mask = tri_mask;
  }
  return false;
}

// ---- Loop-form traversal for rays traced inline in the large resampling
// kernels.  Same box test (child_entries), same culling and tie rules as
// trav_step, hence the same results; the loop form has no resumable state,
// which keeps these kernels' code and local memory small.  Returns the hit
// mask; tnear[] gets the entry distance of each hit child.
template <bool kClosest>
APD uint32_t inline_children(const uint4 w0, const uint4 w2, const uint4 w3, const uint4 w4,
                           const RayPre& r, float tmin, float tmax, float tnear[8]) {
  child_entries(w0, w2, w3, w4, r, tmin, tmax * kGrow, tnear);
  uint32_t mask = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (tnear[i] < __uint_as_float(0x7f800000u)) mask |= 1u << i;
  return mask;
}

// Closest hit in [0, tmax] (returns false on miss).  Tie rule: smaller t, then
// smaller global triangle id.
template <bool kCount = false>
APD bool trace_closest(const DevScene& s, float3 o, float3 d, float tmax, Hit& hit, Visits* vc = nullptr) {
  RayPre r = ray_pre(o, d);
  hit.t = tmax;
  hit.u = 0.0f;
  hit.v = 0.0f;
  hit.tri = kNoHit;
  uint2 stack[kTraversalStack];
  int sp = 0;
  uint32_t node = 0;
  bool have = true;
  while (true) {
    if (!have) {
      if (sp == 0) break;
      uint2 e = stack[--sp];
      if (__uint_as_float(e.y) > hit.t * (1.0f + 4.8e-7f)) continue;
      node = e.x;
    }
    have = false;
    if (kCount) vc->nodes++;
    const uint4* np = s.nodes + 5 * (size_t)node;
    uint4 w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3),
          w4 = __ldg(np + 4);
    float tnear[8];
    uint32_t mask = inline_children<true>(w0, w2, w3, w4, r, 0.0f, hit.t, tnear);
    // leaves first (their hits shrink hit.t before the inner children are ordered)
    uint32_t todo = mask;
    while (todo) {
      int i = __ffs(todo) - 1;
      todo &= todo - 1;
      uint32_t meta = meta_of(w1, i);
      if ((meta & 0xe0u) == 0) continue;
      uint32_t first = w1.y + (meta & 0x1fu);
      uint32_t cnt = __popc(meta >> 5);
      if (kCount) vc->tris += cnt;
      for (uint32_t k = 0; k < cnt; ++k) {
        const float4* tp = s.tris + 3 * (size_t)(first + k);
        float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float t, u, v;
        if (intersect_tri(r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z), 0.0f, hit.t, t, u, v)) {
          uint32_t gid = __float_as_uint(a.w);
          if (t < hit.t || gid < hit.tri) {  // t <= hit.t here: strict or tie
            hit.t = t;
            hit.u = u;
            hit.v = v;
            hit.tri = gid;
          }
        }
      }
    }
    // inner children: continue with the nearest, push the rest
    float best_t = 3.4e38f;
    int best_i = -1;
    todo = mask;
    while (todo) {
      int i = __ffs(todo) - 1;
      todo &= todo - 1;
      uint32_t meta = meta_of(w1, i);
      if ((meta & 0xf0u) != 0x10u) continue;
      if (tnear[i] > hit.t * (1.0f + 4.8e-7f)) continue;
      if (tnear[i] < best_t) {
        if (best_i >= 0 && sp < kTraversalStack)
          stack[sp++] = make_uint2(w1.x + (meta_of(w1, best_i) & 7u), __float_as_uint(best_t));
        best_t = tnear[i];
        best_i = i;
      } else if (sp < kTraversalStack) {
        stack[sp++] = make_uint2(w1.x + (meta & 7u), __float_as_uint(tnear[i]));
      }
    }
    if (best_i >= 0) {
      node = w1.x + (meta_of(w1, best_i) & 7u);
      have = true;
    }
  }
  return hit.tri != kNoHit;
}

// Any hit in [0, tmax] (shadow rays: terminate on first hit).  Same stack
// discipline as trace_closest (continue with one inner child, push the rest),
// so the build-time bound on stack depth (BvhStats::max_stack) covers both.
template <bool kCount = false>
APD bool trace_any(const DevScene& s, float3 o, float3 d, float tmax, Visits* vc = nullptr) {
  RayPre r = ray_pre(o, d);
  uint32_t stack[kTraversalStack];
  int sp = 0;
  uint32_t node = 0;
  bool have = true;
  while (true) {
    if (!have) {
      if (sp == 0) break;
      node = stack[--sp];
    }
    have = false;
    if (kCount) vc->nodes++;
    const uint4* np = s.nodes + 5 * (size_t)node;
    uint4 w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3),
          w4 = __ldg(np + 4);
    float tnear[8];
    uint32_t mask = inline_children<false>(w0, w2, w3, w4, r, 0.0f, tmax, tnear);
    uint32_t todo = mask;
    while (todo) {
      int i = __ffs(todo) - 1;
      todo &= todo - 1;
      uint32_t meta = meta_of(w1, i);
      if ((meta & 0xe0u) != 0) {
        uint32_t first = w1.y + (meta & 0x1fu);
        uint32_t cnt = __popc(meta >> 5);
        for (uint32_t k = 0; k < cnt; ++k) {
          const float4* tp = s.tris + 3 * (size_t)(first + k);
          float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
          float t, u, v;
          if (kCount) vc->tris++;
          if (intersect_tri(r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z), 0.0f, tmax, t, u, v))
            return true;
        }
      } else if (!have) {
        node = w1.x + (meta & 7u);
        have = true;
      } else if (sp < kTraversalStack) {
        stack[sp++] = w1.x + (meta & 7u);
      }
    }
  }
  return false;
}

}  // namespace ap
