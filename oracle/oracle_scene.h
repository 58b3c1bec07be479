// Oracle (test infrastructure only): scene data, watertight ray/triangle test
// and a plain binned-SAH binary BVH for the CPU restatement of the frame.
#pragma once

#include <stdint.h>

#include <vector>

#include "oracle_math.h"

namespace orc {

// MaterialDescriptor (shared/material/material_pool.wgsl:6-41) without the
// texture slots: the synthetic scenes carry constant Disney parameters.
struct Material {
  float color[3];
  float metallic, roughness;
  float emission[3];
  float transmission, eta, subsurface;
  float absorption[3];
  float specular;
  float specular_tint[3];
  float anisotropic, sheen;
  float sheen_tint[3];
  float clearcoat, clearcoat_roughness, alpha_cutoff;
};

// VertexPoolSlice (shared/vertex_pool.wgsl:3-12) plus the emissive instance
// index that BlasInstance (vertex_pool.wgsl:22-27) carries.
struct Instance {
  uint32_t first_vertex, num_vertices, first_index, num_indices;
  uint32_t material_idx;
  uint32_t emissive_idx;      // 0xFFFFFFFF when not emissive
  uint32_t first_global_tri;  // position of triangle 0 in the flattened list
};

struct Sun {
  float direction[3];
  float size;
  float color[3];
  float intensity;
};

struct Scene {
  std::vector<V3> positions;         // world space, per vertex
  std::vector<uint32_t> normals;     // oct30 packed, per vertex
  std::vector<uint32_t> indices;     // 3 per triangle, relative to first_vertex
  std::vector<uint32_t> tri_material;  // per triangle, relative to material_idx
  std::vector<Instance> instances;
  std::vector<Material> materials;
  std::vector<uint32_t> emissive_instances;  // instance index per emissive instance
  std::vector<float> emissive_cdf;
  uint32_t num_emissive_tris = 0;
  // flattened triangle list: global triangle -> instance
  std::vector<uint32_t> tri_instance;
  // equirect environment, RGB f32 row-major (env_w x env_h), may be empty
  std::vector<float> env;
  uint32_t env_w = 0, env_h = 0;
  Sun sun{};

  uint32_t num_tris() const { return (uint32_t)tri_instance.size(); }
  void tri_verts(uint32_t g, V3& a, V3& b, V3& c) const {
    const Instance& in = instances[tri_instance[g]];
    uint32_t l = g - in.first_global_tri;
    a = positions[in.first_vertex + indices[in.first_index + l * 3 + 0]];
    b = positions[in.first_vertex + indices[in.first_index + l * 3 + 1]];
    c = positions[in.first_vertex + indices[in.first_index + l * 3 + 2]];
  }
};

struct Hit {
  float t, u, v;
  uint32_t tri;  // global triangle id, 0xFFFFFFFF on miss
};

// Watertight ray/triangle intersection (S. Woop, C. Benthin, I. Wald,
// "Watertight Ray/Triangle Intersection", JCGT 2(1) 2013): the inside test and
// the barycentrics in binary32 with the double-precision fallback for zero
// edge functions; the distance t in double precision from the original
// vertices (plane distance), rounded once.  Returns true and fills t, u (weight
// of v1), v (weight of v2) when tmin <= t <= tmax.
struct RayPre {
  V3 o, d;
  int kx, ky, kz;
  float sx, sy, sz;
};
inline float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
inline RayPre ray_pre(V3 o, V3 d) {
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
  r.kx = kx; r.ky = ky; r.kz = kz;
  r.sx = comp(d, kx) / comp(d, kz);
  r.sy = comp(d, ky) / comp(d, kz);
  r.sz = 1.0f / comp(d, kz);
  return r;
}
inline bool intersect_tri(const RayPre& r, V3 v0, V3 v1, V3 v2, float tmin, float tmax,
                          float& t, float& u, float& v) {
  V3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
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
  // distance along the ray in double precision from the original vertices
  // (accurate where the float sheared form loses sign for hits near t = 0)
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

// Binary BVH used only by the oracle: binned SAH build, closest hit with the
// total order (t, global triangle id), any hit for shadow rays.
class OracleBvh {
 public:
  void build(const Scene& s);
  Hit closest(const Scene& s, V3 o, V3 d, float tmin, float tmax, uint64_t* nodes_visited,
              uint64_t* tris_tested) const;
  bool any(const Scene& s, V3 o, V3 d, float tmin, float tmax) const;

 private:
  struct Node {
    float lo[3], hi[3];
    uint32_t left_or_first;  // inner: left child; leaf: first index into order
    uint32_t count;          // 0 for inner nodes (right child = left + 1)
  };
  std::vector<Node> nodes_;
  std::vector<uint32_t> order_;
};

}  // namespace orc
