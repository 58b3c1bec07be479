// Device-resident scene layout shared by the host uploader and the kernels.
//
// All meshes of a scene are flattened into one world-space vertex pool (the
// reference's VertexPoolSlice list, shared/vertex_pool.wgsl:3-12); instance
// transforms are applied at upload, so the per-hit world_to_object transform
// of the reference (trace.wgsl:147-158) is the identity here.
#pragma once

#include <stdint.h>

namespace ap {

// One mesh: VertexPoolSlice + BlasInstance::emissive_blas_instance_idx.
struct InstanceDev {
  uint32_t first_vertex;
  uint32_t first_index;       // into indices (3 per triangle)
  uint32_t num_indices;
  uint32_t material_idx;      // first material of the mesh
  uint32_t emissive_idx;      // index into emissive_instances, or 0xFFFFFFFF
  uint32_t first_global_tri;  // first triangle in the flattened triangle list
  uint32_t pad0, pad1;
};

// MaterialDescriptor (shared/material/material_pool.wgsl:6-41) without texture
// slots; same float order as ap_material.
struct MaterialDev {
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

struct SunDev {
  float direction[3];
  float size;
  float color[3];
  float intensity;
  // Derived once per scene upload on the device (k_sun_derive), with the
  // arithmetic the sun functions would otherwise repeat on every call:
  float it;         // intensity x horizon falloff (Sky::sun_intensity)
  float cos_size;   // cos(size * 0.1): the sun disk's angular radius
  float l[3];       // -direction: toward the sun
  float bt[3], tg[3];  // tangent frame around l (perpendicular(l), cross(bt, l))
};

// Compressed 8-wide BVH node, 80 bytes = 5 x uint4:
//   w0: p.x, p.y, p.z (float bits), e.x | e.y << 8 | e.z << 16 | imask << 24
//   w1: child_base, tri_base, meta[0..3], meta[4..7]
//   w2: qlo_x[0..7], qlo_y[0..7]     w3: qlo_z[0..7], qhi_x[0..7]
//   w4: qhi_y[0..7], qhi_z[0..7]
// A child box is p + q * 2^(e - 127) per axis, rounded outward at build time.
// meta: 0 empty; 0x10 | rank for an inner child (node child_base + rank);
// (unary triangle count << 5) | offset for a leaf of 1..3 triangles starting
// at triangle tri_base + offset.
struct WideNode {
  uint32_t w[20];
};

// Triangle record in leaf order, 48 bytes: v0.xyz + global triangle id (bits),
// v1.xyz + 0, v2.xyz + 0.
struct TriRec {
  float v[12];
};

// One emissive triangle, precomputed at upload with the same expressions the
// light sampler would evaluate (80 bytes): vertices, area = |cross(e1, e2)|/2,
// unit normal = normalize(cross(e1, e2)), emission of its material.
struct EmissiveTri {
  float p0[3], area;
  float p1[3], pad0;
  float p2[3], pad1;
  float n[3], pad2;
  float emission[3], pad3;
};

// Instance of a two-level scene (traverse2.cuh), 128 bytes: world-to-object
// and object-to-world transforms (row-major 3x4), the root of its model's
// BLAS in the node pool, its first global triangle id, its model.
struct InstRec {
  float w2o[12];
  uint32_t blas_root, tri_base, model, pad0;
  float o2w[12];
  uint32_t pad1[4];
};

struct DevScene {
  const uint4* nodes;       // 5 per WideNode
  const float4* tris;       // 3 per TriRec
  const float4* positions;  // world position per vertex (w = 0)
  const uint32_t* normals;  // oct30 per vertex
  const float* normals_f;   // the same normals as floats, 3 per vertex
  const uint32_t* indices;  // mesh-local vertex index, 3 per triangle
  const uint32_t* tri_material;
  const uint32_t* tri_instance;  // flattened triangle -> instance
  const InstanceDev* instances;
  const MaterialDev* materials;
  const uint32_t* emissive_instances;  // emissive index -> instance
  const float* emissive_cdf;
  const EmissiveTri* emissive_tris;     // all triangles of the emissive instances
  const uint32_t* emissive_tri_base;    // emissive instance -> first record
  // per emissive instance: {CDF entry (float bits), first emissive-triangle
  // record, triangle count, 0}: what light sampling needs in one 16-byte load
  const uint4* emissive_info;
  uint32_t num_emissive_instances;
  uint32_t num_emissive_tris;
  const float* env;  // equirect RGB, env_w x env_h, or null
  uint32_t env_w, env_h;
  SunDev sun;
  uint32_t num_tris;
};

}  // namespace ap
