// The world of a renderer handle as the reference's world actions build it
// (VisibleWorldActionType, crates/appearance-world/src/visible_world_action.rs:
// 9-125; handled by PathTracerGpu's SceneResources::handle_visible_world_action,
// crates/appearance-path-tracer-gpu/src/scene_resources/mod.rs:107-156):
// models registered under an asset path (the reference loads them from its
// asset database by that path), instances spawned from them with a 4x4
// transform and an entity uuid, moved, destroyed, cleared.  The device scene
// of a handle is the uploaded base scene plus every live instance, flattened
// to world space in spawn order (the reference rebuilds its TLAS before every
// frame); a change marks the world dirty and the next render re-uploads it.
#pragma once

#include <stdint.h>

#include <array>
#include <map>
#include <string>
#include <vector>

#include "../../include/appearance_cuda.h"
#include "scene_layout.h"

namespace ap {

// An owned copy of an ap_scene_desc.
struct HostScene {
  std::vector<float> positions, normals, env;
  std::vector<uint32_t> indices, tri_material;
  std::vector<ap_mesh> meshes;
  std::vector<ap_material> materials;
  uint32_t env_w = 0, env_h = 0;
  float sun[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  void assign(const ap_scene_desc& d);
  ap_scene_desc desc() const;
  uint32_t num_tris() const { return (uint32_t)(indices.size() / 3); }
};

// Wire sizes of the world actions (bytemuck layouts, visible_world_action.rs).
constexpr size_t kSpawnModelBytes = 64 + 16 + 256;  // Mat4, Uuid, asset path
constexpr size_t kTransformModelBytes = 64 + 16;    // Mat4, Uuid
constexpr size_t kDestroyModelBytes = 16;           // Uuid

// The two-level form of a world (traverse2.cuh): one object-space BLAS per
// model in a shared node / triangle pool (triangle records carry the model's
// triangle index), a TLAS over the instances' world boxes (records carry the
// instance index), and the instances: the base scene first (identity), then
// every spawned instance in spawn order, so that global triangle ids are the
// flattened world's.
struct TwoLevelHost {
  std::vector<WideNode> nodes, tlas_nodes;
  std::vector<TriRec> tris, tlas_leaves;
  std::vector<InstRec> insts;
  uint32_t max_stack = 0;  // TLAS stack bound + the largest BLAS bound + 1
  // the models' geometry for shading, in model space: vertex positions
  // (x, y, z, 0) and normals (3 floats), per model triangle its three vertex
  // indices into those arrays and its material index into `materials`; each
  // model's first triangle
  std::vector<float> positions4, normals;
  std::vector<uint32_t> indices, tri_material, model_tri0;
  std::vector<ap_material> materials;
  // per global triangle id, the instance it belongs to
  std::vector<uint32_t> tri_inst;
};

// World-to-object rows (row-major 3x4) of a column-major Mat4: its inverse
// by cofactors in double, rounded to float.
void inverse_rows(const float m[16], float w2o[12]);

struct World {
  struct Instance {
    std::array<uint8_t, 16> uuid;
    std::string path;
    float m[16];  // column-major (glam Mat4)
  };
  HostScene base;
  std::map<std::string, HostScene> models;
  std::vector<Instance> instances;  // spawn order
  bool dirty = false;
  uint64_t version = 0;  // bumped by every change of the base scene, a model or an instance

  // Each returns AP_OK or an AP_E_* status with `err` set.
  int spawn(const uint8_t* bytes, size_t len, std::string* err);
  int transform(const uint8_t* bytes, size_t len, std::string* err);
  int destroy(const uint8_t* bytes, size_t len, std::string* err);
  // Clear: drops the base scene and every instance (the registered models
  // stay, as the reference's asset database does).
  void clear();
  // base + instances, in world space: positions by the instance transform,
  // normals by its inverse transpose (renormalised); a model's materials are
  // appended once, the first time one of its instances is.
  void flatten(HostScene* out) const;
  // The two-level form (false with `err` when a BVH would exceed `max_stack`);
  // the base scene is model 0 with the identity instance when it has meshes.
  bool build_two_level(uint32_t max_stack, TwoLevelHost* out, std::string* err) const;
};

}  // namespace ap
