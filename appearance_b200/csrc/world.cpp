// World actions and the flattening of a handle's world (world.h).
#include "world.h"

#include <cmath>
#include <cstring>

namespace ap {

void HostScene::assign(const ap_scene_desc& d) {
  positions.assign(d.positions, d.positions + 3 * (size_t)d.num_vertices);
  normals.assign(d.normals, d.normals + 3 * (size_t)d.num_vertices);
  indices.assign(d.indices, d.indices + 3 * (size_t)d.num_tris);
  tri_material.assign(d.tri_material, d.tri_material + d.num_tris);
  meshes.assign(d.meshes, d.meshes + d.num_meshes);
  materials.assign(d.materials, d.materials + d.num_materials);
  env_w = d.env && d.env_w && d.env_h ? d.env_w : 0;
  env_h = env_w ? d.env_h : 0;
  if (env_w) env.assign(d.env, d.env + 3 * (size_t)env_w * env_h);
  else env.clear();
  std::memcpy(sun, d.sun, sizeof(sun));
}

ap_scene_desc HostScene::desc() const {
  ap_scene_desc d;
  std::memset(&d, 0, sizeof(d));
  d.positions = positions.data();
  d.normals = normals.data();
  d.num_vertices = (uint32_t)(positions.size() / 3);
  d.indices = indices.data();
  d.tri_material = tri_material.data();
  d.num_tris = (uint32_t)(indices.size() / 3);
  d.meshes = meshes.data();
  d.num_meshes = (uint32_t)meshes.size();
  d.materials = materials.data();
  d.num_materials = (uint32_t)materials.size();
  d.env = env_w ? env.data() : nullptr;
  d.env_w = env_w;
  d.env_h = env_h;
  std::memcpy(d.sun, sun, sizeof(sun));
  return d;
}

namespace {

std::array<uint8_t, 16> uuid_of(const uint8_t* p) {
  std::array<uint8_t, 16> u;
  std::memcpy(u.data(), p, 16);
  return u;
}

}  // namespace

// SpawnModelData {Mat4 transform, Uuid entity, [u8; 256] asset path}
// (visible_world_action.rs:17-48): the path ends at its first NUL.  A uuid
// spawned again replaces its instance (the reference's map insert).
int World::spawn(const uint8_t* b, size_t len, std::string* err) {
  if (!b || len != kSpawnModelBytes) {
    *err = "SpawnModel expects " + std::to_string(kSpawnModelBytes) + " bytes";
    return AP_E_INVALID;
  }
  const char* path = reinterpret_cast<const char*>(b + 80);
  size_t n = 0;
  while (n < 256 && path[n]) ++n;
  std::string p(path, n);
  if (!models.count(p)) {
    *err = "SpawnModel: no model registered under \"" + p + "\" (ap_model_register)";
    return AP_E_INVALID;
  }
  Instance in;
  std::memcpy(in.m, b, 64);
  in.uuid = uuid_of(b + 64);
  in.path = p;
  for (Instance& e : instances)
    if (e.uuid == in.uuid) {
      e = in;
      dirty = true;
      return AP_OK;
    }
  instances.push_back(in);
  dirty = true;
  return AP_OK;
}

// TransformModelData {Mat4 transform, Uuid entity} (visible_world_action.rs:50-55).
// The reference only logs a warning for an unknown entity; here it is an
// error the caller may ignore.
int World::transform(const uint8_t* b, size_t len, std::string* err) {
  if (!b || len != kTransformModelBytes) {
    *err = "TransformModel expects " + std::to_string(kTransformModelBytes) + " bytes";
    return AP_E_INVALID;
  }
  const std::array<uint8_t, 16> u = uuid_of(b + 64);
  for (Instance& e : instances)
    if (e.uuid == u) {
      std::memcpy(e.m, b, 64);
      dirty = true;
      return AP_OK;
    }
  *err = "TransformModel: unknown entity";
  return AP_E_INVALID;
}

// DestroyModelData {Uuid entity} (visible_world_action.rs:57-61); an unknown
// entity is ignored, as the reference's map remove does.
int World::destroy(const uint8_t* b, size_t len, std::string* err) {
  if (!b || len != kDestroyModelBytes) {
    *err = "DestroyModel expects 16 bytes";
    return AP_E_INVALID;
  }
  const std::array<uint8_t, 16> u = uuid_of(b);
  for (size_t i = 0; i < instances.size(); ++i)
    if (instances[i].uuid == u) {
      instances.erase(instances.begin() + (long)i);
      dirty = true;
      break;
    }
  return AP_OK;
}

void World::clear() {
  base = HostScene();
  instances.clear();
  dirty = true;
}

void World::flatten(HostScene* out) const {
  *out = base;
  std::map<std::string, uint32_t> material_base;
  for (const Instance& in : instances) {
    const HostScene& mdl = models.at(in.path);
    uint32_t mat0;
    auto it = material_base.find(in.path);
    if (it == material_base.end()) {
      mat0 = (uint32_t)out->materials.size();
      out->materials.insert(out->materials.end(), mdl.materials.begin(), mdl.materials.end());
      material_base[in.path] = mat0;
    } else {
      mat0 = it->second;
    }
    const float* m = in.m;
    // inverse transpose of the upper 3x3 (column-major a[c][r] = m[4c + r]), in double
    double a[3][3];
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) a[c][r] = m[4 * c + r];
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) -
                       a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2]) +
                       a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
    float nt[3][3];  // nt[r][k]: row r of the inverse transpose
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) {
        // (A^-1)^T[r][k] = cofactor(r, k) / det of A (rows r, columns k)
        const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        const double cof = a[k1][r1] * a[k2][r2] - a[k2][r1] * a[k1][r2];
        nt[r][k] = (float)(det != 0.0 ? cof / det : 0.0);
      }
    const uint32_t v0 = (uint32_t)(out->positions.size() / 3);
    const uint32_t t0 = (uint32_t)(out->indices.size() / 3);
    const size_t nv = mdl.positions.size() / 3;
    for (size_t i = 0; i < nv; ++i) {
      const float x = mdl.positions[3 * i], y = mdl.positions[3 * i + 1], z = mdl.positions[3 * i + 2];
      for (int r = 0; r < 3; ++r) out->positions.push_back(m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r]);
      const float nx = mdl.normals[3 * i], ny = mdl.normals[3 * i + 1], nz = mdl.normals[3 * i + 2];
      float n[3];
      for (int r = 0; r < 3; ++r) n[r] = nt[r][0] * nx + nt[r][1] * ny + nt[r][2] * nz;
      const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      const float s = l > 0.0f ? 1.0f / l : 0.0f;
      for (int r = 0; r < 3; ++r) out->normals.push_back(n[r] * s);
    }
    out->indices.insert(out->indices.end(), mdl.indices.begin(), mdl.indices.end());
    out->tri_material.insert(out->tri_material.end(), mdl.tri_material.begin(), mdl.tri_material.end());
    for (ap_mesh me : mdl.meshes) {
      me.first_vertex += v0;
      me.first_index += 3 * t0;
      me.material_idx += mat0;
      out->meshes.push_back(me);
    }
  }
}

}  // namespace ap
