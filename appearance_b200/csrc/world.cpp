// World actions and the flattening of a handle's world (world.h).
#include "world.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "bvh_build.h"

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
  ++version;
  dirty = true;
  for (Instance& e : instances)
    if (e.uuid == in.uuid) {
      e = in;
      return AP_OK;
    }
  instances.push_back(in);
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
      ++version;
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
      ++version;
      break;
    }
  return AP_OK;
}

void World::clear() {
  base = HostScene();
  instances.clear();
  dirty = true;
  ++version;
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

void inverse_rows(const float m[16], float w2o[12]) {
  double a[4][4];  // a[r][c] of the matrix, m column-major
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) a[r][c] = m[4 * c + r];
  // affine: inverse of the upper 3x3 by cofactors, then -A^-1 t
  const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                     a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                     a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  double inv[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      // inv[r][c] = cofactor(c, r) / det
      const int c1 = (c + 1) % 3, c2 = (c + 2) % 3, r1 = (r + 1) % 3, r2 = (r + 2) % 3;
      const double cof = a[c1][r1] * a[c2][r2] - a[c1][r2] * a[c2][r1];
      inv[r][c] = det != 0.0 ? cof / det : 0.0;
    }
  for (int r = 0; r < 3; ++r) {
    const double t = -(inv[r][0] * a[0][3] + inv[r][1] * a[1][3] + inv[r][2] * a[2][3]);
    for (int c = 0; c < 3; ++c) w2o[4 * r + c] = (float)inv[r][c];
    w2o[4 * r + 3] = (float)t;
  }
}

namespace {

void model_triangles(const HostScene& m, std::vector<float>* tv) {
  tv->resize(9 * (size_t)m.num_tris());
  for (const ap_mesh& me : m.meshes)
    for (uint32_t t = 0; t < me.num_indices / 3; ++t) {
      const uint32_t g = me.first_index / 3 + t;
      for (int k = 0; k < 3; ++k) {
        const uint32_t v = me.first_vertex + m.indices[3 * (size_t)g + k];
        for (int a = 0; a < 3; ++a) (*tv)[9 * (size_t)g + 3 * k + a] = m.positions[3 * (size_t)v + a];
      }
    }
}

}  // namespace

bool World::build_two_level(uint32_t max_stack, TwoLevelHost* out, std::string* err) const {
  *out = TwoLevelHost();
  // models in first-use order: the base scene, then spawned models
  std::vector<const HostScene*> mods;
  std::map<std::string, uint32_t> index;
  std::vector<uint32_t> inst_model;
  std::vector<const float*> inst_m;
  static const float kIdentity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  if (!base.meshes.empty()) {
    mods.push_back(&base);
    inst_model.push_back(0);
    inst_m.push_back(kIdentity);
  }
  for (const Instance& in : instances) {
    auto it = index.find(in.path);
    if (it == index.end()) {
      it = index.emplace(in.path, (uint32_t)mods.size()).first;
      mods.push_back(&models.at(in.path));
    }
    inst_model.push_back(it->second);
    inst_m.push_back(in.m);
  }
  std::vector<uint32_t> root(mods.size());
  std::vector<float> box(6 * mods.size());
  uint32_t blas_stack = 0;
  for (size_t k = 0; k < mods.size(); ++k) {
    std::vector<float> tv;
    model_triangles(*mods[k], &tv);
    WideBvh b;
    if (!build_wide_bvh(tv.data(), mods[k]->num_tris(), max_stack, &b, err)) return false;
    const uint32_t node0 = (uint32_t)out->nodes.size(), tri0 = (uint32_t)out->tris.size();
    for (WideNode n : b.nodes) {
      n.w[4] += node0;  // child base
      n.w[5] += tri0;   // triangle base
      out->nodes.push_back(n);
    }
    out->tris.insert(out->tris.end(), b.tris.begin(), b.tris.end());
    root[k] = node0;
    blas_stack = std::max(blas_stack, b.stats.max_stack);
    // shading geometry: vertices, per-triangle vertex indices and materials
    const HostScene& ms = *mods[k];
    const uint32_t v0 = (uint32_t)(out->positions4.size() / 4), mat0 = (uint32_t)out->materials.size();
    out->model_tri0.push_back((uint32_t)(out->indices.size() / 3));
    for (size_t i = 0; i < ms.positions.size() / 3; ++i) {
      for (int a = 0; a < 3; ++a) out->positions4.push_back(ms.positions[3 * i + a]);
      out->positions4.push_back(0.0f);
    }
    out->normals.insert(out->normals.end(), ms.normals.begin(), ms.normals.end());
    out->materials.insert(out->materials.end(), ms.materials.begin(), ms.materials.end());
    for (const ap_mesh& me : ms.meshes)
      for (uint32_t t = 0; t < me.num_indices / 3; ++t) {
        const uint32_t g = me.first_index / 3 + t;
        for (int c = 0; c < 3; ++c) out->indices.push_back(v0 + me.first_vertex + ms.indices[3 * (size_t)g + c]);
        out->tri_material.push_back(mat0 + me.material_idx + ms.tri_material[g]);
      }
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (size_t i = 0; i < tv.size(); i += 3)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], tv[i + a]);
        hi[a] = std::max(hi[a], tv[i + a]);
      }
    for (int a = 0; a < 3; ++a) {
      box[6 * k + a] = lo[a];
      box[6 * k + 3 + a] = hi[a];
    }
  }
  // instances and their world boxes (the model box's corners under the
  // transform, in double, widened and rounded outward)
  std::vector<float> leaves(9 * inst_model.size());
  uint32_t tri_base = 0;
  for (size_t i = 0; i < inst_model.size(); ++i) {
    const uint32_t k = inst_model[i];
    const float* m = inst_m[i];
    InstRec r;
    std::memset(&r, 0, sizeof(r));
    inverse_rows(m, r.w2o);
    for (int row = 0; row < 3; ++row)
      for (int c = 0; c < 4; ++c) r.o2w[4 * row + c] = m[4 * c + row];
    r.blas_root = root[k];
    r.tri_base = tri_base;
    r.model = k;
    out->insts.push_back(r);
    tri_base += mods[k]->num_tris();
    out->tri_inst.resize(tri_base, (uint32_t)i);
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int corner = 0; corner < 8; ++corner) {
      const double p[3] = {box[6 * k + ((corner & 1) ? 3 : 0)], box[6 * k + 1 + ((corner & 2) ? 3 : 0)],
                           box[6 * k + 2 + ((corner & 4) ? 3 : 0)]};
      for (int row = 0; row < 3; ++row) {
        const double w = (double)m[row] * p[0] + (double)m[4 + row] * p[1] + (double)m[8 + row] * p[2] + m[12 + row];
        lo[row] = std::min(lo[row], w);
        hi[row] = std::max(hi[row], w);
      }
    }
    double ext = 0.0, mag = 0.0;
    for (int a = 0; a < 3; ++a) {
      ext = std::max(ext, hi[a] - lo[a]);
      mag = std::max(mag, std::max(std::fabs(lo[a]), std::fabs(hi[a])));
    }
    const double pad = 1e-4 * ext + 1e-5 * mag;
    for (int a = 0; a < 3; ++a) {
      leaves[9 * i + a] = std::nextafter((float)(lo[a] - pad), -FLT_MAX);
      leaves[9 * i + 3 + a] = std::nextafter((float)(hi[a] + pad), FLT_MAX);
      leaves[9 * i + 6 + a] = leaves[9 * i + a];
    }
  }
  if (inst_model.empty()) return true;
  WideBvh t;
  if (!build_wide_bvh(leaves.data(), (uint32_t)inst_model.size(), max_stack, &t, err)) return false;
  out->tlas_nodes = t.nodes;
  out->tlas_leaves = t.tris;  // v0.w: the instance index (the builder's primitive id)
  out->max_stack = t.stats.max_stack + blas_stack + 1;
  if (out->max_stack > max_stack) {
    *err = "two-level traversal stack of " + std::to_string(out->max_stack) + " entries exceeds " +
           std::to_string(max_stack);
    return false;
  }
  return true;
}

}  // namespace ap
