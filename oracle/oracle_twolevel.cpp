// Oracle (test infrastructure only): closest-hit and any-hit queries over a
// two-level scene, for the parity tests of the library's two-level traversal.
//
// A scene of instances (a model, a 4x4 transform) as the reference builds its
// TLAS over BLAS instances (crates/appearance-path-tracer-gpu/src/
// scene_resources/mod.rs:159-276, TlasInstance with a 4x3 transform): a ray
// meets a model's triangles in object space, its origin and direction mapped
// by the inverse transform (the direction not renormalised, so t is shared
// between the spaces).  Each model has this oracle's binary SAH BVH and
// watertight triangle test (oracle_bvh.cpp); instances are culled with a
// double-precision slab test on a widened world box (a culling aid only: it
// never rejects an instance the ray can hit).  A hit's id is the instance's
// first id (the running sum of the earlier instances' triangle counts) plus
// the model's triangle index; the closest hit is the minimum of (t, id).
// The world-to-object rows are the inverse of the transform by cofactors in
// double, rounded to float: the definition of an instance's transform that
// the library uses too.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <thread>
#include <vector>

#include "oracle_scene.h"
#include "oracle_twolevel.h"

namespace {

struct Inst {
  uint32_t model, tri_base;
  float w2o[12];
  double lo[3], hi[3];
};

struct TwoLevel {
  std::vector<const orc::Scene*> models;
  std::vector<orc::OracleBvh> bvhs;
  std::vector<Inst> insts;
};

void inverse_rows(const float* m, float* w2o) {
  double a[4][4];
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) a[r][c] = m[4 * c + r];
  const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                     a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                     a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  double inv[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int c1 = (c + 1) % 3, c2 = (c + 2) % 3, r1 = (r + 1) % 3, r2 = (r + 2) % 3;
      inv[r][c] = det != 0.0 ? (a[c1][r1] * a[c2][r2] - a[c1][r2] * a[c2][r1]) / det : 0.0;
    }
  for (int r = 0; r < 3; ++r) {
    const double t = -(inv[r][0] * a[0][3] + inv[r][1] * a[1][3] + inv[r][2] * a[2][3]);
    for (int c = 0; c < 3; ++c) w2o[4 * r + c] = (float)inv[r][c];
    w2o[4 * r + 3] = (float)t;
  }
}

void to_object(const Inst& in, orc::V3 o, orc::V3 d, orc::V3* oo, orc::V3* od) {
  const float* m = in.w2o;
  *oo = orc::v3(m[0] * o.x + m[1] * o.y + m[2] * o.z + m[3], m[4] * o.x + m[5] * o.y + m[6] * o.z + m[7],
                m[8] * o.x + m[9] * o.y + m[10] * o.z + m[11]);
  *od = orc::v3(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
                m[8] * d.x + m[9] * d.y + m[10] * d.z);
}

bool box_hit(const Inst& in, orc::V3 o, orc::V3 d, double tmax) {
  double t0 = 0.0, t1 = tmax * (1.0 + 1e-6) + 1e-30;
  const double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
  for (int a = 0; a < 3; ++a) {
    if (dd[a] == 0.0) {
      if (oo[a] < in.lo[a] || oo[a] > in.hi[a]) return false;
      continue;
    }
    double ta = (in.lo[a] - oo[a]) / dd[a], tb = (in.hi[a] - oo[a]) / dd[a];
    if (ta > tb) std::swap(ta, tb);
    t0 = std::max(t0, ta);
    t1 = std::min(t1, tb);
    if (t0 > t1) return false;
  }
  return true;
}

orc::Hit closest(const TwoLevel& s, orc::V3 o, orc::V3 d, float tmax) {
  orc::Hit best{tmax, 0.0f, 0.0f, 0xFFFFFFFFu};
  for (const Inst& in : s.insts) {
    if (!box_hit(in, o, d, best.t)) continue;
    orc::V3 oo, od;
    to_object(in, o, d, &oo, &od);
    const orc::Hit h = s.bvhs[in.model].closest(*s.models[in.model], oo, od, 0.0f, best.t, nullptr, nullptr);
    if (h.tri == 0xFFFFFFFFu) continue;
    const uint32_t gid = in.tri_base + h.tri;
    if (h.t < best.t || gid < best.tri) best = orc::Hit{h.t, h.u, h.v, gid};
  }
  return best;
}

bool any(const TwoLevel& s, orc::V3 o, orc::V3 d, float tmax) {
  for (const Inst& in : s.insts) {
    if (!box_hit(in, o, d, tmax)) continue;
    orc::V3 oo, od;
    to_object(in, o, d, &oo, &od);
    if (s.bvhs[in.model].any(*s.models[in.model], oo, od, 0.0f, tmax)) return true;
  }
  return false;
}

template <class F>
void parallel(uint32_t n, uint32_t threads, F f) {
  std::atomic<uint32_t> next{0};
  auto work = [&]() {
    for (uint32_t i = next.fetch_add(256); i < n; i = next.fetch_add(256))
      for (uint32_t k = i; k < std::min(n, i + 256); ++k) f(k);
  };
  std::vector<std::thread> ts;
  for (uint32_t t = 0; t + 1 < std::max(threads, 1u); ++t) ts.emplace_back(work);
  work();
  for (auto& t : ts) t.join();
}

}  // namespace

namespace orc {
Hit two_level_closest(const void* p, V3 o, V3 d, float tmax) { return closest(*(const TwoLevel*)p, o, d, tmax); }
bool two_level_any(const void* p, V3 o, V3 d, float tmax) { return any(*(const TwoLevel*)p, o, d, tmax); }
}  // namespace orc

extern "C" {

// models: oracle scenes (orc_scene_new) in model space; instance i uses model
// inst_model[i] under the column-major 4x4 inst_m16[16 i ..].
void* orc_two_level_new(void* const* models, uint32_t n_models, const uint32_t* inst_model, const float* inst_m16,
                        uint32_t n_inst) {
  TwoLevel* s = new TwoLevel();
  s->models.assign(reinterpret_cast<const orc::Scene* const*>(models),
                   reinterpret_cast<const orc::Scene* const*>(models) + n_models);
  s->bvhs.resize(n_models);
  std::vector<double> mlo(3 * n_models, DBL_MAX), mhi(3 * n_models, -DBL_MAX);
  for (uint32_t k = 0; k < n_models; ++k) {
    s->bvhs[k].build(*s->models[k]);
    for (const orc::V3& p : s->models[k]->positions) {
      const double q[3] = {p.x, p.y, p.z};
      for (int a = 0; a < 3; ++a) {
        mlo[3 * k + a] = std::min(mlo[3 * k + a], q[a]);
        mhi[3 * k + a] = std::max(mhi[3 * k + a], q[a]);
      }
    }
  }
  uint32_t tri_base = 0;
  for (uint32_t i = 0; i < n_inst; ++i) {
    Inst in;
    in.model = inst_model[i];
    in.tri_base = tri_base;
    tri_base += s->models[in.model]->num_tris();
    const float* m = inst_m16 + 16 * (size_t)i;
    inverse_rows(m, in.w2o);
    for (int a = 0; a < 3; ++a) {
      in.lo[a] = DBL_MAX;
      in.hi[a] = -DBL_MAX;
    }
    for (int corner = 0; corner < 8; ++corner) {
      const double p[3] = {(corner & 1) ? mhi[3 * in.model] : mlo[3 * in.model],
                           (corner & 2) ? mhi[3 * in.model + 1] : mlo[3 * in.model + 1],
                           (corner & 4) ? mhi[3 * in.model + 2] : mlo[3 * in.model + 2]};
      for (int r = 0; r < 3; ++r) {
        const double w = m[r] * p[0] + m[4 + r] * p[1] + m[8 + r] * p[2] + m[12 + r];
        in.lo[r] = std::min(in.lo[r], w);
        in.hi[r] = std::max(in.hi[r], w);
      }
    }
    double ext = 0.0;
    for (int a = 0; a < 3; ++a) ext = std::max(ext, in.hi[a] - in.lo[a]);
    for (int a = 0; a < 3; ++a) {
      const double pad = 1e-3 * ext + 1e-4 * std::max(fabs(in.lo[a]), fabs(in.hi[a]));
      in.lo[a] -= pad;
      in.hi[a] += pad;
    }
    s->insts.push_back(in);
  }
  return s;
}

void orc_two_level_free(void* p) { delete (TwoLevel*)p; }

// out: n x {t, u, v, triangle id} as 32-bit words, as ap_trace_rays writes them.
void orc_two_level_closest(void* p, const float* origins, const float* dirs, uint32_t n, float tmax,
                           uint32_t threads, uint32_t* out) {
  const TwoLevel& s = *(const TwoLevel*)p;
  parallel(n, threads, [&](uint32_t i) {
    const orc::V3 o = orc::v3(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
    const orc::V3 d = orc::v3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    const orc::Hit h = closest(s, o, d, tmax);
    memcpy(out + 4 * (size_t)i, &h.t, 4);
    memcpy(out + 4 * (size_t)i + 1, &h.u, 4);
    memcpy(out + 4 * (size_t)i + 2, &h.v, 4);
    out[4 * (size_t)i + 3] = h.tri;
  });
}

void orc_two_level_any(void* p, const float* origins, const float* dirs, uint32_t n, float tmax, uint32_t threads,
                       uint8_t* out) {
  const TwoLevel& s = *(const TwoLevel*)p;
  parallel(n, threads, [&](uint32_t i) {
    const orc::V3 o = orc::v3(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
    const orc::V3 d = orc::v3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    out[i] = any(s, o, d, tmax) ? 1 : 0;
  });
}

}  // extern "C"
