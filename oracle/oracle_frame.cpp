// Oracle (test infrastructure only): CPU restatement of one frame of the
// reference GPU path tracer (crates/appearance-path-tracer-gpu/src/lib.rs:314-615)
// pass by pass, with the same per-pixel buffers and ping-pong rules, plus a C
// API that the tests, the smoke check and the CPU-baseline leg of bench.py
// load with ctypes.  Nothing in the shipped library calls into this file.
//
// Parity status: the reference (Rust + WGSL on wgpu/Vulkan ray queries) cannot
// be built or run here, so this restatement is pinned only by the reference's
// source text; the CUDA path is checked against it.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <thread>
#include <vector>

#include "oracle_shading.h"

namespace orc {

struct FrameConfig {  // same field order as ap_frame_config in include/appearance_cuda.h
  uint32_t max_bounces, sample_count;
  uint32_t restir_di, restir_gi, svgf, firefly_filter, taa;
  uint32_t di_area_samples, di_bsdf_samples;
  float di_temporal_m_factor;
  uint32_t di_spatial_passes, di_spatial_samples, di_unbiased;
  float gi_temporal_m_cap;
  uint32_t gi_spatial_passes, gi_spatial_samples, gi_unbiased;
  uint32_t svgf_max_history, svgf_atrous_passes;
  float taa_history_influence;
  uint32_t threads;
};

struct RayRec { V3 o; uint32_t d; };
struct Payload { uint32_t throughput, rng; float t; };
struct GTexel { V3 pos; float depth; uint32_t n; uint32_t albedo; };
struct GT { V3 pos; float depth; V3 n; V3 albedo; };

inline GT gt_unpack(const GTexel& g) {
  return GT{g.pos, g.depth, oct30_unpack(g.n), rgb9e5_unpack(g.albedo)};
}
inline GTexel gt_pack(V3 p, float d, V3 n, V3 a) { return GTexel{p, d, oct30_pack(n), rgb9e5_pack(a)}; }
inline bool gt_is_sky(float depth) { return depth == 0.0f; }
inline float depth_cs(float depth_ws, float zn, float zf) {
  float zl = (depth_ws - zn) / zf;
  return (zn * zf) / (zf - zl * (zf - zn));
}

template <class F>
void parallel_rows(uint32_t H, uint32_t threads, F f) {
  if (threads <= 1) {
    for (uint32_t y = 0; y < H; ++y) f(y);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> ts;
  for (uint32_t t = 0; t < threads; ++t)
    ts.emplace_back([&]() {
      for (uint32_t y = next.fetch_add(1); y < H; y = next.fetch_add(1)) f(y);
    });
  for (auto& t : ts) t.join();
}

struct Frame {
  const Scene* scene;
  OracleBvh bvh;
  FrameConfig cfg;
  uint32_t W, H, frame_idx = 0;
  float mats[4][16];  // inv_view, inv_proj, view_proj, prev_view_proj (column-major)
  std::vector<RayRec> rays;
  std::vector<Payload> payloads;
  std::vector<uint32_t> radiance;
  std::vector<DiRes> di, di_inter, di_prev[2];
  std::vector<Ctx> ctx;
  std::vector<GiRes> gi, gi_inter, gi_prev[2];
  std::vector<GTexel> gbuf[2];
  std::vector<V2> velocity;
  std::vector<uint32_t> demod[2];
  std::vector<uint32_t> svgf_rad[2];
  std::vector<V2> svgf_mom[2];
  std::vector<float> svgf_var[2];
  std::vector<uint32_t> svgf_count, svgf_hist;
  uint64_t rays_cast = 0;

  Frame(const Scene* s, uint32_t w, uint32_t h, const FrameConfig& c) : scene(s), cfg(c), W(w), H(h) {
    bvh.build(*s);
    size_t P = (size_t)w * h;
    rays.assign(P, RayRec{v3s(0), 0});
    payloads.assign(P, Payload{0, 0, 0.0f});
    radiance.assign(P, 0);
    DiRes dz{0, 0, 0, 0, LightSample{{0, 0}, 0, 0}};
    di.assign(P, dz); di_inter.assign(P, dz); di_prev[0].assign(P, dz); di_prev[1].assign(P, dz);
    ctx.assign(P, Ctx{0, 0, 0, 0});
    GiRes gz = gi_new();
    gi.assign(P, gz); gi_inter.assign(P, gz); gi_prev[0].assign(P, gz); gi_prev[1].assign(P, gz);
    GTexel g0{v3s(0), 0.0f, 0, 0};
    gbuf[0].assign(P, g0); gbuf[1].assign(P, g0);
    velocity.assign(P, V2{0, 0});
    for (int i = 0; i < 2; ++i) {
      demod[i].assign(P, 0); svgf_rad[i].assign(P, 0); svgf_mom[i].assign(P, V2{0, 0});
      svgf_var[i].assign(P, 0.0f);
    }
    svgf_count.assign(P, 0); svgf_hist.assign(P, 0);
  }

  std::vector<GTexel>& gb() { return gbuf[frame_idx % 2]; }
  std::vector<GTexel>& prev_gb() { return gbuf[(frame_idx + 1) % 2]; }

  // ---- traversal wrappers (helpers/trace.wgsl:7-84) ----
  Hit closest(V3 o, V3 d, float tmax) { return bvh.closest(*scene, o, d, 0.0f, tmax, nullptr, nullptr); }
  bool shadow(V3 origin, V3 dir, float dist, V3 n) {
    V3 o = origin + n * 1e-4f;
    return !bvh.any(*scene, o, dir, 0.0f, dist - 1e-4f * 2.0f);
  }

  // hit attribute fetch shared by trace.wgsl:101-201 and inline_path_tracer.wgsl:69-168
  struct Surface {
    uint32_t material_idx;
    Material mat;
    V3 hit_point, n;  // front-facing shading normal
    bool back_face;
    ShadeFrame frame;
    bool has_cc;
  };
  Surface surface(const Hit& h, V3 origin, V3 direction) {
    Surface s;
    const Scene& sc = *scene;
    uint32_t inst_idx = sc.tri_instance[h.tri];
    const Instance& in = sc.instances[inst_idx];
    uint32_t prim = h.tri - in.first_global_tri;
    float bx = 1.0f - h.u - h.v;
    uint32_t i0 = sc.indices[in.first_index + prim * 3 + 0];
    uint32_t i1 = sc.indices[in.first_index + prim * 3 + 1];
    uint32_t i2 = sc.indices[in.first_index + prim * 3 + 2];
    V3 n0 = oct30_unpack(sc.normals[in.first_vertex + i0]);
    V3 n1 = oct30_unpack(sc.normals[in.first_vertex + i1]);
    V3 n2 = oct30_unpack(sc.normals[in.first_vertex + i2]);
    s.material_idx = in.material_idx + sc.tri_material[in.first_index / 3 + prim];
    s.mat = sc.materials[s.material_idx];
    V3 normal = n0 * bx + n1 * h.u + n2 * h.v;
    V3 hit_n = normalize(normal);
    s.hit_point = origin + direction * h.t;
    V3 ff_n = hit_n, ff_sn = hit_n;
    V3 w_out = -direction;
    s.back_face = dot(w_out, hit_n) < 0.0f;
    if (s.back_face) { ff_n = ff_n * -1.0f; ff_sn = ff_sn * -1.0f; }
    s.n = ff_sn;
    s.frame.n = ff_sn;
    s.frame.t2w = onb(ff_sn);
    s.has_cc = s.mat.clearcoat > 0.0f;
    s.frame.cc_t2w = s.has_cc ? onb(ff_n) : zero_m3();
    return s;
  }

  // ---- helpers/nee.wgsl:122-237 ----
  DiRes sample_ris(V3 hit, V3 wo, const ShadeFrame& fr, const Bsdf& b, float t, bool back_face,
                   uint32_t& rng) {
    const uint32_t NA = cfg.di_area_samples, NB = cfg.di_bsdf_samples;
    DiRes res = di_new();
    LightEval sel{v3s(0), v3s(0)};
    uint32_t n_iter = std::max(NA, NB);
    for (uint32_t i = 0; i < n_iter; ++i) {
      float area_pdf = 0.0f;
      LightSample area_sample{{0, 0}, 0, 0};
      LightEval area_eval{v3s(0), v3s(0)};
      float area_phat = 0.0f;
      if (i < NA) {
        float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng);
        float r3 = rnd(rng), r4 = rnd(rng);
        area_sample = sample_uniform(*scene, r0, r1, r2, V2{r3, r4}, &area_pdf);
        area_eval = load_eval_data(*scene, area_sample, hit);
        V3 wi = normalize(area_eval.point - hit);
        float wdn = dot(wi, fr.n);
        if (wdn > 0.0f && area_pdf > 0.0f) {
          float spdf = 0.0f;
          V3 refl = disney_evaluate(b, fr, wo, wi, &spdf);
          if (spdf > 0.0f) area_phat = luma(refl * wdn * area_eval.emission);
        }
      }
      float bsdf_pdf = 0.0f;
      LightSample bsdf_sample = ls_empty();
      LightEval bsdf_eval{v3s(0), v3s(0)};
      float bsdf_phat = 0.0f;
      if (i < NB) {
        V3 wi = v3s(0);
        bool spec = false;
        float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng);
        V3 refl = disney_sample(b, fr, wo, t, back_face, r0, r1, r2, &wi, &bsdf_pdf, &spec);
        float wdn = dm::fabs_(dot(wi, fr.n));
        V3 contribution = wdn * refl;
        if (dot(contribution, contribution) > 0.0f) {
          Hit h = closest(hit + fr.n * 1e-4f, wi, 1000.0f);
          ++rays_cast;
          if (h.tri != 0xFFFFFFFFu) {
            const Instance& in = scene->instances[scene->tri_instance[h.tri]];
            if (in.emissive_idx != U32_MAX)
              bsdf_sample = LightSample{{h.u, h.v}, in.emissive_idx, h.tri - in.first_global_tri};
          } else {
            bsdf_sample = ls_sun(inverse_direction_to_sun(*scene, wi));
          }
          if (!ls_is_empty(bsdf_sample)) {
            bsdf_eval = load_eval_data(*scene, bsdf_sample, hit);
            bsdf_phat = luma(contribution * bsdf_eval.emission);
          }
        }
      }
      if (i < NA) {
        float aw = 0.0f;
        if (area_pdf > 0.0f) {
          float mis = area_pdf / ((float)NA * area_pdf + (float)NB * bsdf_pdf);
          aw = mis * area_phat * (1.0f / dm::fmax(area_pdf, 1e-8f));
        }
        if (di_update(res, aw, rng, area_sample, area_phat)) sel = area_eval;
      }
      if (i < NB) {
        float bw = 0.0f;
        if (bsdf_pdf > 0.0f) {
          float mis = bsdf_pdf / ((float)NB * bsdf_pdf + (float)NA * area_pdf);
          bw = mis * bsdf_phat * (1.0f / dm::fmax(bsdf_pdf, 1e-8f));
        }
        if (di_update(res, bw, rng, bsdf_sample, bsdf_phat)) sel = bsdf_eval;
      }
    }
    if (res.phat > 1e-6f) {
      V3 dir = normalize(sel.point - hit);
      float dist = distance(sel.point, hit);
      ++rays_cast;
      if (shadow(hit, dir, dist, fr.n)) res.W = (1.0f / res.phat) * res.wsum;
    }
    return res;
  }

  // ---- helpers/inline_path_tracer.wgsl:51-256 with the approx() config ----
  V3 inline_trace(V3 origin, V3 direction, V3& throughput, V3& first_hit, uint32_t& rng) {
    V3 acc = v3s(0);
    Hit h = closest(origin + direction * 1e-4f, direction, 1000.0f - 1e-4f * 2.0f);
    ++rays_cast;
    if (h.tri != 0xFFFFFFFFu) {
      Surface s = surface(h, origin, direction);
      Bsdf b = bsdf_from_material(s.mat);
      V3 wo = -direction;
      float pdf = 0.0f;
      float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng), r3 = rnd(rng), r4 = rnd(rng);
      LightSample ls = sample_uniform(*scene, r0, r1, r2, V2{r3, r4}, &pdf);
      DiRes dr{1.0f, 1.0f / pdf, 1.0f, 1.0f, ls};
      if (dr.W > 0.0f) {
        LightEval ev = load_eval_data(*scene, ls, s.hit_point);
        V3 sdir = normalize(ev.point - s.hit_point);
        float sdist = distance(ev.point, s.hit_point);
        float ndl = dot(sdir, s.n);
        if (ndl > 0.0f) {
          ++rays_cast;
          if (shadow(s.hit_point, sdir, sdist, s.n)) {
            float spdf = 0.0f;
            V3 refl = disney_evaluate(b, s.frame, wo, sdir, &spdf);
            acc = acc + throughput * refl * ev.emission * ndl * dr.W;
          }
        }
      }
      first_hit = s.hit_point;
      return acc;
    }
    first_hit = origin + direction * 1000.0f;
    acc = acc + throughput * sky_radiance(*scene, direction, true);
    return acc;
  }

  GiRes gi_sample_ris(V3 hit, V3 wo, const ShadeFrame& fr, const Bsdf& b, V3 throughput, float t,
                      bool back_face, uint32_t& rng) {
    GiRes res = gi_new();
    V3 wi = v3s(0);
    float pdf = 0.0f;
    bool spec = false;
    float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng);
    V3 refl = disney_sample(b, fr, wo, t, back_face, r0, r1, r2, &wi, &pdf, &spec);
    if (pdf > 1e-6f) {
      float cos_in = dm::fabs_(dot(wi, fr.n));
      V3 local = cos_in * refl;
      V3 tr = throughput * local;
      uint32_t phat_rng = rng;
      V3 point = v3s(0);
      V3 contribution = inline_trace(hit, wi, tr, point, rng);
      float phat = luma(contribution);
      float w = phat / pdf;
      gi_update(res, w, rng, point, phat, phat_rng);
    }
    if (res.phat > 0.0f && res.M * res.wsum > 0.0f)
      res.W = (1.0f / res.phat) * (1.0f / res.M * res.wsum);
    return res;
  }

  // GiReservoir::phat (inline_path_tracer.wgsl:299-331)
  float gi_phat(const GiRes& r, const Ctx& c, V3 throughput, V3 hit, V3 wo) {
    const Material& m = scene->materials[c.material_idx];
    Bsdf b = bsdf_from_material(m);
    ShadeFrame fr;
    fr.n = oct30_unpack(c.n);
    fr.t2w = onb(fr.n);
    fr.cc_t2w = onb(oct30_unpack(c.n_cc));
    V3 wi = normalize(r.point - hit);
    float spdf = 0.0f;
    V3 refl = disney_evaluate(b, fr, wo, wi, &spdf);
    float cos_in = dm::fabs_(dot(wi, fr.n));
    V3 local = cos_in * refl;
    V3 gi_origin = hit + wi * 0.0001f;
    V3 tr = throughput * local;
    uint32_t prng = r.phat_rng;
    V3 pt = v3s(0);
    V3 contribution = inline_trace(gi_origin, wi, tr, pt, prng);
    return luma(contribution);
  }

  // LightSample::phat (di_reservoir.wgsl:58-97)
  float ls_phat(const LightSample& l, const Ctx& c, V3 hit, V3 wo, bool vis) {
    LightEval ev = load_eval_data(*scene, l, hit);
    const Material& m = scene->materials[c.material_idx];
    Bsdf b = bsdf_from_material(m);
    ShadeFrame fr;
    fr.n = oct30_unpack(c.n);
    fr.t2w = onb(fr.n);
    fr.cc_t2w = onb(oct30_unpack(c.n_cc));
    V3 wi = normalize(ev.point - hit);
    float wdn = dot(wi, fr.n);
    if (wdn > 0.0f) {
      bool visible = true;
      if (vis) {
        float dist = distance(ev.point, hit);
        ++rays_cast;
        visible = shadow(hit, wi, dist, fr.n);
      }
      if (visible) {
        float spdf = 0.0f;
        V3 refl = disney_evaluate(b, fr, wo, wi, &spdf);
        return luma(refl * wdn * ev.emission);
      }
    }
    return 0.0f;
  }

  DiRes di_combine(const DiRes& r1, const DiRes& r2, uint32_t& rng) {
    DiRes c = di_new();
    di_update(c, r1.phat * r1.W * r1.M, rng, r1.sample, r1.phat);
    di_update(c, r2.phat * r2.W * r2.M, rng, r2.sample, r2.phat);
    c.M = r1.M + r2.M;
    if (c.phat > 1e-6f && c.M * c.wsum > 1e-6f) c.W = (1.0f / c.phat) * (1.0f / c.M * c.wsum);
    return c;
  }
  DiRes di_combine_unbiased(const DiRes& r1, V3 h1, const Ctx& c1, V3 wo1, const DiRes& r2, V3 h2,
                            const Ctx& c2, V3 wo2, uint32_t& rng) {
    DiRes c = di_new();
    di_update(c, r1.phat * r1.W * r1.M, rng, r1.sample, r1.phat);
    di_update(c, r2.phat * r2.W * r2.M, rng, r2.sample, r2.phat);
    c.M = r1.M + r2.M;
    float z = 0.0f;
    if (ls_phat(c.sample, c1, h1, wo1, true) > 0.0f) z = z + r1.M;
    if (ls_phat(c.sample, c2, h2, wo2, true) > 0.0f) z = z + r2.M;
    if (c.phat > 1e-6f && z * c.wsum > 1e-6f) c.W = (1.0f / c.phat) * (1.0f / z * c.wsum);
    return c;
  }
  GiRes gi_combine(const GiRes& r1, const GiRes& r2, uint32_t& rng) {
    GiRes c = gi_new();
    gi_update(c, r1.phat * r1.W * r1.M, rng, r1.point, r1.phat, r1.phat_rng);
    gi_update(c, r2.phat * r2.W * r2.M, rng, r2.point, r2.phat, r2.phat_rng);
    c.M = r1.M + r2.M;
    if (c.phat > 0.0f && c.M * c.wsum > 0.0f) c.W = (1.0f / c.phat) * (1.0f / c.M * c.wsum);
    return c;
  }
  GiRes gi_combine_unbiased(const GiRes& r1, V3 h1, const Ctx& c1, V3 wo1, V3 t1, const GiRes& r2,
                            V3 h2, const Ctx& c2, V3 wo2, V3 t2, uint32_t& rng) {
    GiRes c = gi_new();
    gi_update(c, r1.phat * r1.W * r1.M, rng, r1.point, r1.phat, r1.phat_rng);
    gi_update(c, r2.phat * r2.W * r2.M, rng, r2.point, r2.phat, r2.phat_rng);
    c.M = r1.M + r2.M;
    float z = 0.0f;
    if (gi_phat(c, c1, t1, h1, wo1) > 0.0f) z = z + r1.M;
    if (gi_phat(c, c2, t2, h2, wo2) > 0.0f) z = z + r2.M;
    if (c.phat > 0.0f && z * c.wsum > 0.0f) c.W = (1.0f / c.phat) * (1.0f / z * c.wsum);
    return c;
  }

  // ---- mat4 helpers ----
  static void mul4(const float* m, const float v[4], float out[4]) {
    for (int r = 0; r < 4; ++r)
      out[r] = m[0 * 4 + r] * v[0] + m[1 * 4 + r] * v[1] + m[2 * 4 + r] * v[2] + m[3 * 4 + r] * v[3];
  }

  // ---- raygen.wgsl:21-39 ----
  void raygen() {
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        float pcx = (float)x + 0.5f, pcy = (float)y + 0.5f;
        float ux = (pcx / (float)W) * 2.0f - 1.0f;
        float uy = (pcy / (float)H) * 2.0f - 1.0f;
        uy = -uy;
        float o4[4] = {0, 0, 0, 1}, origin[4], t4[4] = {ux, uy, 1.0f, 1.0f}, target[4];
        mul4(mats[0], o4, origin);
        mul4(mats[1], t4, target);
        V3 tn = normalize(v3(target[0], target[1], target[2]));
        float d4[4] = {tn.x, tn.y, tn.z, 0.0f}, dir[4];
        mul4(mats[0], d4, dir);
        rays[(size_t)y * W + x] = RayRec{v3(origin[0], origin[1], origin[2]), oct30_pack(v3(dir[0], dir[1], dir[2]))};
      }
    });
  }

  // screen-space motion of the primary hit point (gbuffer.wgsl:44-53)
  V2 velocity_of(V3 p) {
    float p4[4] = {p.x, p.y, p.z, 1.0f}, cs[4], pcs[4];
    mul4(mats[2], p4, cs);
    mul4(mats[3], p4, pcs);
    float px = (pcs[0] / pcs[3] + 1.0f) / 2.0f, py = 1.0f - (pcs[1] / pcs[3] + 1.0f) / 2.0f;
    float cx = (cs[0] / cs[3] + 1.0f) / 2.0f, cy = 1.0f - (cs[1] / cs[3] + 1.0f) / 2.0f;
    return V2{cx - px, cy - py};
  }

  // ---- trace.wgsl:62-262 ----
  void trace(uint32_t bounce, uint32_t seed) {
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        RayRec ray = rays[id];
        V3 origin = ray.o;
        V3 direction = oct30_unpack(ray.d);
        Payload pl = payloads[id];
        if (bounce == 0) {
          pl.throughput = rgb9e5_pack(v3s(1.0f));
          pl.rng = pcg_hash(id ^ xor_shift(seed));
          pl.t = 0.0f;
        }
        if (pl.t < 0.0f) continue;
        V3 acc = rgb9e5_unpack(radiance[id]);
        V3 T = rgb9e5_unpack(pl.throughput);
        uint32_t rng = pl.rng;
        V3 g_pos = v3s(0), g_n = v3s(0), g_alb = v3s(0);
        float g_depth = 0.0f;
        V2 vel{0.0f, 0.0f};
        float depth_ws = 0.0f;
        Hit h = closest(origin + direction * 1e-4f, direction, 1000.0f);
        if (h.tri != 0xFFFFFFFFu) {
          depth_ws = depth_ws + h.t;
          Surface s = surface(h, origin, direction);
          V3 emission = mv3(s.mat.emission);
          if (bounce == 0) acc = acc + T * emission;
          V3 wo = -direction;
          Bsdf b = bsdf_from_material(s.mat);
          if (bounce == 0) {
            g_pos = s.hit_point;
            g_depth = depth_ws;
            g_n = s.n;
            g_alb = mv3(s.mat.color) + emission;
            vel = velocity_of(s.hit_point);
          }
          DiRes dr = sample_ris(s.hit_point, wo, s.frame, b, h.t, s.back_face, rng);
          di[id] = dr;
          ctx[id] = Ctx{s.material_idx, rgb9e5_pack(T), oct30_pack(s.n), oct30_pack(s.frame.cc_t2w.c2)};
          pl.t = depth_ws;
          bool killed = false;
          if (bounce + 1 < cfg.max_bounces) {
            if (bounce > 1) {
              float rr = dm::fmax(T.x, dm::fmax(T.y, T.z));
              if (rr < rnd(rng)) {
                pl.t = -1.0f;
                killed = true;
              } else {
                T = T * (1.0f / rr);
              }
            }
            if (!killed) gi[id] = gi_sample_ris(s.hit_point, wo, s.frame, b, T, h.t, s.back_face, rng);
          }
        } else {
          g_alb = v3s(1.0f);
          acc = acc + T * sky_radiance(*scene, direction, true);
          pl.t = -1.0f;
        }
        radiance[id] = rgb9e5_pack(acc);
        pl.throughput = rgb9e5_pack(T);
        pl.rng = rng;
        payloads[id] = pl;
        if (bounce == 0) {
          gbw[id] = gt_pack(g_pos, g_depth, g_n, g_alb);
          velocity[id] = vel;
        }
      }
    });
  }

  // ---- apply_di.wgsl:48-111 ----
  void apply_di() {
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        RayRec ray = rays[id];
        V3 origin = ray.o, direction = oct30_unpack(ray.d);
        Payload pl = payloads[id];
        if (pl.t < 0.0f) continue;
        DiRes dr = di[id];
        if (dr.W == 0.0f) continue;
        Ctx c = ctx[id];
        V3 acc = rgb9e5_unpack(radiance[id]);
        V3 T = rgb9e5_unpack(c.throughput);
        const Material& m = scene->materials[c.material_idx];
        Bsdf b = bsdf_from_material(m);
        V3 hit = origin + direction * pl.t;
        ShadeFrame fr;
        fr.n = oct30_unpack(c.n);
        fr.t2w = onb(fr.n);
        LightEval ev = load_eval_data(*scene, dr.sample, hit);
        fr.cc_t2w = onb(oct30_unpack(c.n_cc));
        V3 sdir = normalize(ev.point - hit);
        float sdist = distance(ev.point, hit);
        float ndl = dot(sdir, fr.n);
        if (ndl > 0.0f) {
          if (shadow(hit, sdir, sdist, fr.n)) {
            V3 wo = -direction;
            float spdf = 0.0f;
            V3 refl = disney_evaluate(b, fr, wo, sdir, &spdf);
            V3 contribution = T * refl * ev.emission * ndl * dr.W;
            acc = acc + contribution;
          }
        }
        radiance[id] = rgb9e5_pack(acc);
      }
    });
  }

  // ---- apply_gi.wgsl:44-99 ----
  void apply_gi() {
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        RayRec ray = rays[id];
        V3 origin = ray.o, direction = oct30_unpack(ray.d);
        Payload pl = payloads[id];
        if (pl.t < 0.0f) continue;
        V3 hit = origin + direction * pl.t;
        GiRes gr = gi[id];
        if (gr.W > 0.0f) {
          Ctx c = ctx[id];
          V3 T = rgb9e5_unpack(pl.throughput);
          const Material& m = scene->materials[c.material_idx];
          Bsdf b = bsdf_from_material(m);
          ShadeFrame fr;
          fr.n = oct30_unpack(c.n);
          fr.t2w = onb(fr.n);
          fr.cc_t2w = onb(oct30_unpack(c.n_cc));
          V3 wo = -direction;
          V3 wi = normalize(gr.point - hit);
          float spdf = 0.0f;
          V3 refl = disney_evaluate(b, fr, wo, wi, &spdf);
          float cos_in = dm::fabs_(dot(fr.n, wi));
          V3 contribution = refl * cos_in * gr.W;
          T = T * contribution;
          pl.throughput = rgb9e5_pack(T);
          rays[id] = RayRec{hit, oct30_pack(wi)};
        } else {
          pl.t = -1.0f;
        }
        payloads[id] = pl;
      }
    });
  }

  // bilinear previous-frame G-buffer (gbuffer_bindings.wgsl:20-50)
  GT sample_prev_gbuffer(V2 pos) {
    std::vector<GTexel>& pg = prev_gb();
    uint32_t ix = dm::f2u(dm::floor_(pos.x)), iy = dm::f2u(dm::floor_(pos.y));
    float fx = dm::fract(pos.x), fy = dm::fract(pos.y);
    uint32_t x1 = std::min(ix + 1, W - 1), y1 = std::min(iy + 1, H - 1);
    GT t00 = gt_unpack(pg[iy * W + ix]), t10 = gt_unpack(pg[iy * W + x1]);
    GT t01 = gt_unpack(pg[y1 * W + ix]), t11 = gt_unpack(pg[y1 * W + x1]);
    V3 p0 = mix3(t00.pos, t10.pos, fx), p1 = mix3(t01.pos, t11.pos, fx);
    float d0 = mixf(t00.depth, t10.depth, fx), d1 = mixf(t01.depth, t11.depth, fx);
    V3 n0 = mix3(t00.n, t10.n, fx), n1 = mix3(t01.n, t11.n, fx);
    V3 a0 = mix3(t00.albedo, t10.albedo, fx), a1 = mix3(t01.albedo, t11.albedo, fx);
    return GT{mix3(p0, p1, fy), mixf(d0, d1, fy), normalize(mix3(n0, n1, fy)), mix3(a0, a1, fy)};
  }
  static bool history_valid(const GT& cur, const GT& prev) {  // GBufferTexel::is_disoccluded
    bool ds = dm::fabs_(cur.depth - prev.depth) <= 0.1f * prev.depth;
    bool ns = dot(cur.n, prev.n) > 0.906f;
    return ds && ns;
  }
  bool prev_point(uint32_t x, uint32_t y, V2* out) {
    V2 v = velocity[y * W + x];
    float px = (float)x - ((float)W * v.x), py = (float)y - ((float)H * v.y);
    *out = V2{px, py};
    return px >= 0.0f && py >= 0.0f && px <= (float)(W - 1) && py <= (float)(H - 1);
  }
  uint32_t stochastic_prev_id(V2 p, float r0, float r1) {
    uint32_t px = dm::f2u(dm::floor_(p.x + r0)), py = dm::f2u(dm::floor_(p.y + r1));
    uint64_t id = (uint64_t)py * W + px;
    return (uint32_t)std::min<uint64_t>(id, (uint64_t)W * H - 1);
  }

  // ---- restir_di_temporal.wgsl:68-176 (BILINEAR = false) ----
  void di_temporal(std::vector<DiRes>& in, std::vector<DiRes>& out, std::vector<DiRes>& prev_in,
                   std::vector<DiRes>& prev_out) {
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        RayRec ray = rays[id];
        V3 origin = ray.o, direction = oct30_unpack(ray.d);
        Payload pl = payloads[id];
        if (pl.t < 0.0f) continue;
        uint32_t rng = pl.rng;
        V3 hit = origin + direction * pl.t;
        Ctx c = ctx[id];
        DiRes r = in[id];
        V2 pp;
        if (prev_point(x, y, &pp)) {
          GT cur = gt_unpack(gbw[id]);
          GT prv = sample_prev_gbuffer(pp);
          if (history_valid(cur, prv)) {
            float r0 = rnd(rng), r1 = rnd(rng);
            uint32_t pid = stochastic_prev_id(pp, r0, r1);
            DiRes pr = prev_in[pid];
            pr.M = dm::fmin(pr.M, cfg.di_temporal_m_factor * r.M);
            pr.phat = ls_phat(pr.sample, c, hit, -direction, cfg.di_unbiased > 0);
            r = di_combine(r, pr, rng);
          }
        }
        out[id] = r;
        if (cfg.di_spatial_passes == 0) prev_out[id] = r;
        pl.rng = rng;
        payloads[id] = pl;
      }
    });
  }

  static uint32_t mirror(int32_t x, int32_t mx) {
    int32_t v = ((x + mx) % (2 * mx)) - mx;
    return (uint32_t)(v < 0 ? -v : v);
  }
  static float ign_animated(uint32_t px, uint32_t py, uint32_t frame) {
    uint32_t fid = frame % 64;
    float x = (float)px + 5.588238f * (float)fid;
    float y = (float)py + 5.588238f * (float)fid;
    return dm::fract(52.9829189f * dm::fract(0.06711056f * x + 0.00583715f * y));
  }

  // ---- restir_di_spatial.wgsl:70-163 and restir_gi_spatial.wgsl:71-166 ----
  template <bool GI>
  void spatial(uint32_t pass_idx, uint32_t pass_count, uint32_t seed, uint32_t nsamples,
               bool unbiased, void* in_v, void* out_v, void* prev_v) {
    std::vector<GTexel>& gbw = gb();
    const float GOLDEN_ANGLE = 2.39996322972865332f;
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        RayRec ray = rays[id];
        V3 origin = ray.o, direction = oct30_unpack(ray.d);
        Payload pl = payloads[id];
        if (pl.t < 0.0f) continue;
        uint32_t rng = pl.rng;
        V3 T = rgb9e5_unpack(pl.throughput);
        V3 hit = origin + direction * pl.t;
        Ctx c = ctx[id];
        const GTexel& cg = gbw[id];
        float cdepth = depth_cs(cg.depth, 0.001f, 10000.0f);
        V3 cn = oct30_unpack(cg.n);
        float radius = (float)(W + H) / 2.0f * 0.05f;
        uint32_t frame_arg = GI ? seed * 3 + pass_idx : seed * pass_count + pass_idx;
        float roff = ign_animated(x, y, frame_arg);
        uint32_t psx = pass_idx == 0 ? (x >> 2) : (x >> 1);
        uint32_t psy = pass_idx == 0 ? (y >> 2) : (y >> 1);
        uint32_t aseed = hash_combine(psx, hash_combine(psy, frame_arg));
        float aoff = (float)aseed * (1.0f / 4294967296.0f) * TWO_PI;
        DiRes rdi = GI ? di_new() : ((std::vector<DiRes>*)in_v)->at(id);
        GiRes rgi = GI ? ((std::vector<GiRes>*)in_v)->at(id) : gi_new();
        for (uint32_t i = 0; i < nsamples; ++i) {
          float angle = (float)i * GOLDEN_ANGLE + aoff;
          float cur_r = dm::pow_((float)i / (float)nsamples, 0.5f) * radius + roff;
          float sa, ca;
          dm::sincos_(angle, &sa, &ca);
          int32_t ox = dm::f2i(cur_r * ca), oy = dm::f2i(cur_r * sa);
          uint32_t nx = std::min(mirror((int32_t)x + ox, (int32_t)W), W - 1);
          uint32_t ny = std::min(mirror((int32_t)y + oy, (int32_t)H), H - 1);
          uint32_t nid = ny * W + nx;
          if (nid == id) continue;
          bool valid = true;
          const GTexel& ng = gbw[nid];
          if (gt_is_sky(ng.depth)) {
            valid = false;
          } else {
            float nd = depth_cs(ng.depth, 0.001f, 10000.0f);
            bool vd = (dm::fabs_(cdepth - nd) / cdepth) < 0.1f;
            bool vn = dot(cn, oct30_unpack(ng.n)) > 0.906f;
            valid = vd && vn;
          }
          if (valid) {
            V3 wo = -direction;
            if (!GI) {
              DiRes nr = ((std::vector<DiRes>*)in_v)->at(nid);
              nr.phat = ls_phat(nr.sample, c, hit, wo, unbiased);
              valid = nr.phat > 0.0f;
              if (!unbiased) {
                rdi = di_combine(rdi, nr, rng);
              } else {
                V3 nwo = -oct30_unpack(rays[nid].d);
                rdi = di_combine_unbiased(rdi, hit, c, wo, nr, ng.pos, ctx[nid], nwo, rng);
              }
            } else {
              GiRes nr = ((std::vector<GiRes>*)in_v)->at(nid);
              nr.phat = gi_phat(nr, c, T, hit, wo);
              valid = nr.phat > 0.0f;
              if (!unbiased) {
                rgi = gi_combine(rgi, nr, rng);
              } else {
                V3 nwo = -oct30_unpack(rays[nid].d);
                V3 nT = rgb9e5_unpack(payloads[nid].throughput);
                rgi = gi_combine_unbiased(rgi, hit, c, wo, T, nr, ng.pos, ctx[nid], nwo, nT, rng);
              }
            }
          }
          if (!valid) radius = dm::fmax(radius * 0.5f, 3.0f);
        }
        if (!GI) {
          ((std::vector<DiRes>*)out_v)->at(id) = rdi;
          if (pass_idx == pass_count - 1) ((std::vector<DiRes>*)prev_v)->at(id) = rdi;
        } else {
          ((std::vector<GiRes>*)out_v)->at(id) = rgi;
          if (pass_idx == pass_count - 1) ((std::vector<GiRes>*)prev_v)->at(id) = rgi;
        }
        pl.rng = rng;
        payloads[id] = pl;
      }
    });
  }

  // ---- restir_gi_temporal.wgsl:67-116 ----
  void gi_temporal(std::vector<GiRes>& in, std::vector<GiRes>& out, std::vector<GiRes>& prev_in,
                   std::vector<GiRes>& prev_out) {
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        RayRec ray = rays[id];
        V3 origin = ray.o, direction = oct30_unpack(ray.d);
        Payload pl = payloads[id];
        if (pl.t < 0.0f) continue;
        uint32_t rng = pl.rng;
        V3 T = rgb9e5_unpack(pl.throughput);
        V3 hit = origin + direction * pl.t;
        Ctx c = ctx[id];
        GiRes r = in[id];
        V2 pp;
        if (prev_point(x, y, &pp)) {
          float r0 = rnd(rng), r1 = rnd(rng);
          uint32_t pid = stochastic_prev_id(pp, r0, r1);
          GT cur = gt_unpack(gbw[id]);
          GT prv = sample_prev_gbuffer(pp);
          if (history_valid(cur, prv)) {
            GiRes pr = prev_in[pid];
            pr.M = dm::fmin(pr.M, cfg.gi_temporal_m_cap);
            pr.phat = gi_phat(pr, c, T, hit, -direction);
            r = gi_combine(r, pr, rng);
          }
        }
        out[id] = r;
        if (cfg.gi_spatial_passes == 0) prev_out[id] = r;
        pl.rng = rng;
        payloads[id] = pl;
      }
    });
  }

  // restir_di_pass.rs:125-590 buffer wiring
  void restir_di(uint32_t seed) {
    std::vector<DiRes>& prev_in = di_prev[frame_idx % 2];
    std::vector<DiRes>& prev_out = di_prev[(frame_idx + 1) % 2];
    di_temporal(di, di_inter, prev_in, prev_out);
    uint32_t n = cfg.di_spatial_passes;
    for (uint32_t i = 0; i < n; ++i) {
      std::vector<DiRes>& in = (i % 2 != 0) ? di : di_inter;
      std::vector<DiRes>& out = (i % 2 == 0) ? di : di_inter;
      spatial<false>(i, n, seed, cfg.di_spatial_samples, cfg.di_unbiased > 0, &in, &out, &prev_out);
    }
    if (n % 2 == 0) di = di_inter;
  }
  // restir_gi_pass.rs:111-586 buffer wiring
  void restir_gi(uint32_t seed) {
    std::vector<GiRes>& prev_in = gi_prev[frame_idx % 2];
    std::vector<GiRes>& prev_out = gi_prev[(frame_idx + 1) % 2];
    gi_temporal(gi, gi_inter, prev_in, prev_out);
    uint32_t n = cfg.gi_spatial_passes;
    if (n == 0) gi = gi_inter;
    for (uint32_t i = 0; i < n; ++i) {
      std::vector<GiRes>& in = (i % 2 != 0) ? gi : gi_inter;
      std::vector<GiRes>& out = (i % 2 == 0) ? gi : gi_inter;
      spatial<true>(i, n, seed, cfg.gi_spatial_samples, cfg.gi_unbiased > 0, &in, &out, &prev_out);
    }
    if (n > 0 && n % 2 == 0) gi = gi_inter;
  }

  // ---- demodulate_radiance.wgsl:24-42 ----
  void demodulate(bool remodulate, std::vector<uint32_t>& in, std::vector<uint32_t>& out) {
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        V3 alb = rgb9e5_unpack(gbw[id].albedo);
        V3 r = rgb9e5_unpack(in[id]);
        if (remodulate) {
          r = r * alb;
        } else {
          r = v3(alb.x > 0.0f ? r.x / alb.x : 0.0f, alb.y > 0.0f ? r.y / alb.y : 0.0f,
                 alb.z > 0.0f ? r.z / alb.z : 0.0f);
        }
        out[id] = rgb9e5_pack(r);
      }
    });
  }

  // ---- firefly_filter.wgsl:20-85 (neighbours read from the unfiltered input) ----
  void firefly(std::vector<uint32_t>& buf) {
    std::vector<uint32_t> src = buf;
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        if (gt_is_sky(gbw[id].depth)) continue;
        V3 cur = rgb9e5_unpack(src[id]);
        float min_l = dm::F32_MAX, max_l = 0.0f;
        V3 min_c = cur, max_c = v3s(0.0f);
        float cur_l = luma(cur);
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy) {
            if (dx == 0 && dy == 0) continue;
            int sx = (int)x + dx, sy = (int)y + dy;
            if (sx < 0 || sy < 0 || sx >= (int)W || sy >= (int)H) continue;
            uint32_t sid = (uint32_t)sy * W + (uint32_t)sx;
            if (gt_is_sky(gbw[sid].depth)) continue;
            V3 nc = rgb9e5_unpack(src[sid]);
            float nl = luma(nc);
            if (nl < min_l) { min_l = nl; min_c = nc; }
            else if (nl > max_l) { max_l = nl; max_c = nc; }
          }
        V3 rec;
        if (cur_l < min_l) rec = min_c;
        else if (cur_l > max_l) rec = max_c;
        else rec = cur;
        if (min_l > max_l) rec = cur;
        buf[id] = rgb9e5_pack(rec);
      }
    });
  }

  // ---- svgf_temporal.wgsl:87-139 ----
  void svgf_temporal(std::vector<uint32_t>& demodv) {
    uint32_t f = frame_idx;
    std::vector<uint32_t>& out_rad = svgf_rad[(f + 1) % 2];
    std::vector<V2>& in_mom = svgf_mom[f % 2];
    std::vector<V2>& out_mom = svgf_mom[(f + 1) % 2];
    std::vector<float>& out_var = svgf_var[(f + 1) % 2];
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        GT cur = gt_unpack(gbw[id]);
        V3 rad = rgb9e5_unpack(demodv[id]);
        if (gt_is_sky(cur.depth)) {
          out_rad[id] = rgb9e5_pack(rad);
          continue;
        }
        V2 mom{luma(rad), 0.0f};
        mom.y = sqr(mom.x);
        V3 trad = v3s(0.0f);
        V2 tmom{0.0f, 0.0f};
        uint32_t count = 0;
        V2 pp;
        if (prev_point(x, y, &pp)) {
          GT prv = sample_prev_gbuffer(pp);
          if (history_valid(cur, prv)) {
            uint32_t ix = dm::f2u(dm::floor_(pp.x)), iy = dm::f2u(dm::floor_(pp.y));
            float fx = dm::fract(pp.x), fy = dm::fract(pp.y);
            uint32_t x1 = std::min(ix + 1, W - 1), y1 = std::min(iy + 1, H - 1);
            uint32_t i00 = iy * W + ix, i10 = iy * W + x1, i01 = y1 * W + ix, i11 = y1 * W + x1;
            V3 c0 = mix3(rgb9e5_unpack(svgf_hist[i00]), rgb9e5_unpack(svgf_hist[i10]), fx);
            V3 c1 = mix3(rgb9e5_unpack(svgf_hist[i01]), rgb9e5_unpack(svgf_hist[i11]), fx);
            trad = mix3(c0, c1, fy);
            V2 m00 = in_mom[i00], m10 = in_mom[i10], m01 = in_mom[i01], m11 = in_mom[i11];
            V2 m0{mixf(m00.x, m10.x, fx), mixf(m00.y, m10.y, fx)};
            V2 m1{mixf(m01.x, m11.x, fx), mixf(m01.y, m11.y, fx)};
            tmom = V2{mixf(m0.x, m1.x, fy), mixf(m0.y, m1.y, fy)};
            count = std::min(svgf_count[id] + 1, cfg.svgf_max_history);
          }
        }
        float alpha = 1.0f / (1.0f + (float)count);
        tmom = V2{mixf(tmom.x, mom.x, alpha), mixf(tmom.y, mom.y, alpha)};
        trad = mix3(trad, rad, alpha);
        out_var[id] = dm::fmax(tmom.y - sqr(tmom.x), 0.0f);
        out_rad[id] = rgb9e5_pack(trad);
        out_mom[id] = tmom;
        svgf_count[id] = count;
      }
    });
  }

  // ---- svgf_atrous.wgsl:48-117 ----
  void svgf_atrous(uint32_t pass_idx, std::vector<uint32_t>& in_rad, std::vector<uint32_t>& out_rad,
                   std::vector<float>& in_var, std::vector<float>& out_var) {
    const float KW[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    std::vector<GTexel>& gbw = gb();
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        GT cur = gt_unpack(gbw[id]);
        if (gt_is_sky(cur.depth)) continue;
        int32_t step = 1 << pass_idx;
        V3 rsum = rgb9e5_unpack(in_rad[id]);
        float vsum = in_var[id];
        float wsum = 1.0f;
        float cl = luma(rsum);
        float cv = vsum;
        for (int dy = -2; dy <= 2; ++dy)
          for (int dx = -2; dx <= 2; ++dx) {
            if (dy == 0 && dx == 0) continue;
            int sx = (int)x + dx * step, sy = (int)y + dy * step;
            if (sx < 0 || sy < 0 || sx >= (int)W || sy >= (int)H) continue;
            uint32_t sid = (uint32_t)sy * W + (uint32_t)sx;
            GT sg = gt_unpack(gbw[sid]);
            if (gt_is_sky(sg.depth)) continue;
            V3 srad = rgb9e5_unpack(in_rad[sid]);
            float sl = luma(srad);
            // PHI_NORMAL 128, PHI_DEPTH 0.1, PHI_LUMA 4 (svgf_atrous.wgsl:24-26)
            float nw = dm::pow_(dm::fmax(dot(cur.n, sg.n), 0.0f), 128.0f);
            float dd = dm::fabs_(cur.depth - sg.depth);
            float dw = dm::exp_(-sqr(dd) / (2.0f * sqr(0.1f)));
            float ld = dm::fabs_(cl - sl);
            float lw = dm::exp_(-ld / (dm::fmax(4.0f * dm::sqrt_(cv), 1e-8f)));
            float w = nw * dw * lw;
            w = w * (KW[dx < 0 ? -dx : dx] * KW[dy < 0 ? -dy : dy]);
            rsum = rsum + srad * w;
            vsum = vsum + in_var[sid] * sqr(w);
            wsum = wsum + w;
          }
        rsum = rsum / wsum;
        vsum = vsum / sqr(wsum);
        out_rad[id] = rgb9e5_pack(rsum);
        out_var[id] = vsum;
        if (pass_idx == 0) svgf_hist[id] = rgb9e5_pack(rsum);
      }
    });
  }

  void svgf(std::vector<uint32_t>& demodv) {
    uint32_t f = frame_idx;
    svgf_temporal(demodv);
    for (uint32_t i = 0; i < cfg.svgf_atrous_passes; ++i) {
      std::vector<uint32_t>& in_rad = svgf_rad[(f + 1 + i) % 2];
      std::vector<uint32_t>& out_rad = svgf_rad[(f + i) % 2];
      std::vector<float>& in_var = svgf_var[(f + 1 + i) % 2];
      std::vector<float>& out_var = svgf_var[(f + i) % 2];
      svgf_atrous(i, in_rad, out_rad, in_var, out_var);
      if (i == cfg.svgf_atrous_passes - 1) demodv = out_rad;
    }
  }

  // ---- taa.wgsl:67-171 (neighbours read from the pre-TAA input) ----
  static float mitchell(float x_, float B, float C) {
    float x = dm::fabs_(2.0f * x_);
    float ods = 1.0f / 6.0f;
    if (x > 1.0f)
      return ((-B - 6.0f * C) * x * x * x + (6.0f * B + 30.0f * C) * x * x +
              (-12.0f * B - 48.0f * C) * x + (8.0f * B + 24.0f * C)) * ods;
    return ((12.0f - 9.0f * B - 6.0f * C) * x * x * x + (-18.0f + 12.0f * B + 6.0f * C) * x * x +
            (6.0f - 2.0f * B)) * ods;
  }
  void taa(std::vector<uint32_t>& buf, std::vector<uint32_t>& prevb) {
    std::vector<uint32_t> src = buf;
    std::vector<GTexel>& gbw = gb();
    std::vector<GTexel>& pgb = prev_gb();
    const float hist_inf = cfg.taa_history_influence;
    parallel_rows(H, cfg.threads, [&](uint32_t y) {
      for (uint32_t x = 0; x < W; ++x) {
        uint32_t id = y * W + x;
        const GTexel& cg = gbw[id];
        if (gt_is_sky(cg.depth)) continue;
        V3 cur = rgb9e5_unpack(src[id]);
        float wsum = sqr(mitchell(0.0f, 0.33f, 0.33f));
        V3 rec = cur * wsum;
        V3 m1 = cur, m2 = cur * cur;
        float cnt = 1.0f;
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy) {
            if (dx == 0 && dy == 0) continue;
            int sx = (int)x + dx, sy = (int)y + dy;
            if (sx < 0 || sy < 0 || sx >= (int)W || sy >= (int)H) continue;
            uint32_t sid = (uint32_t)sy * W + (uint32_t)sx;
            V3 sc = vmax(rgb9e5_unpack(src[sid]), v3s(0.0f));
            float w = mitchell((float)dx, 0.33f, 0.33f) * mitchell((float)dy, 0.33f, 0.33f);
            w = w * (1.0f / (1.0f + luma(sc)));
            rec = rec + sc * w;
            wsum = wsum + w;
            m1 = m1 + sc;
            m2 = m2 + sc * sc;
            cnt = cnt + 1.0f;
          }
        rec = rec / dm::fmax(wsum, 1e-5f);
        V3 hist;
        uint32_t pid;
        V2 pp;
        if (prev_point(x, y, &pp)) {
          uint32_t fx = dm::f2u(dm::floor_(pp.x)), fy = dm::f2u(dm::floor_(pp.y));
          uint32_t cx = dm::f2u(dm::ceil_(pp.x)), cy = dm::f2u(dm::ceil_(pp.y));
          pid = fy * W + fx;
          uint32_t i00 = std::min(fy, H - 1) * W + std::min(fx, W - 1);
          uint32_t i10 = std::min(cy, H - 1) * W + std::min(fx, W - 1);
          uint32_t i01 = std::min(fy, H - 1) * W + std::min(cx, W - 1);
          uint32_t i11 = std::min(cy, H - 1) * W + std::min(cx, W - 1);
          V3 h00 = rgb9e5_unpack(prevb[i00]), h10 = rgb9e5_unpack(prevb[i10]);
          V3 h01 = rgb9e5_unpack(prevb[i01]), h11 = rgb9e5_unpack(prevb[i11]);
          float tx = dm::fract(pp.x), ty = dm::fract(pp.y);
          V3 a = h00 * (1.0f - tx) + h10 * tx;
          V3 b = h01 * (1.0f - tx) + h11 * tx;
          hist = a * (1.0f - ty) + b * ty;
        } else {
          hist = rgb9e5_unpack(prevb[id]);
          pid = id;
        }
        const GTexel& pg = pgb[pid];
        float cdcs = depth_cs(cg.depth, 0.001f, 10000.0f);
        float pdcs = depth_cs(pg.depth, 0.001f, 10000.0f);
        bool vdd = (dm::fabs_(cdcs - pdcs) / cdcs) < 0.1f;
        V3 mean = m1 / cnt;
        V3 sd = vabs(m2 - (m1 * m1) / cnt);
        sd = sd / (cnt - 1.0f);
        sd = vsqrt(sd);
        V3 lo = mean - sd, hi = mean + sd;
        V3 center = 0.5f * (hi + lo);
        V3 ext = 0.5f * (hi - lo);
        V3 rtc = hist - center;
        V3 rtcu = vabs(rtc / ext);
        float mx = dm::fmax(rtcu.x, dm::fmax(rtcu.y, rtcu.z));
        V3 clipped = mx > 1.0f ? center + rtc / mx : hist;
        float hwf = vdd ? 1.0f : 0.0f;
        float blend = 1.0f - (hist_inf * hwf);
        float cw = dm::saturate(blend * (1.0f / (1.0f + luma(rec))));
        float hw = dm::saturate((1.0f - blend) * (1.0f / (1.0f + luma(clipped))));
        rec = (cw * rec + hw * clipped) / (cw + hw);
        buf[id] = rgb9e5_pack(rec);
      }
    });
  }

  // PathTracerGpu::render (lib.rs:314-615) for the whole image; writes linear
  // HDR RGB (radiance / sample_count, resolve.wgsl:48-49 before the tonemap).
  void render(float* out_rgb) {
    std::fill(radiance.begin(), radiance.end(), 0u);
    std::vector<uint32_t>& dm_cur = demod[frame_idx % 2];
    std::vector<uint32_t>& dm_prev = demod[(frame_idx + 1) % 2];
    for (uint32_t sample = 0; sample < cfg.sample_count; ++sample) {
      uint32_t seed = frame_idx * cfg.sample_count + sample;
      raygen();
      for (uint32_t i = 0; i < cfg.max_bounces; ++i) {
        trace(i, seed);
        if (i == 0) {
          if (cfg.restir_di) restir_di(seed);
          if (cfg.restir_gi) restir_gi(seed);
        }
        apply_di();
        if (i + 1 < cfg.max_bounces) apply_gi();
      }
    }
    demodulate(false, radiance, dm_cur);
    if (cfg.firefly_filter) firefly(dm_cur);
    if (cfg.svgf) svgf(dm_cur);
    if (cfg.taa && frame_idx > 0) taa(dm_cur, dm_prev);
    demodulate(true, dm_cur, radiance);
    if (out_rgb) {
      for (size_t i = 0; i < radiance.size(); ++i) {
        V3 r = rgb9e5_unpack(radiance[i]);
        r = r / (float)cfg.sample_count;
        out_rgb[3 * i + 0] = r.x;
        out_rgb[3 * i + 1] = r.y;
        out_rgb[3 * i + 2] = r.z;
      }
    }
    frame_idx += 1;
  }
};

}  // namespace orc

// ============================================================================
// C API for ctypes (tests / smoke / bench cpu_baseline only).
using namespace orc;

struct OrcMesh {  // one mesh instance of the flattened scene
  uint32_t first_vertex, num_vertices, first_index, num_indices, material_idx, emissive;
};

extern "C" {

void* orc_scene_new(const float* positions, const float* normals, uint32_t num_vertices,
                    const uint32_t* indices, const uint32_t* tri_material, uint32_t num_tris,
                    const OrcMesh* meshes, uint32_t num_meshes, const float* materials,
                    uint32_t num_materials, const float* env, uint32_t env_w, uint32_t env_h,
                    const float* sun8) {
  Scene* s = new Scene();
  s->positions.resize(num_vertices);
  s->normals.resize(num_vertices);
  for (uint32_t i = 0; i < num_vertices; ++i) {
    s->positions[i] = v3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
    s->normals[i] = oct30_pack(v3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]));
  }
  s->indices.assign(indices, indices + 3 * (size_t)num_tris);
  s->tri_material.assign(tri_material, tri_material + num_tris);
  s->materials.resize(num_materials);
  static_assert(sizeof(Material) == 26 * sizeof(float), "material layout");
  memcpy(s->materials.data(), materials, sizeof(Material) * num_materials);
  uint32_t g = 0;
  for (uint32_t m = 0; m < num_meshes; ++m) {
    Instance in;
    in.first_vertex = meshes[m].first_vertex;
    in.num_vertices = meshes[m].num_vertices;
    in.first_index = meshes[m].first_index;
    in.num_indices = meshes[m].num_indices;
    in.material_idx = meshes[m].material_idx;
    in.emissive_idx = 0xFFFFFFFFu;
    in.first_global_tri = g;
    if (meshes[m].emissive) {
      in.emissive_idx = (uint32_t)s->emissive_instances.size();
      s->emissive_instances.push_back(m);
      s->num_emissive_tris += in.num_indices / 3;
    }
    s->instances.push_back(in);
    for (uint32_t t = 0; t < in.num_indices / 3; ++t) s->tri_instance.push_back(m);
    g += in.num_indices / 3;
  }
  // vertex_pool.rs:338-348
  float cdf = 0.0f;
  for (uint32_t e : s->emissive_instances) {
    float pdf = (float)(s->instances[e].num_indices / 3) / (float)s->num_emissive_tris;
    cdf = cdf + pdf;
    s->emissive_cdf.push_back(cdf);
  }
  if (env && env_w && env_h) {
    s->env.assign(env, env + 3 * (size_t)env_w * env_h);
    s->env_w = env_w;
    s->env_h = env_h;
  }
  memcpy(&s->sun, sun8, sizeof(float) * 8);
  return s;
}

void orc_scene_free(void* s) { delete (Scene*)s; }

// Closest hit for a batch of rays: out4[i] = {t, u, v, tri as float bits}.
void orc_closest(void* sp, const float* origins, const float* dirs, uint32_t n, float tmax,
                 uint32_t threads, float* out4, uint64_t* counts2) {
  Scene* s = (Scene*)sp;
  OracleBvh bvh;
  bvh.build(*s);
  std::vector<uint64_t> nodes(n, 0), tris(n, 0);
  parallel_rows(n, threads, [&](uint32_t i) {
    V3 o = v3(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
    V3 d = v3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    Hit h = bvh.closest(*s, o, d, 0.0f, tmax, &nodes[i], &tris[i]);
    out4[4 * i + 0] = h.t;
    out4[4 * i + 1] = h.u;
    out4[4 * i + 2] = h.v;
    memcpy(&out4[4 * i + 3], &h.tri, 4);
  });
  if (counts2) {
    counts2[0] = counts2[1] = 0;
    for (uint32_t i = 0; i < n; ++i) { counts2[0] += nodes[i]; counts2[1] += tris[i]; }
  }
}

// Any hit: out[i] = 1 when occluded in [0, tmax[i]].
void orc_any(void* sp, const float* origins, const float* dirs, const float* tmax, uint32_t n,
             uint32_t threads, uint8_t* out) {
  Scene* s = (Scene*)sp;
  OracleBvh bvh;
  bvh.build(*s);
  parallel_rows(n, threads, [&](uint32_t i) {
    V3 o = v3(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
    V3 d = v3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    out[i] = bvh.any(*s, o, d, 0.0f, tmax[i]) ? 1 : 0;
  });
}

void* orc_frame_new(void* scene, uint32_t w, uint32_t h, const FrameConfig* cfg) {
  return new Frame((Scene*)scene, w, h, *cfg);
}
void orc_frame_free(void* f) { delete (Frame*)f; }

// mats16x4: inv_view, inv_proj, view_proj, prev_view_proj, column-major.
void orc_frame_render(void* fp, const float* mats16x4, float* out_rgb) {
  Frame* f = (Frame*)fp;
  memcpy(f->mats, mats16x4, sizeof(f->mats));
  f->render(out_rgb);
}

uint64_t orc_frame_rays_cast(void* fp) { return ((Frame*)fp)->rays_cast; }

// Raw per-pixel buffers for stage-by-stage comparisons.
// which: 0 radiance(u32) 1 payload(3 u32) 2 gbuffer(6 u32, current) 3 di(8 u32)
//        4 gi(8 u32) 5 ctx(4 u32) 6 velocity(2 f32) 7 rays(4 u32)
void orc_frame_buffer(void* fp, uint32_t which, uint32_t* out) {
  Frame* f = (Frame*)fp;
  size_t P = (size_t)f->W * f->H;
  // after render() frame_idx has advanced: the frame just drawn used the other parity
  uint32_t cur = (f->frame_idx + 1) % 2;
  switch (which) {
    case 0: memcpy(out, f->radiance.data(), 4 * P); break;
    case 1: for (size_t i = 0; i < P; ++i) memcpy(out + 3 * i, &f->payloads[i], 12); break;
    case 2: for (size_t i = 0; i < P; ++i) memcpy(out + 6 * i, &f->gbuf[cur][i], 24); break;
    case 3: for (size_t i = 0; i < P; ++i) memcpy(out + 8 * i, &f->di[i], 32); break;
    case 4: for (size_t i = 0; i < P; ++i) memcpy(out + 8 * i, &f->gi[i], 32); break;
    case 5: for (size_t i = 0; i < P; ++i) memcpy(out + 4 * i, &f->ctx[i], 16); break;
    case 6: for (size_t i = 0; i < P; ++i) memcpy(out + 2 * i, &f->velocity[i], 8); break;
    case 7: for (size_t i = 0; i < P; ++i) memcpy(out + 4 * i, &f->rays[i], 16); break;
    default: break;
  }
}

// Display resolve (resolve.wgsl:29-59 with block.wgsl:3-16): radiance / spp
// through the ACES fit (hdr_to_sdr, resolve.wgsl:29-38), added to the
// accumulation, written as RGBA8 (round to nearest) at the 64x64-block-
// swizzled texture position; positions outside the texture are dropped.
void orc_resolve_rgba8(const uint32_t* radiance, uint32_t w, uint32_t h, uint32_t spp, float* accum4,
                       uint32_t accum_count, uint8_t* texture) {
  const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  const uint32_t B = 64, blocks_per_row = (w + B - 1) / B;
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      uint32_t i = y * w + x;
      V3 r = rgb9e5_unpack(radiance[i]);
      float hdr[3] = {r.x / (float)spp, r.y / (float)spp, r.z / (float)spp};
      float acc[3];
      for (int k = 0; k < 3; ++k) {
        float sdr = (hdr[k] * (a * hdr[k] + b)) / (hdr[k] * (c * hdr[k] + d) + e);
        sdr = dm::fmin(dm::fmax(sdr, 0.0f), 1.0f);
        acc[k] = accum4[4 * i + k] + sdr;
        accum4[4 * i + k] = acc[k];
      }
      accum4[4 * i + 3] = 0.0f;
      uint32_t block_index = (y / B) * blocks_per_row + x / B;
      uint32_t pixel_index = block_index * (B * B) + (y % B) * B + x % B;
      uint32_t px = pixel_index % w, py = pixel_index / w;
      if (px >= w || py >= h) continue;
      uint8_t* o = texture + 4 * ((size_t)py * w + px);
      for (int k = 0; k < 3; ++k) o[k] = (uint8_t)std::nearbyint(acc[k] / (float)(accum_count + 1) * 255.0f);
      o[3] = 255;
    }
}

// Packing / RNG / Disney entry points for the golden-vector tests.
uint32_t orc_rgb9e5_pack(const float* rgb) { return rgb9e5_pack(v3(rgb[0], rgb[1], rgb[2])); }
void orc_rgb9e5_unpack(uint32_t d, float* rgb) {
  V3 v = rgb9e5_unpack(d);
  rgb[0] = v.x; rgb[1] = v.y; rgb[2] = v.z;
}
uint32_t orc_oct30_pack(const float* d) { return oct30_pack(v3(d[0], d[1], d[2])); }
void orc_oct30_unpack(uint32_t p, float* d) {
  V3 v = oct30_unpack(p);
  d[0] = v.x; d[1] = v.y; d[2] = v.z;
}
uint32_t orc_pcg_hash(uint32_t x) { return pcg_hash(x); }
uint32_t orc_xor_shift(uint32_t x) { return xor_shift(x); }
uint32_t orc_hash_combine(uint32_t x, uint32_t y) { return hash_combine(x, y); }

// Disney sample/evaluate at a shading point with normal n (world space).
// in: mat (26 floats), n[3], wo[3], wi[3], r[3]; out: eval[4] = rgb,pdf;
// sample[7] = rgb, pdf, wi.xyz
void orc_disney(const float* mat, const float* n3, const float* wo3, const float* wi3,
                const float* r3, float* eval4, float* sample7) {
  Material m;
  memcpy(&m, mat, sizeof(m));
  Bsdf b = bsdf_from_material(m);
  ShadeFrame fr;
  fr.n = v3(n3[0], n3[1], n3[2]);
  fr.t2w = onb(fr.n);
  fr.cc_t2w = m.clearcoat > 0.0f ? onb(fr.n) : zero_m3();
  V3 wo = v3(wo3[0], wo3[1], wo3[2]), wi = v3(wi3[0], wi3[1], wi3[2]);
  float pdf = 0.0f;
  V3 e = disney_evaluate(b, fr, wo, wi, &pdf);
  eval4[0] = e.x; eval4[1] = e.y; eval4[2] = e.z; eval4[3] = pdf;
  V3 swi = v3s(0.0f);
  float spdf = 0.0f;
  bool spec = false;
  V3 s = disney_sample(b, fr, wo, 1.0f, false, r3[0], r3[1], r3[2], &swi, &spdf, &spec);
  sample7[0] = s.x; sample7[1] = s.y; sample7[2] = s.z; sample7[3] = spdf;
  sample7[4] = swi.x; sample7[5] = swi.y; sample7[6] = swi.z;
}

}  // extern "C"

// Elementary functions of detmath.h, for the accuracy tests.
extern "C" void orc_detmath(uint32_t fn, const float* x, const float* y, float* out, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i) {
    float a = x[i], b = y ? y[i] : 0.0f, r = 0.0f;
    switch (fn) {
      case 0: r = dm::sin_(a); break;
      case 1: r = dm::cos_(a); break;
      case 2: r = dm::exp_(a); break;
      case 3: r = dm::log_(a); break;
      case 4: r = dm::pow_(a, b); break;
      case 5: r = dm::atan2_(a, b); break;
      case 6: r = dm::acos_(a); break;
      default: r = 0.0f; break;
    }
    out[i] = r;
  }
}
