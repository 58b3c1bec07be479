// Oracle (test infrastructure only): Disney BSDF, sky, light sampling and
// reservoir arithmetic restated from the reference WGSL, scalar C++.
#pragma once

#include "oracle_scene.h"

namespace orc {

constexpr float PI = dm::PI;
constexpr float TWO_PI = dm::TWO_PI;
constexpr float INV_PI = dm::INV_PI;
constexpr uint32_t U32_MAX = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// Material -> DisneyBsdf (material_pool_bindings.wgsl:188-214,
// disney_bsdf.wgsl:226-244).  No textures: color.a (luminance) is 1.
struct Bsdf {
  V3 color;
  float metallic;
  V3 transmittance;
  float subsurface, luminance, specular, roughness;
  V3 spec_tint;
  float anisotropic, sheen;
  V3 sheen_tint;
  float clearcoat, clearcoat_gloss, transmission, eta;
};

inline V3 mv3(const float* p) { return v3(p[0], p[1], p[2]); }

inline Bsdf bsdf_from_material(const Material& m) {
  Bsdf b;
  b.color = mv3(m.color);
  b.metallic = m.metallic;
  b.transmittance = mv3(m.absorption);
  b.subsurface = m.subsurface;
  b.luminance = 1.0f;
  b.specular = dm::fmax(m.specular, 1.0f - m.roughness);
  b.roughness = m.roughness;
  b.spec_tint = mv3(m.specular_tint);
  b.anisotropic = m.anisotropic;
  b.sheen = m.sheen;
  b.sheen_tint = mv3(m.sheen_tint);
  b.clearcoat = m.clearcoat;
  b.clearcoat_gloss = 1.0f - m.clearcoat_roughness;
  b.transmission = m.transmission;
  b.eta = m.eta;
  return b;
}

// Frame of reference for one shading point: both bases the Disney lobes use.
struct ShadeFrame {
  V3 n;          // front-facing shading normal
  M3 t2w, cc_t2w;  // world_to_tangent = transpose(t2w)
};

V3 disney_sample(const Bsdf& b, const ShadeFrame& f, V3 wow, float distance, bool back_face,
                 float r0, float r1, float r2, V3* wiw, float* pdf, bool* specular);
V3 disney_evaluate(const Bsdf& b, const ShadeFrame& f, V3 wow, V3 wiw, float* pdf);

// ---------------------------------------------------------------------------
// Sky (sky_bindings.wgsl:4-78, math.wgsl:101-106, sampling.wgsl:57-73).
V3 sky_radiance(const Scene& s, V3 direction, bool skip_sun);
float sun_intensity(const Scene& s, V3 direction);
V3 direction_to_sun(const Scene& s, V2 uv);
V2 inverse_direction_to_sun(const Scene& s, V3 direction);

// ---------------------------------------------------------------------------
// Light samples (light_sample.wgsl:4-83, helpers/nee.wgsl:16-115).
struct LightSample {
  V2 uv;
  uint32_t inst;  // emissive instance index, U32_MAX-1 sun, U32_MAX empty
  uint32_t tri;
};
inline LightSample ls_empty() { return LightSample{{0.0f, 0.0f}, U32_MAX, 0}; }
inline LightSample ls_sun(V2 uv) { return LightSample{uv, U32_MAX - 1, 0}; }
inline bool ls_is_empty(const LightSample& l) { return l.inst == U32_MAX; }
inline bool ls_is_sun(const LightSample& l) { return l.inst == U32_MAX - 1; }

struct LightEval {
  V3 emission, point;
};
LightEval load_eval_data(const Scene& s, const LightSample& l, V3 hit_point);
LightSample sample_uniform(const Scene& s, float r0, float r1, float r2, V2 r34, float* pdf);

// DiReservoir (di_reservoir.wgsl:6-56); GiReservoir (gi_reservoir.wgsl:6-74).
struct DiRes {
  float M, W, wsum, phat;
  LightSample sample;
};
inline DiRes di_new() { return DiRes{0, 0, 0, 0, ls_empty()}; }
inline bool di_update(DiRes& r, float w, uint32_t& rng, const LightSample& s, float phat) {
  r.wsum = r.wsum + w;
  r.M = r.M + 1.0f;
  if (rnd(rng) <= (w / r.wsum)) {
    r.sample = s;
    r.phat = phat;
    return true;
  }
  return false;
}
struct GiRes {
  float M, W, wsum, phat;
  V3 point;
  uint32_t phat_rng;
};
inline GiRes gi_new() { return GiRes{0, 0, 0, 0, v3s(0), 0}; }
inline bool gi_update(GiRes& r, float w, uint32_t& rng, V3 point, float phat, uint32_t prng) {
  r.wsum = r.wsum + w;
  r.M = r.M + 1.0f;
  if (rnd(rng) <= (w / r.wsum)) {
    r.point = point;
    r.phat = phat;
    r.phat_rng = prng;
    return true;
  }
  return false;
}

// LightSampleCtx (light_sample.wgsl:23-30) without the texture coordinate.
struct Ctx {
  uint32_t material_idx;
  uint32_t throughput;  // rgb9e5
  uint32_t n;           // oct30
  uint32_t n_cc;        // oct30
};

}  // namespace orc
