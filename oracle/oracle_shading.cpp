// Oracle (test infrastructure only): Disney BSDF (appleseed-derived, as in
// shared/material/disney_bsdf.wgsl and ggxmdf.wgsl), sky and light sampling.
#include "oracle_shading.h"

namespace orc {

namespace {

using dm::fabs_;
using dm::fmax;
using dm::fmin;

// ---- ggxmdf.wgsl:20-213 ----
inline V2 alpha_from_roughness(float roughness, float anisotropy) {
  float sq = sqr(roughness);
  float aspect_factor = anisotropy < 0.0f ? 0.9f : -0.9f;
  float aspect = dm::sqrt_(1.0f + anisotropy * aspect_factor);
  return V2{fmax(0.001f, sq / aspect), fmax(0.001f, sq * aspect)};
}

struct Ggx { float ax, ay; };
inline float ggx_d(Ggx g, V3 m) {
  if (m.z == 0.0f) return sqr(g.ax) * INV_PI;
  float cos2 = sqr(m.z);
  float sin_t = dm::sqrt_(fmax(0.0f, 1.0f - cos2));
  float tan2 = (1.0f - cos2) / cos2;
  float sr;
  if (g.ax == g.ay || sin_t == 0.0f) sr = 1.0f / sqr(g.ax);
  else sr = sqr(m.x / (sin_t * g.ax)) + sqr(m.y / (sin_t * g.ay));
  return 1.0f / (PI * g.ax * g.ay * sqr(cos2) * sqr(1.0f + tan2 * sr));
}
inline float ggx_lambda(Ggx g, V3 v) {
  if (v.z == 0.0f) return 0.0f;
  float cos2 = sqr(v.z);
  float sin_t = dm::sqrt_(fmax(0.0f, 1.0f - cos2));
  float pr;
  if (g.ax == g.ay || sin_t == 0.0f) pr = g.ax;
  else pr = dm::sqrt_(sqr((v.x * g.ax) / sin_t) + sqr((v.y * g.ay) / sin_t));
  float tan2 = sqr(sin_t) / cos2;
  float a2_rcp = sqr(pr) * tan2;
  return (-1.0f + dm::sqrt_(1.0f + a2_rcp)) * 0.5f;
}
inline float ggx_g(Ggx g, V3 wi, V3 wo) {
  return 1.0f / (1.0f + ggx_lambda(g, wo) + ggx_lambda(g, wi));
}
inline float ggx_g1(Ggx g, V3 v) { return 1.0f / (1.0f + ggx_lambda(g, v)); }
inline V3 ggx_sample(Ggx g, V3 v, float r0, float r1) {
  float sgn = v.z < 0.0f ? -1.0f : 1.0f;
  V3 st = normalize(v3(sgn * v.x * g.ax, sgn * v.y * g.ay, sgn * v.z));
  V3 t1 = v.z < 0.9999f ? normalize(cross(st, v3(0.0f, 0.0f, 1.0f))) : v3(1.0f, 0.0f, 0.0f);
  V3 t2 = cross(t1, st);
  float a = 1.0f / (1.0f + st.z);
  float r = dm::sqrt_(r0);
  float phi = r1 < a ? r1 / a * PI : PI + (r1 - a) / (1.0f - a) * PI;
  float cphi, sphi;
  dm::sincos_(phi, &sphi, &cphi);
  float p1 = r * cphi;
  float p2 = r * sphi;
  if (r1 >= a) p2 = p2 * st.z;
  V3 h = p1 * t1 + p2 * t2 + dm::sqrt_(fmax(0.0f, 1.0f - sqr(p1) - sqr(p2))) * st;
  return normalize(v3(h.x * g.ax, h.y * g.ay, fmax(0.0f, h.z)));
}
inline float ggx_pdf(Ggx g, V3 v, V3 m) {
  float c = v.z;
  if (c == 0.0f) return 0.0f;
  return ggx_g1(g, v) * fabs_(dot(v, m)) * ggx_d(g, m) / fabs_(c);
}

struct Gtr1 { float ax; };
inline float gtr1_d(Gtr1 g, V3 m) {
  float alpha = dm::clamp(g.ax, 0.001f, 0.999f);
  float a2 = sqr(alpha);
  float a = (a2 - 1.0f) / (PI * dm::log_(a2));
  float b = (1.0f / (1.0f + (a2 - 1.0f) * sqr(m.z)));
  return a * b;
}
inline float gtr1_lambda(Gtr1 g, V3 v) {
  if (v.z == 0.0f) return 0.0f;
  float cos2 = sqr(v.z);
  float sin_t = dm::sqrt_(fmax(0.0f, 1.0f - cos2));
  if (sin_t == 0.0f) return 0.0f;
  float cot2 = cos2 / sqr(sin_t);
  float cot = dm::sqrt_(cot2);
  float alpha2 = sqr(dm::clamp(g.ax, 0.001f, 0.999f));
  float a = dm::sqrt_(cot2 + alpha2);
  float b = dm::sqrt_(cot2 + 1.0f);
  float c = dm::log_(cot + b);
  float d = dm::log_(cot + a);
  return (a - b + cot * (c - d)) / (cot * dm::log_(alpha2));
}
inline float gtr1_g(Gtr1 g, V3 wi, V3 wo) {
  return 1.0f / (1.0f + gtr1_lambda(g, wo) + gtr1_lambda(g, wi));
}
inline V3 gtr1_sample(Gtr1 g, float r0, float r1) {
  float alpha = dm::clamp(g.ax, 0.001f, 0.999f);
  float a2 = sqr(alpha);
  float cos2 = (1.0f - dm::pow_(a2, 1.0f - r0)) / (1.0f - a2);
  float sin_t = dm::sqrt_(fmax(0.0f, 1.0f - cos2));
  float phi = TWO_PI * r1;
  float sphi, cphi;
  dm::sincos_(phi, &sphi, &cphi);
  return v3(cphi * sin_t, sphi * sin_t, dm::sqrt_(cos2));
}
inline float gtr1_pdf(Gtr1 g, V3 m) { return gtr1_d(g, m) * fabs_(m.z); }

// ---- disney_bsdf.wgsl:22-206 ----
inline float schlick_fresnel(float u) {
  float m = dm::clamp(1.0f - u, 0.0f, 1.0f);
  float m4 = sqr(sqr(m));
  return m4 * m;
}
inline float fresnel_dielectric(float eta, float cos_i, float cos_t) {
  if (cos_i == 0.0f && cos_t == 0.0f) return 1.0f;
  float k0 = eta * cos_t;
  float k1 = eta * cos_i;
  return 0.5f * (sqr((cos_i - k0) / (cos_i + k0)) + sqr((cos_t - k1) / (cos_t + k1)));
}
inline float fresnel_reflectance(float cos_i, float eta, float* cos_t) {
  float sin_t2 = (1.0f - sqr(cos_i)) * sqr(eta);
  if (sin_t2 > 1.0f) {
    *cos_t = 0.0f;
    return 1.0f;
  }
  *cos_t = fmin(dm::sqrt_(fmax(1.0f - sin_t2, 0.0f)), 1.0f);
  return fresnel_dielectric(eta, fabs_(cos_i), *cos_t);
}
inline V3 eval_reflection(V3 color, V3 wo, V3 wi, V3 m, Ggx g, float f) {
  float denom = fabs_(4.0f * wo.z * wi.z);
  if (denom == 0.0f) return v3s(0.0f);
  float d = ggx_d(g, m);
  float gg = ggx_g(g, wi, wo);
  return color * (f * d * gg / denom);
}
inline V3 eval_refraction(float eta, V3 color, bool adjoint, V3 wo, V3 wi, V3 m, Ggx g, float t) {
  if (wo.z == 0.0f || wi.z == 0.0f) return v3s(0.0f);
  float cos_ih = dot(m, wi);
  float cos_oh = dot(m, wo);
  float dots = (cos_ih * cos_oh) / (wi.z * wo.z);
  float sd = cos_oh + eta * cos_ih;
  if (fabs_(sd) < 1e-6f) return v3s(0.0f);
  float d = ggx_d(g, m);
  float gg = ggx_g(g, wi, wo);
  float mult = fabs_(dots) * t * d * gg / sqr(sd);
  if (!adjoint) mult = mult * sqr(eta);
  return color * mult;
}
inline float reflection_jacobian(float cos_oh) {
  if (cos_oh == 0.0f) return 0.0f;
  return 1.0f / (4.0f * fabs_(cos_oh));
}
inline float refraction_jacobian(V3 wo, V3 wi, V3 m, float eta) {
  float cos_ih = dot(m, wi);
  float cos_oh = dot(m, wo);
  float sd = cos_oh + eta * cos_ih;
  if (fabs_(sd) < 1e-6f) return 0.0f;
  return fabs_(cos_ih) * sqr(eta / sd);
}
inline V3 improve_normalization(V3 v) { return v * ((3.0f - dot(v, v)) * 0.5f); }
inline V3 refracted_direction(V3 wo, V3 m, float cos_wom, float cos_t, float rcp_eta) {
  V3 wi;
  if (cos_wom > 0.0f) wi = (rcp_eta * cos_wom - cos_t) * m - rcp_eta * wo;
  else wi = (rcp_eta * cos_wom + cos_t) * m - rcp_eta * wo;
  return improve_normalization(wi);
}
inline V3 half_reflection(V3 wo, V3 wi) {
  V3 h = normalize(wo + wi);
  return h.z < 0.0f ? -h : h;
}
inline V3 half_refraction(V3 wo, V3 wi, float eta) {
  V3 h = normalize(wo + eta * wi);
  return h.z < 0.0f ? -h : h;
}
inline float choose_reflection_probability(float rw, float tw, float f) {
  float rp = f * rw;
  float tp = (1.0f - f) * tw;
  float sum = rp + tp;
  return sum == 0.0f ? 1.0f : rp / sum;
}
inline V3 diffuse_cos_weighted(float r0, float r1) {
  float term1 = TWO_PI * r0;
  float term2 = dm::sqrt_(1.0f - r1);
  float s, c;
  dm::sincos_(term1, &s, &c);
  return v3(c * term2, s * term2, dm::sqrt_(r1));
}
inline V3 mix_spectra(V3 a, V3 b, float t) { return (1.0f - t) * a + t * b; }
inline V3 mix_spectra_with_one(V3 a, float t) { return (1.0f - t) * a + v3s(t); }

inline float clearcoat_roughness(const Bsdf& b) { return mixf(0.1f, 0.001f, b.clearcoat_gloss); }
inline V3 specular_fresnel(const Bsdf& b, V3 o, V3 h) {
  V3 value = b.spec_tint;
  value = value * (b.specular * 0.08f);
  value = mix_spectra(value, b.color, b.metallic);
  float cos_oh = fabs_(dot(o, h));
  return mix_spectra_with_one(value, schlick_fresnel(cos_oh));
}
inline V3 clearcoat_fresnel(const Bsdf& b, V3 o, V3 h) {
  float cos_oh = fabs_(dot(o, h));
  return v3s(mixf(0.04f, 1.0f, schlick_fresnel(cos_oh)) * 0.25f * b.clearcoat);
}

void sample_mf(const Bsdf& b, float r0, float r1, float ax, float ay, V3 wol, bool cc, V3* wil,
               float* pdf, V3* value) {
  if (wol.z == 0.0f) {
    *value = v3s(0.0f);
    *pdf = 0.0f;
    return;
  }
  if (cc) {
    Gtr1 g{ax};
    V3 m = gtr1_sample(g, r0, r1);
    *wil = reflect(wol * -1.0f, m);
    if (wil->z == 0.0f) return;
    float cos_oh = dot(wol, m);
    *pdf = gtr1_pdf(g, m) / fabs_(4.0f * cos_oh);
    if (*pdf < 1e-6f) return;
    float d = gtr1_d(g, m);
    float gg = gtr1_g(g, *wil, wol);
    *value = clearcoat_fresnel(b, wol, m);
    *value = *value * (d * gg);
  } else {
    Ggx g{ax, ay};
    V3 m = ggx_sample(g, wol, r0, r1);
    *wil = reflect(wol * -1.0f, m);
    if (wil->z == 0.0f) return;
    float cos_oh = dot(wol, m);
    *pdf = ggx_pdf(g, wol, m) / fabs_(4.0f * cos_oh);
    if (*pdf < 1e-6f) return;
    float d = ggx_d(g, m);
    float gg = ggx_g(g, *wil, wol);
    *value = specular_fresnel(b, wol, m);
    *value = *value * (d * gg);
  }
}

float evaluate_mf(const Bsdf& b, float ax, float ay, V3 wol, V3 wil, V3 m, bool cc, V3* bsdf) {
  if (wol.z == 0.0f || wil.z == 0.0f) return 0.0f;
  float cos_oh = dot(wol, m);
  if (cos_oh == 0.0f) return 0.0f;
  if (cc) {
    Gtr1 g{ax};
    float d = gtr1_d(g, m);
    float gg = gtr1_g(g, wil, wol);
    *bsdf = clearcoat_fresnel(b, wol, m);
    *bsdf = *bsdf * (d * gg / fabs_(4.0f * wol.z * wil.z));
    return gtr1_pdf(g, m) / fabs_(4.0f * cos_oh);
  }
  Ggx g{ax, ay};
  float d = ggx_d(g, m);
  float gg = ggx_g(g, wil, wol);
  *bsdf = specular_fresnel(b, wol, m);
  *bsdf = *bsdf * (d * gg / fabs_(4.0f * wol.z * wil.z));
  return ggx_pdf(g, wol, m) / fabs_(4.0f * cos_oh);
}

float evaluate_diffuse(const Bsdf& b, V3 i_n, V3 wow, V3 wiw, V3 m, V3* value) {
  float cos_on = dot(i_n, wow);
  float cos_in = dot(i_n, wiw);
  float cos_ih = dot(wiw, m);
  float fl = schlick_fresnel(cos_in);
  float fv = schlick_fresnel(cos_on);
  float fd = 0.0f;
  if (b.subsurface != 1.0f) {
    float fd90 = 0.5f + 2.0f * sqr(cos_ih) * b.roughness;
    fd = mixf(1.0f, fd90, fl) * mixf(1.0f, fd90, fv);
  }
  if (b.subsurface > 0.0f) {
    float fss90 = sqr(cos_ih) * b.roughness;
    float fss = mixf(1.0f, fss90, fl) * mixf(1.0f, fss90, fv);
    float ss = 1.25f * (fss * (1.0f / (fabs_(cos_on) + fabs_(cos_in)) - 0.5f) + 0.5f);
    fd = mixf(fd, ss, b.subsurface);
  }
  *value = b.color * fd * INV_PI * (1.0f - b.metallic);
  return fabs_(cos_in) * INV_PI;
}

float evaluate_sheen(const Bsdf& b, V3 wow, V3 wiw, V3 m, V3* value) {
  V3 h = normalize(wow + wiw);
  (void)h;
  float cos_ih = dot(wiw, m);
  float fh = schlick_fresnel(cos_ih);
  *value = b.sheen_tint;
  *value = *value * (fh * b.sheen * (1.0f - b.metallic));
  return 1.0f / (2.0f * PI);
}

}  // namespace

// disney_bsdf.wgsl:380-565
V3 disney_sample(const Bsdf& b, const ShadeFrame& f, V3 wow, float distance, bool back_face,
                 float r0, float r1, float r2, V3* wiw, float* pdf, bool* specular) {
  const bool adjoint = false;
  float flip = back_face ? -1.0f : 1.0f;
  if (r0 < b.transmission) {
    *specular = true;
    float r3 = r0 / b.transmission;
    V3 wol = mul_t(f.t2w, wow);
    float eta = flip < 0.0f ? 1.0f / b.eta : b.eta;
    if (eta == 1.0f) return v3s(0.0f);
    V2 alpha = alpha_from_roughness(b.roughness, b.anisotropic);
    Ggx g{alpha.x, alpha.y};
    V3 m = ggx_sample(g, wol, r1, r3);
    float rcp_eta = 1.0f / eta;
    float cos_wom = dm::clamp(dot(wol, m), -1.0f, 1.0f);
    float cos_t;
    float fr = fresnel_reflectance(cos_wom, eta, &cos_t);
    float jac;
    V3 wil, ret;
    if (r2 < fr) {
      wil = reflect(wol * -1.0f, m);
      if (wil.z * wol.z <= 0.0f) return v3s(0.0f);
      ret = eval_reflection(b.color, wol, wil, m, g, fr);
      *pdf = fr;
      jac = reflection_jacobian(cos_wom);
    } else {
      wil = refracted_direction(wol, m, cos_wom, cos_t, eta);
      if (wil.z * wol.z > 0.0f) return v3s(0.0f);
      ret = eval_refraction(rcp_eta, b.color, adjoint, wol, wil, m, g, 1.0f - fr);
      *pdf = 1.0f - fr;
      jac = refraction_jacobian(wol, wil, m, rcp_eta);
    }
    *pdf = *pdf * (jac * ggx_pdf(g, wol, m));
    if (*pdf > 1e-6f) *wiw = mul(f.t2w, wil);
    if (back_face) {
      V3 beer = v3(dm::exp_(-b.transmittance.x * distance * 2.0f),
                   dm::exp_(-b.transmittance.y * distance * 2.0f),
                   dm::exp_(-b.transmittance.z * distance * 2.0f));
      ret = ret * beer;
    }
    return ret;
  }

  float r3 = (r0 - b.transmission) / (1.0f - b.transmission);
  float w[4] = {mixf(b.luminance, 0.0f, b.metallic), mixf(b.sheen, 0.0f, b.metallic),
                mixf(b.specular, 1.0f, b.metallic), b.clearcoat * 0.25f};
  float wsum = w[0] + w[1] + w[2] + w[3];
  if (wsum == 0.0f) {
    *pdf = 0.0f;
    return v3s(0.0f);
  }
  float inv = 1.0f / wsum;
  for (int k = 0; k < 4; ++k) w[k] = w[k] * inv;
  float cdf0 = w[0], cdf1 = w[0] + w[1], cdf2 = w[0] + w[1] + w[2];

  float probability = 0.0f, component_pdf = 0.0f;
  V3 value = v3s(0.0f);
  if (r3 < cdf1) {
    float rr = r3 / cdf1;
    *wiw = mul(f.t2w, diffuse_cos_weighted(rr, r1));
    V3 m = normalize(*wiw + wow);
    if (r3 < cdf0) {
      component_pdf = evaluate_diffuse(b, f.n, wow, *wiw, m, &value);
      probability = w[0] * component_pdf;
      w[0] = 0.0f;
    } else {
      component_pdf = evaluate_sheen(b, wow, *wiw, m, &value);
      probability = w[1] * component_pdf;
      w[1] = 0.0f;
    }
  } else {
    V3 wol, wil = v3s(0.0f);
    if (r3 < cdf2) {
      wol = mul_t(f.t2w, wow);
      float rr = (r3 - cdf1) / (cdf2 - cdf1);
      V2 alpha = alpha_from_roughness(b.roughness, b.anisotropic);
      sample_mf(b, rr, r1, alpha.x, alpha.y, wol, false, &wil, &component_pdf, &value);
      probability = w[2] * component_pdf;
      w[2] = 0.0f;
    } else {
      wol = mul_t(f.cc_t2w, wow);
      float rr = (r3 - cdf2) / (1.0f - cdf2);
      float alpha = clearcoat_roughness(b);
      sample_mf(b, rr, r1, alpha, alpha, wol, true, &wil, &component_pdf, &value);
      probability = w[3] * component_pdf;
      w[3] = 0.0f;
    }
    value = value * (1.0f / fabs_(4.0f * wol.z * wil.z));
    if (r3 < cdf2) *wiw = mul(f.t2w, wil);
    else *wiw = mul(f.cc_t2w, wil);
  }

  V3 contrib;
  if (w[0] + w[1] > 0.0f) {
    V3 m = normalize(*wiw + wow);
    if (w[0] > 0.0f) {
      probability = probability + w[0] * evaluate_diffuse(b, f.n, wow, *wiw, m, &contrib);
      value = value + contrib;
    }
    if (w[1] > 0.0f) {
      probability = probability + w[1] * evaluate_sheen(b, wow, *wiw, m, &contrib);
      value = value + contrib;
    }
  }
  if (w[2] + w[3] > 0.0f) {
    if (w[2] > 0.0f) {
      V3 wol = mul_t(f.t2w, wow);
      V3 wil = mul_t(f.t2w, *wiw);
      V3 m = normalize(wol + wil);
      V2 alpha = alpha_from_roughness(b.roughness, b.anisotropic);
      contrib = v3s(0.0f);
      probability = probability + w[2] * evaluate_mf(b, alpha.x, alpha.y, wol, wil, m, false, &contrib);
      value = value + contrib;
    }
    if (w[3] > 0.0f) {
      V3 wol = mul_t(f.cc_t2w, wow);
      V3 wil = mul_t(f.cc_t2w, *wiw);
      V3 m = normalize(wol + wil);
      float alpha = clearcoat_roughness(b);
      contrib = v3s(0.0f);
      probability = probability + w[3] * evaluate_mf(b, alpha, alpha, wol, wil, m, true, &contrib);
      value = value + contrib;
    }
  }
  *pdf = probability > 1e-6f ? probability : 0.0f;
  return value;
}

// disney_bsdf.wgsl:567-682
V3 disney_evaluate(const Bsdf& b, const ShadeFrame& f, V3 wow, V3 wiw, float* pdf) {
  if (b.transmission > 0.5f) {
    V3 wol = mul_t(f.t2w, wow);
    V3 wil = mul_t(f.t2w, wiw);
    float eta = wol.z > 0.0f ? b.eta : 1.0f / b.eta;
    if (eta == 1.0f) {
      *pdf = 0.0f;
      return v3s(0.0f);
    }
    V2 alpha = alpha_from_roughness(b.roughness, b.anisotropic);
    Ggx g{alpha.x, alpha.y};
    float jac;
    V3 ret, m;
    if (wil.z * wol.z >= 0.0f) {
      m = half_reflection(wol, wil);
      float cos_wom = dot(wol, m);
      float cos_t;
      float fr = fresnel_reflectance(cos_wom, 1.0f / eta, &cos_t);
      ret = eval_reflection(b.color, wol, wil, m, g, fr);
      *pdf = choose_reflection_probability(1.0f, 1.0f, fr);
      jac = reflection_jacobian(cos_wom);
    } else {
      m = half_refraction(wol, wil, eta);
      float cos_wom = dot(wol, m);
      float cos_t;
      float fr = fresnel_reflectance(cos_wom, 1.0f / eta, &cos_t);
      ret = eval_refraction(eta, b.color, false, wol, wil, m, g, 1.0f - fr);
      *pdf = 1.0f - choose_reflection_probability(1.0f, 1.0f, fr);
      jac = refraction_jacobian(wol, wil, m, eta);
    }
    *pdf = *pdf * (jac * ggx_pdf(g, wol, m));
    return ret;
  }

  float w[4] = {mixf(b.luminance, 0.0f, b.metallic), mixf(b.sheen, 0.0f, b.metallic),
                mixf(b.specular, 1.0f, b.metallic), b.clearcoat * 0.25f};
  float wsum = w[0] + w[1] + w[2] + w[3];
  if (wsum == 0.0f) {
    *pdf = 0.0f;
    return v3s(0.0f);
  }
  float inv = 1.0f / wsum;
  for (int k = 0; k < 4; ++k) w[k] = w[k] * inv;
  *pdf = 0.0f;
  V3 value = v3s(0.0f);
  if (w[0] + w[1] > 0.0f) {
    V3 m = normalize(wiw + wow);
    if (w[0] > 0.0f) {
      V3 c;
      *pdf = *pdf + w[0] * evaluate_diffuse(b, f.n, wow, wiw, m, &c);
      value = value + c;
    }
    if (w[1] > 0.0f) {
      V3 c;
      *pdf = *pdf + w[1] * evaluate_sheen(b, wow, wiw, m, &c);
      value = value + c;
    }
  }
  if (w[2] + w[3] > 0.0f) {
    if (w[2] > 0.0f) {
      V3 wol = mul_t(f.t2w, wow);
      V3 wil = mul_t(f.t2w, wiw);
      V3 m = normalize(wol + wil);
      V2 alpha = alpha_from_roughness(b.roughness, b.anisotropic);
      V3 c = v3s(0.0f);
      float spdf = w[2] * evaluate_mf(b, alpha.x, alpha.y, wol, wil, m, false, &c);
      if (spdf > 0.0f) {
        *pdf = *pdf + w[2] * spdf;
        value = value + c;
      }
    }
    if (w[3] > 0.0f) {
      V3 wol = mul_t(f.cc_t2w, wow);
      V3 wil = mul_t(f.cc_t2w, wiw);
      V3 m = normalize(wol + wil);
      float alpha = clearcoat_roughness(b);
      V3 c = v3s(0.0f);
      float cpdf = w[3] * evaluate_mf(b, alpha, alpha, wol, wil, m, true, &c);
      if (cpdf > 0.0f) {
        *pdf = *pdf + w[3] * cpdf;
        value = value + c;
      }
    }
  }
  return value;
}

// ---------------------------------------------------------------------------
namespace {
inline V3 perpendicular(V3 u) {
  V3 a = vabs(u);
  uint32_t xm = ((a.x - a.y) < 0.0f && (a.x - a.z) < 0.0f) ? 1u : 0u;
  uint32_t ym = (a.y - a.z) < 0.0f ? (1u ^ xm) : 0u;
  uint32_t zm = 1u ^ (xm | ym);
  return cross(u, v3((float)xm, (float)ym, (float)zm));
}
inline V3 perturb_direction(V2 uv, V3 direction, float angle) {
  float h = dm::cos_(angle);
  float phi = 2.0f * PI * uv.x;
  float z = h + (1.0f - h) * uv.y;
  float sin_t = dm::sqrt_(1.0f - z * z);
  float sp, cp;
  dm::sincos_(phi, &sp, &cp);
  float x = cp * sin_t;
  float y = sp * sin_t;
  V3 bitangent = perpendicular(direction);
  V3 tangent = cross(bitangent, direction);
  return bitangent * x + tangent * y + direction * z;
}
inline V3 sun_dir(const Scene& s) { return mv3(s.sun.direction); }
}  // namespace

float sun_intensity(const Scene& s, V3 direction) {
  const float CUTOFF = PI / 1.95f;
  V3 l = -sun_dir(s);
  float zc = dot(l, v3(0.0f, 1.0f, 0.0f));
  float intensity = s.sun.intensity * dm::fmax(0.0f, 1.0f - dm::exp_(-((CUTOFF - dm::acos_(zc)) / 1.4f)));
  float cos_theta = dot(direction, l);
  float dc = dm::cos_(s.sun.size * 0.1f);
  intensity = intensity * (cos_theta > dc ? 1.0f : 0.0f);
  return intensity;
}

V3 direction_to_sun(const Scene& s, V2 uv) {
  return normalize(perturb_direction(uv, -sun_dir(s), s.sun.size * 0.1f));
}

V2 inverse_direction_to_sun(const Scene& s, V3 direction) {
  V3 sd = -sun_dir(s);
  V3 bitangent = perpendicular(sd);
  V3 tangent = cross(bitangent, sd);
  float z = dot(direction, sd);
  float x = dot(direction, bitangent);
  float y = dot(direction, tangent);
  float phi = dm::atan2_(y, x);
  float q = phi / (2.0f * PI);
  float ux = q - truncf(q / 1.0f) * 1.0f;
  float c = dm::cos_(s.sun.size * 0.1f);
  float uy = (z - c) / (1.0f - c);
  return V2{ux, uy};
}

// Sky::sky: bilinear, repeat-addressed lookup of the equirect environment at
// unit_vector_to_panorama_coords(direction), plus the analytic sun disk.
V3 sky_radiance(const Scene& s, V3 direction, bool skip_sun) {
  V3 col = v3s(0.0f);
  if (s.env_w > 0) {
    float phi = dm::atan2_(direction.z, direction.x) + PI;
    float theta = dm::acos_(direction.y);
    float u = phi / (2.0f * PI);
    float v = theta * INV_PI;
    float x = u * (float)s.env_w - 0.5f;
    float y = v * (float)s.env_h - 0.5f;
    float fx0 = dm::floor_(x), fy0 = dm::floor_(y);
    float tx = x - fx0, ty = y - fy0;
    int32_t ix = dm::f2i(fx0), iy = dm::f2i(fy0);
    int32_t W = (int32_t)s.env_w, H = (int32_t)s.env_h;
    int32_t x0 = ((ix % W) + W) % W, x1 = (((ix + 1) % W) + W) % W;
    int32_t y0 = ((iy % H) + H) % H, y1 = (((iy + 1) % H) + H) % H;
    auto tex = [&](int32_t xx, int32_t yy) {
      const float* p = &s.env[3 * ((size_t)yy * s.env_w + (size_t)xx)];
      return v3(p[0], p[1], p[2]);
    };
    V3 a = tex(x0, y0) * (1.0f - tx) + tex(x1, y0) * tx;
    V3 b = tex(x0, y1) * (1.0f - tx) + tex(x1, y1) * tx;
    col = a * (1.0f - ty) + b * ty;
  }
  if (!skip_sun) {
    float intensity = sun_intensity(s, direction);
    col = col + (intensity * 1000.0f) * mv3(s.sun.color);
  }
  return col;
}

// helpers/nee.wgsl:16-57 (+ an empty or out-of-range sample evaluates to zero
// emission at the origin, where the reference reads out of bounds).
LightEval load_eval_data(const Scene& s, const LightSample& l, V3 hit_point) {
  if (ls_is_sun(l)) {
    V3 direction = direction_to_sun(s, l.uv);
    V3 point = direction * 1e6f;
    V3 emission = sun_intensity(s, direction) * mv3(s.sun.color);
    return LightEval{emission, point};
  }
  if (l.inst >= (uint32_t)s.emissive_instances.size()) return LightEval{v3s(0.0f), v3s(0.0f)};
  const Instance& in = s.instances[s.emissive_instances[l.inst]];
  uint32_t tri = l.tri < in.num_indices / 3 ? l.tri : in.num_indices / 3 - 1;
  uint32_t fi = in.first_index + tri * 3;
  V3 p0 = s.positions[in.first_vertex + s.indices[fi + 0]];
  V3 p1 = s.positions[in.first_vertex + s.indices[fi + 1]];
  V3 p2 = s.positions[in.first_vertex + s.indices[fi + 2]];
  float bx = 1.0f - l.uv.x - l.uv.y;
  V3 point = p0 * bx + p1 * l.uv.x + p2 * l.uv.y;
  V3 direction = normalize(point - hit_point);
  float dist = distance(point, hit_point);
  V3 p01 = p1 - p0, p02 = p2 - p0;
  V3 tn = normalize(cross(p01, p02));
  const Material& m = s.materials[in.material_idx + s.tri_material[in.first_index / 3 + tri]];
  float cos_out = dm::fmax(-dot(tn, direction), 0.0f);
  float solid_angle = dm::fmin(TWO_PI, cos_out / (sqr(dist) + 0.0001f));
  V3 emission = mv3(m.emission) * solid_angle * 10.0f;
  return LightEval{emission, point};
}

// helpers/nee.wgsl:59-115
LightSample sample_uniform(const Scene& s, float r0, float r1, float r2, V2 r34, float* pdf) {
  float sun_p = s.num_emissive_tris > 0 ? 0.5f : 1.0f;
  if (r0 < sun_p) {
    *pdf = sun_p;
    return ls_sun(r34);
  }
  for (uint32_t i = 0; i < (uint32_t)s.emissive_instances.size(); ++i) {
    if (r1 <= s.emissive_cdf[i]) {
      const Instance& in = s.instances[s.emissive_instances[i]];
      uint32_t ntri = in.num_indices / 3;
      uint32_t local = dm::f2u(r2 * (float)ntri);
      if (local >= ntri) local = ntri - 1;
      uint32_t fi = in.first_index + local * 3;
      V3 p0 = s.positions[in.first_vertex + s.indices[fi + 0]];
      V3 p1 = s.positions[in.first_vertex + s.indices[fi + 1]];
      V3 p2 = s.positions[in.first_vertex + s.indices[fi + 2]];
      V3 p01 = p1 - p0, p02 = p2 - p0;
      float area = length(cross(p01, p02)) * 0.5f;
      float p = 1.0f / (float)s.num_emissive_tris;
      p = p / area;
      *pdf = dm::fmax(1e-6f, p * (1.0f - sun_p));
      return LightSample{r34, i, local};
    }
  }
  *pdf = 0.0f;
  return ls_empty();
}

}  // namespace orc
