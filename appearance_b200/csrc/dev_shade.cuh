// Device shading: Disney BSDF (appleseed-derived, as the reference's
// shared/material/disney_bsdf.wgsl + ggxmdf.wgsl), sky and sun
// (shared/sky_bindings.wgsl), light sampling (helpers/nee.wgsl:16-115) and the
// ReSTIR reservoir update (shared/restir/*.wgsl).
#pragma once

#include "dev_common.cuh"
#include "scene_layout.h"

namespace ap {

constexpr float kPi = dm::PI;
constexpr float kTwoPi = dm::TWO_PI;
constexpr float kInvPi = dm::INV_PI;
constexpr uint32_t kU32Max = 0xFFFFFFFFu;

struct Bsdf {
  float3 color;
  float metallic;
  float3 transmittance;
  float subsurface, luminance, specular, roughness;
  float3 spec_tint;
  float anisotropic, sheen;
  float3 sheen_tint;
  float clearcoat, clearcoat_gloss, transmission, eta;
};

APD float3 ld3(const float* p) { return f3(p[0], p[1], p[2]); }

// Material::from_material_descriptor + DisneyBsdf::from_material
// (material_pool_bindings.wgsl:188-214, disney_bsdf.wgsl:226-244).
APD Bsdf load_bsdf(const MaterialDev* __restrict__ m) {
  Bsdf b;
  b.color = ld3(m->color);
  b.metallic = m->metallic;
  b.transmittance = ld3(m->absorption);
  b.subsurface = m->subsurface;
  b.luminance = 1.0f;
  b.specular = dm::fmax(m->specular, 1.0f - m->roughness);
  b.roughness = m->roughness;
  b.spec_tint = ld3(m->specular_tint);
  b.anisotropic = m->anisotropic;
  b.sheen = m->sheen;
  b.sheen_tint = ld3(m->sheen_tint);
  b.clearcoat = m->clearcoat;
  b.clearcoat_gloss = 1.0f - m->clearcoat_roughness;
  b.transmission = m->transmission;
  b.eta = m->eta;
  return b;
}

struct Frame {
  float3 n;
  Mat3 t2w, cc_t2w;
};

// ---- GGX / GTR1 (ggxmdf.wgsl:20-213) ----
APD float2 alpha_from_roughness(float roughness, float aniso) {
  float sq = sqr(roughness);
  float af = aniso < 0.0f ? 0.9f : -0.9f;
  float aspect = dm::sqrt_(1.0f + aniso * af);
  return make_float2(dm::fmax(0.001f, sq / aspect), dm::fmax(0.001f, sq * aspect));
}
APD float ggx_d(float ax, float ay, float3 m) {
  if (m.z == 0.0f) return sqr(ax) * kInvPi;
  float c2 = sqr(m.z);
  float st = dm::sqrt_(dm::fmax(0.0f, 1.0f - c2));
  float t2 = (1.0f - c2) / c2;
  float sr = (ax == ay || st == 0.0f) ? 1.0f / sqr(ax) : sqr(m.x / (st * ax)) + sqr(m.y / (st * ay));
  return 1.0f / (kPi * ax * ay * sqr(c2) * sqr(1.0f + t2 * sr));
}
APD float ggx_lambda(float ax, float ay, float3 v) {
  if (v.z == 0.0f) return 0.0f;
  float c2 = sqr(v.z);
  float st = dm::sqrt_(dm::fmax(0.0f, 1.0f - c2));
  float pr = (ax == ay || st == 0.0f) ? ax : dm::sqrt_(sqr((v.x * ax) / st) + sqr((v.y * ay) / st));
  float t2 = sqr(st) / c2;
  float a2 = sqr(pr) * t2;
  return (-1.0f + dm::sqrt_(1.0f + a2)) * 0.5f;
}
APD float ggx_g(float ax, float ay, float3 wi, float3 wo) {
  return 1.0f / (1.0f + ggx_lambda(ax, ay, wo) + ggx_lambda(ax, ay, wi));
}
APD float3 ggx_sample(float ax, float ay, float3 v, float r0, float r1) {
  float sgn = v.z < 0.0f ? -1.0f : 1.0f;
  float3 st = normalize(f3(sgn * v.x * ax, sgn * v.y * ay, sgn * v.z));
  float3 t1 = v.z < 0.9999f ? normalize(cross(st, f3(0.0f, 0.0f, 1.0f))) : f3(1.0f, 0.0f, 0.0f);
  float3 t2 = cross(t1, st);
  float a = 1.0f / (1.0f + st.z);
  float r = dm::sqrt_(r0);
  float phi = r1 < a ? r1 / a * kPi : kPi + (r1 - a) / (1.0f - a) * kPi;
  float sp, cp;
  dm::sincos_(phi, &sp, &cp);
  float p1 = r * cp;
  float p2 = r * sp;
  if (r1 >= a) p2 = p2 * st.z;
  float3 h = p1 * t1 + p2 * t2 + dm::sqrt_(dm::fmax(0.0f, 1.0f - sqr(p1) - sqr(p2))) * st;
  return normalize(f3(h.x * ax, h.y * ay, dm::fmax(0.0f, h.z)));
}
APD float ggx_pdf(float ax, float ay, float3 v, float3 m) {
  if (v.z == 0.0f) return 0.0f;
  float g1 = 1.0f / (1.0f + ggx_lambda(ax, ay, v));
  return g1 * dm::fabs_(dot(v, m)) * ggx_d(ax, ay, m) / dm::fabs_(v.z);
}
APD float gtr1_d(float ax, float3 m) {
  float a2 = sqr(dm::clamp(ax, 0.001f, 0.999f));
  float a = (a2 - 1.0f) / (kPi * dm::log_(a2));
  float b = (1.0f / (1.0f + (a2 - 1.0f) * sqr(m.z)));
  return a * b;
}
APD float gtr1_lambda(float ax, float3 v) {
  if (v.z == 0.0f) return 0.0f;
  float c2 = sqr(v.z);
  float st = dm::sqrt_(dm::fmax(0.0f, 1.0f - c2));
  if (st == 0.0f) return 0.0f;
  float cot2 = c2 / sqr(st);
  float cot = dm::sqrt_(cot2);
  float a2 = sqr(dm::clamp(ax, 0.001f, 0.999f));
  float a = dm::sqrt_(cot2 + a2);
  float b = dm::sqrt_(cot2 + 1.0f);
  float c = dm::log_(cot + b);
  float d = dm::log_(cot + a);
  return (a - b + cot * (c - d)) / (cot * dm::log_(a2));
}
APD float gtr1_g(float ax, float3 wi, float3 wo) {
  return 1.0f / (1.0f + gtr1_lambda(ax, wo) + gtr1_lambda(ax, wi));
}
APD float3 gtr1_sample(float ax, float r0, float r1) {
  float a2 = sqr(dm::clamp(ax, 0.001f, 0.999f));
  float c2 = (1.0f - dm::pow_(a2, 1.0f - r0)) / (1.0f - a2);
  float st = dm::sqrt_(dm::fmax(0.0f, 1.0f - c2));
  float phi = kTwoPi * r1;
  float sp, cp;
  dm::sincos_(phi, &sp, &cp);
  return f3(cp * st, sp * st, dm::sqrt_(c2));
}

// ---- Disney lobes (disney_bsdf.wgsl:22-378) ----
APD float schlick(float u) {
  float m = dm::clamp(1.0f - u, 0.0f, 1.0f);
  float m4 = sqr(sqr(m));
  return m4 * m;
}
APD float fresnel_refl(float ci, float eta, float* ct) {
  float st2 = (1.0f - sqr(ci)) * sqr(eta);
  if (st2 > 1.0f) {
    *ct = 0.0f;
    return 1.0f;
  }
  *ct = dm::fmin(dm::sqrt_(dm::fmax(1.0f - st2, 0.0f)), 1.0f);
  float cti = dm::fabs_(ci), ctt = *ct;
  if (cti == 0.0f && ctt == 0.0f) return 1.0f;
  float k0 = eta * ctt, k1 = eta * cti;
  return 0.5f * (sqr((cti - k0) / (cti + k0)) + sqr((ctt - k1) / (ctt + k1)));
}
APD float3 eval_reflection(float3 color, float3 wo, float3 wi, float3 m, float ax, float ay, float f) {
  float denom = dm::fabs_(4.0f * wo.z * wi.z);
  if (denom == 0.0f) return f3s(0.0f);
  float d = ggx_d(ax, ay, m);
  float g = ggx_g(ax, ay, wi, wo);
  return color * (f * d * g / denom);
}
APD float3 eval_refraction(float eta, float3 color, float3 wo, float3 wi, float3 m, float ax, float ay, float t) {
  if (wo.z == 0.0f || wi.z == 0.0f) return f3s(0.0f);
  float cih = dot(m, wi), coh = dot(m, wo);
  float dots = (cih * coh) / (wi.z * wo.z);
  float sd = coh + eta * cih;
  if (dm::fabs_(sd) < 1e-6f) return f3s(0.0f);
  float d = ggx_d(ax, ay, m);
  float g = ggx_g(ax, ay, wi, wo);
  float mult = dm::fabs_(dots) * t * d * g / sqr(sd);
  mult = mult * sqr(eta);  // adjoint == false
  return color * mult;
}
APD float refl_jacobian(float coh) { return coh == 0.0f ? 0.0f : 1.0f / (4.0f * dm::fabs_(coh)); }
APD float refr_jacobian(float3 wo, float3 wi, float3 m, float eta) {
  float cih = dot(m, wi), coh = dot(m, wo);
  float sd = coh + eta * cih;
  if (dm::fabs_(sd) < 1e-6f) return 0.0f;
  return dm::fabs_(cih) * sqr(eta / sd);
}
APD float3 refracted_dir(float3 wo, float3 m, float cwm, float ct, float rcp_eta) {
  float3 wi = cwm > 0.0f ? (rcp_eta * cwm - ct) * m - rcp_eta * wo : (rcp_eta * cwm + ct) * m - rcp_eta * wo;
  return wi * ((3.0f - dot(wi, wi)) * 0.5f);
}
APD float clearcoat_alpha(const Bsdf& b) { return mixf(0.1f, 0.001f, b.clearcoat_gloss); }
APD float3 spec_fresnel(const Bsdf& b, float3 o, float3 h) {
  float3 v = b.spec_tint;
  v = v * (b.specular * 0.08f);
  v = (1.0f - b.metallic) * v + b.metallic * b.color;
  float s = schlick(dm::fabs_(dot(o, h)));
  return (1.0f - s) * v + f3s(s);
}
APD float3 cc_fresnel(const Bsdf& b, float3 o, float3 h) {
  return f3s(mixf(0.04f, 1.0f, schlick(dm::fabs_(dot(o, h)))) * 0.25f * b.clearcoat);
}
APD void sample_mf(const Bsdf& b, float r0, float r1, float ax, float ay, float3 wol, bool cc, float3* wil,
                   float* pdf, float3* value) {
  if (wol.z == 0.0f) {
    *value = f3s(0.0f);
    *pdf = 0.0f;
    return;
  }
  float3 m = cc ? gtr1_sample(ax, r0, r1) : ggx_sample(ax, ay, wol, r0, r1);
  *wil = reflect(wol * -1.0f, m);
  if (wil->z == 0.0f) return;
  float coh = dot(wol, m);
  *pdf = (cc ? gtr1_d(ax, m) * dm::fabs_(m.z) : ggx_pdf(ax, ay, wol, m)) / dm::fabs_(4.0f * coh);
  if (*pdf < 1e-6f) return;
  if (cc) {
    float d = gtr1_d(ax, m);
    float g = gtr1_g(ax, *wil, wol);
    *value = cc_fresnel(b, wol, m);
    *value = *value * (d * g);
  } else {
    float d = ggx_d(ax, ay, m);
    float g = ggx_g(ax, ay, *wil, wol);
    *value = spec_fresnel(b, wol, m);
    *value = *value * (d * g);
  }
}
APD float eval_mf(const Bsdf& b, float ax, float ay, float3 wol, float3 wil, float3 m, bool cc, float3* out) {
  if (wol.z == 0.0f || wil.z == 0.0f) return 0.0f;
  float coh = dot(wol, m);
  if (coh == 0.0f) return 0.0f;
  if (cc) {
    float d = gtr1_d(ax, m);
    float g = gtr1_g(ax, wil, wol);
    *out = cc_fresnel(b, wol, m);
    *out = *out * (d * g / dm::fabs_(4.0f * wol.z * wil.z));
    return gtr1_d(ax, m) * dm::fabs_(m.z) / dm::fabs_(4.0f * coh);
  }
  float d = ggx_d(ax, ay, m);
  float g = ggx_g(ax, ay, wil, wol);
  *out = spec_fresnel(b, wol, m);
  *out = *out * (d * g / dm::fabs_(4.0f * wol.z * wil.z));
  return ggx_pdf(ax, ay, wol, m) / dm::fabs_(4.0f * coh);
}
APD float eval_diffuse(const Bsdf& b, float3 n, float3 wo, float3 wi, float3 m, float3* out) {
  float con = dot(n, wo), cin = dot(n, wi), cih = dot(wi, m);
  float fl = schlick(cin), fv = schlick(con);
  float fd = 0.0f;
  if (b.subsurface != 1.0f) {
    float fd90 = 0.5f + 2.0f * sqr(cih) * b.roughness;
    fd = mixf(1.0f, fd90, fl) * mixf(1.0f, fd90, fv);
  }
  if (b.subsurface > 0.0f) {
    float fss90 = sqr(cih) * b.roughness;
    float fss = mixf(1.0f, fss90, fl) * mixf(1.0f, fss90, fv);
    float ss = 1.25f * (fss * (1.0f / (dm::fabs_(con) + dm::fabs_(cin)) - 0.5f) + 0.5f);
    fd = mixf(fd, ss, b.subsurface);
  }
  *out = b.color * fd * kInvPi * (1.0f - b.metallic);
  return dm::fabs_(cin) * kInvPi;
}
APD float eval_sheen(const Bsdf& b, float3 wi, float3 m, float3* out) {
  float fh = schlick(dot(wi, m));
  *out = b.sheen_tint;
  *out = *out * (fh * b.sheen * (1.0f - b.metallic));
  return 1.0f / (2.0f * kPi);
}

// DisneyBsdf::sample (disney_bsdf.wgsl:380-565).  `wiw` and `pdf` keep the
// caller's values on the early returns, as in the reference.
APD float3 disney_sample(const Bsdf& b, const Frame& f, float3 wow, float distance, bool back_face, float r0,
                         float r1, float r2, float3* wiw, float* pdf) {
  if (r0 < b.transmission) {
    float r3 = r0 / b.transmission;
    float3 wol = mul_t(f.t2w, wow);
    float eta = back_face ? 1.0f / b.eta : b.eta;
    if (eta == 1.0f) return f3s(0.0f);
    float2 al = alpha_from_roughness(b.roughness, b.anisotropic);
    float3 m = ggx_sample(al.x, al.y, wol, r1, r3);
    float rcp_eta = 1.0f / eta;
    float cwm = dm::clamp(dot(wol, m), -1.0f, 1.0f);
    float ct;
    float fr = fresnel_refl(cwm, eta, &ct);
    float jac;
    float3 wil, ret;
    if (r2 < fr) {
      wil = reflect(wol * -1.0f, m);
      if (wil.z * wol.z <= 0.0f) return f3s(0.0f);
      ret = eval_reflection(b.color, wol, wil, m, al.x, al.y, fr);
      *pdf = fr;
      jac = refl_jacobian(cwm);
    } else {
      wil = refracted_dir(wol, m, cwm, ct, eta);
      if (wil.z * wol.z > 0.0f) return f3s(0.0f);
      ret = eval_refraction(rcp_eta, b.color, wol, wil, m, al.x, al.y, 1.0f - fr);
      *pdf = 1.0f - fr;
      jac = refr_jacobian(wol, wil, m, rcp_eta);
    }
    *pdf = *pdf * (jac * ggx_pdf(al.x, al.y, wol, m));
    if (*pdf > 1e-6f) *wiw = mul(f.t2w, wil);
    if (back_face) {
      float3 beer = f3(dm::exp_(-b.transmittance.x * distance * 2.0f), dm::exp_(-b.transmittance.y * distance * 2.0f),
                       dm::exp_(-b.transmittance.z * distance * 2.0f));
      ret = ret * beer;
    }
    return ret;
  }
  float r3 = (r0 - b.transmission) / (1.0f - b.transmission);
  float w0 = mixf(b.luminance, 0.0f, b.metallic), w1 = mixf(b.sheen, 0.0f, b.metallic);
  float w2 = mixf(b.specular, 1.0f, b.metallic), w3 = b.clearcoat * 0.25f;
  float ws = w0 + w1 + w2 + w3;
  if (ws == 0.0f) {
    *pdf = 0.0f;
    return f3s(0.0f);
  }
  float inv = 1.0f / ws;
  w0 = w0 * inv; w1 = w1 * inv; w2 = w2 * inv; w3 = w3 * inv;
  float cdf0 = w0, cdf1 = w0 + w1, cdf2 = w0 + w1 + w2;
  float prob = 0.0f, cpdf = 0.0f;
  float3 value = f3s(0.0f);
  if (r3 < cdf1) {
    float rr = r3 / cdf1;
    float term1 = kTwoPi * rr, term2 = dm::sqrt_(1.0f - r1);
    float s, c;
    dm::sincos_(term1, &s, &c);
    *wiw = mul(f.t2w, f3(c * term2, s * term2, dm::sqrt_(r1)));
    float3 m = normalize(*wiw + wow);
    if (r3 < cdf0) {
      cpdf = eval_diffuse(b, f.n, wow, *wiw, m, &value);
      prob = w0 * cpdf;
      w0 = 0.0f;
    } else {
      cpdf = eval_sheen(b, *wiw, m, &value);
      prob = w1 * cpdf;
      w1 = 0.0f;
    }
  } else {
    float3 wol, wil = f3s(0.0f);
    bool spec = r3 < cdf2;
    if (spec) {
      wol = mul_t(f.t2w, wow);
      float rr = (r3 - cdf1) / (cdf2 - cdf1);
      float2 al = alpha_from_roughness(b.roughness, b.anisotropic);
      sample_mf(b, rr, r1, al.x, al.y, wol, false, &wil, &cpdf, &value);
      prob = w2 * cpdf;
      w2 = 0.0f;
    } else {
      wol = mul_t(f.cc_t2w, wow);
      float rr = (r3 - cdf2) / (1.0f - cdf2);
      float a = clearcoat_alpha(b);
      sample_mf(b, rr, r1, a, a, wol, true, &wil, &cpdf, &value);
      prob = w3 * cpdf;
      w3 = 0.0f;
    }
    value = value * (1.0f / dm::fabs_(4.0f * wol.z * wil.z));
    *wiw = spec ? mul(f.t2w, wil) : mul(f.cc_t2w, wil);
  }
  float3 contrib;
  if (w0 + w1 > 0.0f) {
    float3 m = normalize(*wiw + wow);
    if (w0 > 0.0f) {
      prob = prob + w0 * eval_diffuse(b, f.n, wow, *wiw, m, &contrib);
      value = value + contrib;
    }
    if (w1 > 0.0f) {
      prob = prob + w1 * eval_sheen(b, *wiw, m, &contrib);
      value = value + contrib;
    }
  }
  if (w2 + w3 > 0.0f) {
    if (w2 > 0.0f) {
      float3 wol = mul_t(f.t2w, wow), wil = mul_t(f.t2w, *wiw);
      float3 m = normalize(wol + wil);
      float2 al = alpha_from_roughness(b.roughness, b.anisotropic);
      contrib = f3s(0.0f);
      prob = prob + w2 * eval_mf(b, al.x, al.y, wol, wil, m, false, &contrib);
      value = value + contrib;
    }
    if (w3 > 0.0f) {
      float3 wol = mul_t(f.cc_t2w, wow), wil = mul_t(f.cc_t2w, *wiw);
      float3 m = normalize(wol + wil);
      float a = clearcoat_alpha(b);
      contrib = f3s(0.0f);
      prob = prob + w3 * eval_mf(b, a, a, wol, wil, m, true, &contrib);
      value = value + contrib;
    }
  }
  *pdf = prob > 1e-6f ? prob : 0.0f;
  return value;
}

// The parts of DisneyBsdf::evaluate that depend only on the material and the
// outgoing direction, computed once per shading point with the same
// expressions the per-direction evaluation would repeat: lobe weights, GGX
// and clearcoat roughness, wo in both tangent frames, the Smith lambda of wo,
// the GTR1 normalisation and the specular Fresnel base.
struct DisneyCtx {
  float w0, w1, w2, w3;  // normalised lobe weights; all 0 when their sum is 0
  float ax, ay, one_lam_wo, g1_wo;  // GGX: alphas, 1 + lambda(wo), 1 / (1 + lambda(wo))
  float3 wol, spec_f0;              // wo in the specular frame, spec_fresnel's base colour
  float cca, cc_a2, cc_da, cc_log_a2, cc_one_lam_wo;  // clearcoat (GTR1)
  float3 wol_cc;
  bool zero;
};

APD float gtr1_lambda_c(float a2, float log_a2, float3 v) {  // gtr1_lambda with a2 and log(a2) given
  if (v.z == 0.0f) return 0.0f;
  float c2 = sqr(v.z);
  float st = dm::sqrt_(dm::fmax(0.0f, 1.0f - c2));
  if (st == 0.0f) return 0.0f;
  float cot2 = c2 / sqr(st);
  float cot = dm::sqrt_(cot2);
  float a = dm::sqrt_(cot2 + a2);
  float b = dm::sqrt_(cot2 + 1.0f);
  float c = dm::log_(cot + b);
  float d = dm::log_(cot + a);
  return (a - b + cot * (c - d)) / (cot * log_a2);
}

APD DisneyCtx disney_ctx(const Bsdf& b, const Frame& f, float3 wow) {
  DisneyCtx c;
  float w0 = mixf(b.luminance, 0.0f, b.metallic), w1 = mixf(b.sheen, 0.0f, b.metallic);
  float w2 = mixf(b.specular, 1.0f, b.metallic), w3 = b.clearcoat * 0.25f;
  float ws = w0 + w1 + w2 + w3;
  c.zero = ws == 0.0f;
  if (c.zero) {
    c.w0 = c.w1 = c.w2 = c.w3 = 0.0f;
  } else {
    float inv = 1.0f / ws;
    c.w0 = w0 * inv; c.w1 = w1 * inv; c.w2 = w2 * inv; c.w3 = w3 * inv;
  }
  if (c.w2 > 0.0f) {
    c.wol = mul_t(f.t2w, wow);
    float2 al = alpha_from_roughness(b.roughness, b.anisotropic);
    c.ax = al.x;
    c.ay = al.y;
    c.one_lam_wo = 1.0f + ggx_lambda(c.ax, c.ay, c.wol);
    c.g1_wo = 1.0f / c.one_lam_wo;
    float3 v = b.spec_tint;
    v = v * (b.specular * 0.08f);
    c.spec_f0 = (1.0f - b.metallic) * v + b.metallic * b.color;
  }
  if (c.w3 > 0.0f) {
    c.wol_cc = mul_t(f.cc_t2w, wow);
    c.cca = clearcoat_alpha(b);
    c.cc_a2 = sqr(dm::clamp(c.cca, 0.001f, 0.999f));
    c.cc_log_a2 = dm::log_(c.cc_a2);
    c.cc_da = (c.cc_a2 - 1.0f) / (kPi * c.cc_log_a2);
    c.cc_one_lam_wo = 1.0f + gtr1_lambda_c(c.cc_a2, c.cc_log_a2, c.wol_cc);
  }
  return c;
}

// DisneyBsdf::evaluate (disney_bsdf.wgsl:567-682) for the reflective lobes,
// with the shading point's DisneyCtx; same arithmetic as eval_diffuse,
// eval_sheen and eval_mf.
APD float3 disney_eval_ctx(const Bsdf& b, const DisneyCtx& c, const Frame& f, float3 wow, float3 wiw, float* pdf) {
  if (c.zero) {
    *pdf = 0.0f;
    return f3s(0.0f);
  }
  *pdf = 0.0f;
  float3 value = f3s(0.0f);
  if (c.w0 + c.w1 > 0.0f) {
    float3 m = normalize(wiw + wow);
    if (c.w0 > 0.0f) {
      float3 o;
      *pdf = *pdf + c.w0 * eval_diffuse(b, f.n, wow, wiw, m, &o);
      value = value + o;
    }
    if (c.w1 > 0.0f) {
      float3 o;
      *pdf = *pdf + c.w1 * eval_sheen(b, wiw, m, &o);
      value = value + o;
    }
  }
  if (c.w2 + c.w3 > 0.0f) {
    if (c.w2 > 0.0f) {
      const float3 wol = c.wol, wil = mul_t(f.t2w, wiw);
      const float3 m = normalize(wol + wil);
      float sp = 0.0f;
      float3 o = f3s(0.0f);
      if (wol.z != 0.0f && wil.z != 0.0f) {
        const float coh = dot(wol, m);
        if (coh != 0.0f) {
          const float d = ggx_d(c.ax, c.ay, m);
          const float g = 1.0f / (c.one_lam_wo + ggx_lambda(c.ax, c.ay, wil));
          const float sf = schlick(dm::fabs_(dot(wol, m)));
          o = (1.0f - sf) * c.spec_f0 + f3s(sf);
          o = o * (d * g / dm::fabs_(4.0f * wol.z * wil.z));
          sp = (c.g1_wo * dm::fabs_(dot(wol, m)) * d / dm::fabs_(wol.z)) / dm::fabs_(4.0f * coh);
        }
      }
      sp = c.w2 * sp;
      if (sp > 0.0f) {
        *pdf = *pdf + c.w2 * sp;
        value = value + o;
      }
    }
    if (c.w3 > 0.0f) {
      const float3 wol = c.wol_cc, wil = mul_t(f.cc_t2w, wiw);
      const float3 m = normalize(wol + wil);
      float cp = 0.0f;
      float3 o = f3s(0.0f);
      if (wol.z != 0.0f && wil.z != 0.0f) {
        const float coh = dot(wol, m);
        if (coh != 0.0f) {
          const float d = c.cc_da * (1.0f / (1.0f + (c.cc_a2 - 1.0f) * sqr(m.z)));
          const float g = 1.0f / (c.cc_one_lam_wo + gtr1_lambda_c(c.cc_a2, c.cc_log_a2, wil));
          o = cc_fresnel(b, wol, m);
          o = o * (d * g / dm::fabs_(4.0f * wol.z * wil.z));
          cp = d * dm::fabs_(m.z) / dm::fabs_(4.0f * coh);
        }
      }
      cp = c.w3 * cp;
      if (cp > 0.0f) {
        *pdf = *pdf + c.w3 * cp;
        value = value + o;
      }
    }
  }
  return value;
}

// DisneyBsdf::evaluate (disney_bsdf.wgsl:567-682).
APD float3 disney_eval(const Bsdf& b, const Frame& f, float3 wow, float3 wiw, float* pdf) {
  if (b.transmission > 0.5f) {
    float3 wol = mul_t(f.t2w, wow), wil = mul_t(f.t2w, wiw);
    float eta = wol.z > 0.0f ? b.eta : 1.0f / b.eta;
    if (eta == 1.0f) {
      *pdf = 0.0f;
      return f3s(0.0f);
    }
    float2 al = alpha_from_roughness(b.roughness, b.anisotropic);
    float jac;
    float3 ret, m;
    if (wil.z * wol.z >= 0.0f) {
      m = normalize(wol + wil);
      if (m.z < 0.0f) m = -m;
      float cwm = dot(wol, m);
      float ct;
      float fr = fresnel_refl(cwm, 1.0f / eta, &ct);
      ret = eval_reflection(b.color, wol, wil, m, al.x, al.y, fr);
      float rp = fr * 1.0f, tp = (1.0f - fr) * 1.0f, sum = rp + tp;
      *pdf = sum == 0.0f ? 1.0f : rp / sum;
      jac = refl_jacobian(cwm);
    } else {
      m = normalize(wol + eta * wil);
      if (m.z < 0.0f) m = -m;
      float cwm = dot(wol, m);
      float ct;
      float fr = fresnel_refl(cwm, 1.0f / eta, &ct);
      ret = eval_refraction(eta, b.color, wol, wil, m, al.x, al.y, 1.0f - fr);
      float rp = fr * 1.0f, tp = (1.0f - fr) * 1.0f, sum = rp + tp;
      *pdf = 1.0f - (sum == 0.0f ? 1.0f : rp / sum);
      jac = refr_jacobian(wol, wil, m, eta);
    }
    *pdf = *pdf * (jac * ggx_pdf(al.x, al.y, wol, m));
    return ret;
  }
  return disney_eval_ctx(b, disney_ctx(b, f, wow), f, wow, wiw, pdf);
}

// ---- sky and sun (sky_bindings.wgsl:4-78, sampling.wgsl:57-73, math.wgsl:88-106) ----
APD float3 perpendicular(float3 u) {
  float3 a = vabs(u);
  uint32_t xm = ((a.x - a.y) < 0.0f && (a.x - a.z) < 0.0f) ? 1u : 0u;
  uint32_t ym = (a.y - a.z) < 0.0f ? (1u ^ xm) : 0u;
  uint32_t zm = 1u ^ (xm | ym);
  return cross(u, f3((float)xm, (float)ym, (float)zm));
}
APD float3 sun_dir(const SunDev& s) { return ld3(s.direction); }
// The per-scene part of the sun functions, evaluated once (k_sun_derive).
APD void sun_derive(SunDev& s) {
  const float cutoff = kPi / 1.95f;
  float3 l = -sun_dir(s);
  float zc = dot(l, f3(0.0f, 1.0f, 0.0f));
  s.it = s.intensity * dm::fmax(0.0f, 1.0f - dm::exp_(-((cutoff - dm::acos_(zc)) / 1.4f)));
  s.cos_size = dm::cos_(s.size * 0.1f);
  float3 bt = perpendicular(l);
  float3 tg = cross(bt, l);
  s.l[0] = l.x; s.l[1] = l.y; s.l[2] = l.z;
  s.bt[0] = bt.x; s.bt[1] = bt.y; s.bt[2] = bt.z;
  s.tg[0] = tg.x; s.tg[1] = tg.y; s.tg[2] = tg.z;
}
APD float sun_intensity(const SunDev& s, float3 direction) {
  float ct = dot(direction, ld3(s.l));
  return s.it * (ct > s.cos_size ? 1.0f : 0.0f);
}
APD float3 direction_to_sun(const SunDev& s, float2 uv) {
  float3 dir = ld3(s.l);
  float h = s.cos_size;
  float phi = 2.0f * kPi * uv.x;
  float z = h + (1.0f - h) * uv.y;
  float st = dm::sqrt_(1.0f - z * z);
  float sp, cp;
  dm::sincos_(phi, &sp, &cp);
  float x = cp * st, y = sp * st;
  return normalize(ld3(s.bt) * x + ld3(s.tg) * y + dir * z);
}
APD float2 inverse_direction_to_sun(const SunDev& s, float3 d) {
  float3 sd = ld3(s.l);
  float z = dot(d, sd), x = dot(d, ld3(s.bt)), y = dot(d, ld3(s.tg));
  float phi = dm::atan2_(y, x);
  float q = phi / (2.0f * kPi);
  float ux = q - truncf(q / 1.0f) * 1.0f;
  float c = s.cos_size;
  return make_float2(ux, (z - c) / (1.0f - c));
}
// Sky::sky: bilinear, repeat-addressed equirect lookup plus the optional sun disk.
APD float3 sky_radiance(const DevScene& sc, float3 d, bool skip_sun) {
  float3 col = f3s(0.0f);
  if (sc.env_w > 0) {
    float phi = dm::atan2_(d.z, d.x) + kPi;
    float theta = dm::acos_(d.y);
    float u = phi / (2.0f * kPi), v = theta * kInvPi;
    float x = u * (float)sc.env_w - 0.5f, y = v * (float)sc.env_h - 0.5f;
    float fx0 = floorf(x), fy0 = floorf(y);
    float tx = x - fx0, ty = y - fy0;
    int ix = dm::f2i(fx0), iy = dm::f2i(fy0);
    int W = (int)sc.env_w, H = (int)sc.env_h;
    int x0 = ((ix % W) + W) % W, x1 = (((ix + 1) % W) + W) % W;
    int y0 = ((iy % H) + H) % H, y1 = (((iy + 1) % H) + H) % H;
    const float* e = sc.env;
    float3 t00 = ld3(e + 3 * ((size_t)y0 * W + x0)), t10 = ld3(e + 3 * ((size_t)y0 * W + x1));
    float3 t01 = ld3(e + 3 * ((size_t)y1 * W + x0)), t11 = ld3(e + 3 * ((size_t)y1 * W + x1));
    float3 a = t00 * (1.0f - tx) + t10 * tx;
    float3 b = t01 * (1.0f - tx) + t11 * tx;
    col = a * (1.0f - ty) + b * ty;
  }
  if (!skip_sun) col = col + (sun_intensity(sc.sun, d) * 1000.0f) * ld3(sc.sun.color);
  return col;
}

// ---- light samples (light_sample.wgsl:4-83, helpers/nee.wgsl:16-115) ----
struct LightSample {
  float2 uv;
  uint32_t inst;  // emissive instance, kU32Max-1 = sun, kU32Max = empty
  uint32_t tri;
};
APD LightSample ls_empty() { return LightSample{make_float2(0.0f, 0.0f), kU32Max, 0}; }
APD bool ls_is_sun(const LightSample& l) { return l.inst == kU32Max - 1; }
APD bool ls_is_empty(const LightSample& l) { return l.inst == kU32Max; }

struct LightEval {
  float3 emission, point;
};

APD void tri_positions(const DevScene& s, const InstanceDev& in, uint32_t tri, float3* p0, float3* p1, float3* p2) {
  uint32_t fi = in.first_index + tri * 3;
  float4 a = s.positions[in.first_vertex + s.indices[fi + 0]];
  float4 b = s.positions[in.first_vertex + s.indices[fi + 1]];
  float4 c = s.positions[in.first_vertex + s.indices[fi + 2]];
  *p0 = f3(a.x, a.y, a.z);
  *p1 = f3(b.x, b.y, b.z);
  *p2 = f3(c.x, c.y, c.z);
}

// `lights` is the scene's emissive_info table, or a copy of it in shared
// memory (the candidate-heavy kernels stage it once per block).
APD LightEval load_eval(const DevScene& s, const LightSample& l, float3 hit, const uint4* lights) {
  if (ls_is_sun(l)) {
    float3 dir = direction_to_sun(s.sun, l.uv);
    return LightEval{sun_intensity(s.sun, dir) * ld3(s.sun.color), dir * 1e6f};
  }
  if (l.inst >= s.num_emissive_instances) return LightEval{f3s(0.0f), f3s(0.0f)};
  const uint4 li = lights[l.inst];
  const uint32_t ntri = li.z;
  const uint32_t tri = l.tri < ntri ? l.tri : ntri - 1;
  const EmissiveTri* et = s.emissive_tris + li.y + tri;
  const float4* q = reinterpret_cast<const float4*>(et);
  float4 a = __ldg(q + 0), b = __ldg(q + 1), c = __ldg(q + 2), nn = __ldg(q + 3), em = __ldg(q + 4);
  float3 p0 = f3(a.x, a.y, a.z), p1 = f3(b.x, b.y, b.z), p2 = f3(c.x, c.y, c.z);
  float bx = 1.0f - l.uv.x - l.uv.y;
  float3 point = p0 * bx + p1 * l.uv.x + p2 * l.uv.y;
  float3 dir = normalize(point - hit);
  float dd = dist(point, hit);
  float cos_out = dm::fmax(-dot(f3(nn.x, nn.y, nn.z), dir), 0.0f);
  float sa = dm::fmin(kTwoPi, cos_out / (sqr(dd) + 0.0001f));
  return LightEval{f3(em.x, em.y, em.z) * sa * 10.0f, point};
}
APD LightEval load_eval(const DevScene& s, const LightSample& l, float3 hit) {
  return load_eval(s, l, hit, s.emissive_info);
}

// First emissive instance whose CDF entry is >= r (the reference scans
// linearly, nee.wgsl:60-61; the CDF is non-decreasing, so the binary search
// returns the same index), or num_emissive_instances when there is none.
APD uint32_t cdf_search(const uint4* lights, uint32_t n, float r) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (r <= __uint_as_float(lights[mid].x)) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

APD LightSample sample_uniform(const DevScene& s, float r0, float r1, float r2, float2 r34, float* pdf,
                               const uint4* lights) {
  float sun_p = s.num_emissive_tris > 0 ? 0.5f : 1.0f;
  if (r0 < sun_p) {
    *pdf = sun_p;
    return LightSample{r34, kU32Max - 1, 0};
  }
  uint32_t i = cdf_search(lights, s.num_emissive_instances, r1);
  if (i < s.num_emissive_instances) {
    const uint4 li = lights[i];
    uint32_t ntri = li.z;
    uint32_t local = dm::f2u(r2 * (float)ntri);
    if (local >= ntri) local = ntri - 1;
    float area = __ldg(&s.emissive_tris[li.y + local].area);
    float p = 1.0f / (float)s.num_emissive_tris;
    p = p / area;
    *pdf = dm::fmax(1e-6f, p * (1.0f - sun_p));
    return LightSample{r34, i, local};
  }
  *pdf = 0.0f;
  return ls_empty();
}
APD LightSample sample_uniform(const DevScene& s, float r0, float r1, float r2, float2 r34, float* pdf) {
  return sample_uniform(s, r0, r1, r2, r34, pdf, s.emissive_info);
}

// ---- reservoirs (di_reservoir.wgsl:6-56, gi_reservoir.wgsl:6-74) ----
struct DiRes {
  float M, W, wsum, phat;
  LightSample s;
};
struct GiRes {
  float M, W, wsum, phat;
  float3 point;
  uint32_t phat_rng;
};
APD bool di_update(DiRes& r, float w, uint32_t& rng, const LightSample& s, float phat) {
  r.wsum = r.wsum + w;
  r.M = r.M + 1.0f;
  if (rnd(rng) <= (w / r.wsum)) {
    r.s = s;
    r.phat = phat;
    return true;
  }
  return false;
}
APD bool gi_update(GiRes& r, float w, uint32_t& rng, float3 point, float phat, uint32_t prng) {
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
APD uint4 di_pack_a(const DiRes& r) {
  return make_uint4(__float_as_uint(r.M), __float_as_uint(r.W), __float_as_uint(r.wsum), __float_as_uint(r.phat));
}
APD uint4 di_pack_b(const DiRes& r) {
  return make_uint4(__float_as_uint(r.s.uv.x), __float_as_uint(r.s.uv.y), r.s.inst, r.s.tri);
}
APD DiRes di_unpack(uint4 a, uint4 b) {
  DiRes r;
  r.M = __uint_as_float(a.x); r.W = __uint_as_float(a.y); r.wsum = __uint_as_float(a.z); r.phat = __uint_as_float(a.w);
  r.s.uv = make_float2(__uint_as_float(b.x), __uint_as_float(b.y));
  r.s.inst = b.z;
  r.s.tri = b.w;
  return r;
}
APD uint4 gi_pack_a(const GiRes& r) {
  return make_uint4(__float_as_uint(r.M), __float_as_uint(r.W), __float_as_uint(r.wsum), __float_as_uint(r.phat));
}
APD uint4 gi_pack_b(const GiRes& r) {
  return make_uint4(__float_as_uint(r.point.x), __float_as_uint(r.point.y), __float_as_uint(r.point.z), r.phat_rng);
}
APD GiRes gi_unpack(uint4 a, uint4 b) {
  GiRes r;
  r.M = __uint_as_float(a.x); r.W = __uint_as_float(a.y); r.wsum = __uint_as_float(a.z); r.phat = __uint_as_float(a.w);
  r.point = f3(__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z));
  r.phat_rng = b.w;
  return r;
}

}  // namespace ap
