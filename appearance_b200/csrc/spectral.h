// Spectral (hero-wavelength) path tracing: the algorithm of the reference's
// CPU tracer, crates/appearance-path-tracer (PathIntegrator::li and
// ::sample_ld, path_integrator.rs:34-307; SampledWavelengths::sample_visible,
// radiometry/spectrum.rs:117-160; SampledSpectrum::to_xyz, spectrum.rs:62-74),
// restated for one thread per path.  Shared, unchanged, by the CUDA kernel
// (csrc/spectral.cu) and the CPU restatement (oracle/oracle_spectral.cpp), so
// both compute the same arithmetic in the same order.
//
// Differences from the reference, each because its data or code is not
// usable here: the CIE 1931 matching functions are the analytic multi-lobe fit
// of Wyman, Sloan and Shirley (JCGT 2013) instead of tabulated data; RGB
// upsampling uses sigmoid polynomials (Jakob and Hanika 2019) fitted by this
// library (spectral_fit.cpp) under a 6504 K blackbody standing in for D65;
// the conductor has a Schlick Fresnel with the upsampled base colour as F0
// instead of gold's tabulated complex index; shading uses the geometric
// normal; samples come from an independent PCG stream instead of ZSobol; the
// environment is looked up with the exact equirect mapping, interpolating the
// spectra of the four nearest texels.  Emissive triangles, which the
// reference tracer lacks, add their emission when a path hits them.
#pragma once

#include <stdint.h>

#include "detmath.h"

#ifdef __CUDACC__
#define SPHD __host__ __device__ __forceinline__
#else
#define SPHD inline
#endif

namespace spec {

constexpr float kLambdaMin = 360.0f, kLambdaMax = 830.0f;
constexpr float kPi = 3.14159265358979323846f;

struct V3 {
  float x, y, z;
};
SPHD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
SPHD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
SPHD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
SPHD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
SPHD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
SPHD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SPHD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
SPHD V3 normalize(V3 a) {
  float l = dm::sqrt_(dot(a, a));
  return l > 0.0f ? a * (1.0f / l) : a;
}
SPHD float dist(V3 a, V3 b) { return dm::sqrt_(dot(a - b, a - b)); }

// Four wavelengths and their values (SampledWavelengths / SampledSpectrum).
struct S4 {
  float v[4];
};
SPHD S4 s4(float a) { return S4{{a, a, a, a}}; }
SPHD S4 operator*(S4 a, S4 b) { return S4{{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}}; }
SPHD S4 operator*(S4 a, float s) { return S4{{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
SPHD S4 operator+(S4 a, S4 b) { return S4{{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}}; }
SPHD float max4(S4 a) { return dm::fmax(dm::fmax(a.v[0], a.v[1]), dm::fmax(a.v[2], a.v[3])); }
SPHD bool nonzero(S4 a) { return a.v[0] != 0.0f || a.v[1] != 0.0f || a.v[2] != 0.0f || a.v[3] != 0.0f; }

// ---- sampling --------------------------------------------------------------

SPHD uint32_t pcg(uint32_t v) {
  uint32_t state = v * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
struct Rng {
  uint32_t s;
  SPHD float next() {
    s = pcg(s);
    return (float)(s >> 8) * (1.0f / 16777216.0f);
  }
};
SPHD Rng rng_for(uint32_t pixel, uint32_t sample, uint32_t seed) {
  return Rng{pcg(pixel * 9781u ^ pcg(sample * 6271u + seed * 28411u + 1u))};
}

// Visible-wavelength importance sampling (pbrt-v4; spectrum.rs:155-180):
// lambda(u) = 538 - 138.888889 atanh(0.85691062 - 1.82750197 u),
// pdf(lambda) = 0.0039398042 / cosh^2(0.0072 (lambda - 538)) on [360, 830].
SPHD float sample_visible_wavelength(float u) {
  float x = 0.85691062f - 1.82750197f * u;
  float at = 0.5f * dm::log_((1.0f + x) / (1.0f - x));
  return 538.0f - 138.888889f * at;
}
SPHD float visible_wavelength_pdf(float l) {
  if (!(l >= kLambdaMin && l <= kLambdaMax)) return 0.0f;
  float a = 0.0072f * (l - 538.0f);
  float e = dm::exp_(a), ei = dm::exp_(-a);
  float c = 0.5f * (e + ei);
  return 0.0039398042f / (c * c);
}
struct Wavelengths {
  S4 lambda, pdf;
};
SPHD Wavelengths sample_visible(float u) {  // spectrum.rs:117-131
  Wavelengths w;
  for (int i = 0; i < 4; ++i) {
    float up = u + (float)i / 4.0f;
    if (up > 1.0f) up -= 1.0f;
    w.lambda.v[i] = sample_visible_wavelength(up);
    w.pdf.v[i] = visible_wavelength_pdf(w.lambda.v[i]);
  }
  return w;
}

// ---- colour ------------------------------------------------------------------

// CIE 1931 2-degree matching functions, multi-lobe Gaussian fit (Wyman, Sloan
// and Shirley, "Simple Analytic Approximations to the CIE XYZ Color Matching
// Functions", JCGT 2(2), 2013).
SPHD float lobe(float l, float mu, float s1, float s2) {
  float t = (l - mu) / (l < mu ? s1 : s2);
  return dm::exp_(-0.5f * t * t);
}
SPHD float cie_x(float l) {
  return 1.056f * lobe(l, 599.8f, 37.9f, 31.0f) + 0.362f * lobe(l, 442.0f, 16.0f, 26.7f) -
         0.065f * lobe(l, 501.1f, 20.4f, 26.2f);
}
SPHD float cie_y(float l) { return 0.821f * lobe(l, 568.8f, 46.9f, 40.5f) + 0.286f * lobe(l, 530.9f, 16.3f, 31.1f); }
SPHD float cie_z(float l) { return 1.217f * lobe(l, 437.0f, 11.8f, 36.0f) + 0.681f * lobe(l, 459.0f, 26.0f, 13.8f); }
// Integral of cie_y over [360, 830] nm (trapezoid, 0.5 nm steps, double), the
// normaliser of to_xyz (spectrum.rs:62-74).
constexpr float kCieYIntegral = 106.922074f;

// Sigmoid polynomial (Jakob and Hanika 2019): s(lambda) = sigmoid(c0 x^2 +
// c1 x + c2), x = (lambda - 360) / 470, sigmoid(t) = 1/2 + t / (2 sqrt(1 + t^2)).
SPHD float sigmoid_poly(const float* c, float l) {
  float x = (l - kLambdaMin) * (1.0f / (kLambdaMax - kLambdaMin));
  float t = (c[0] * x + c[1]) * x + c[2];
  return 0.5f + t / (2.0f * dm::sqrt_(1.0f + t * t));
}
// Blackbody radiance at 6504 K (Planck), normalised to 1 at 560 nm: the
// illuminant of the RGB upsampling (the reference uses D65).
// B(l) / B(560) = (560 / l)^5 (exp(x560) - 1) / (exp(x) - 1), x = c2 / (l T),
// c2 = hc/k = 1.4387769e7 nm K.
SPHD float illuminant(float l) {
  const float kC2T = 1.4387769e7f / 6504.0f;
  float r = 560.0f / l, r2 = r * r;
  return r2 * r2 * r * (dm::exp_(kC2T / 560.0f) - 1.0f) / (dm::exp_(kC2T / l) - 1.0f);
}

// Albedo (RgbAlbedoSpectrum) and emission (RgbIlluminantSpectrum: scale x
// sigmoid x illuminant) samples at the four wavelengths.
SPHD S4 albedo4(const float* c, const S4& lambda) {
  S4 r;
  for (int i = 0; i < 4; ++i) r.v[i] = sigmoid_poly(c, lambda.v[i]);
  return r;
}
SPHD S4 illuminant4(const S4& lambda) {
  S4 r;
  for (int i = 0; i < 4; ++i) r.v[i] = illuminant(lambda.v[i]);
  return r;
}
// emission4 with the illuminant at the four wavelengths given (illuminant4):
// the same products in the same order, for callers evaluating several spectra
// at one set of wavelengths.
SPHD S4 emission4_ill(const float* c, float scale, const S4& lambda, const S4& ill) {
  S4 r;
  for (int i = 0; i < 4; ++i) r.v[i] = scale * sigmoid_poly(c, lambda.v[i]) * ill.v[i];
  return r;
}
SPHD S4 emission4(const float* c, float scale, const S4& lambda) {
  return emission4_ill(c, scale, lambda, illuminant4(lambda));
}

// Unbounded RGB (an emitter's radiance, an environment texel, a predicted
// radiance) as an illuminant spectrum: the sigmoid coefficients of
// rgb / (2 max) interpolated trilinearly in a 33^3 table over rgb / max
// (`tab`, 3 floats per entry, built by spectral_fit.cpp), and the scale
// 2 max(rgb) x norm (RgbIlluminantSpectrum).  out: 3 coefficients, scale.
SPHD void illum_lookup(const float* tab, float norm, const float rgb[3], float out[4]) {
  const float m = dm::fmax(rgb[0], dm::fmax(rgb[1], rgb[2]));
  if (!(m > 0.0f)) {
    out[0] = 0.0f;
    out[1] = 0.0f;
    out[2] = -1e4f;  // sigmoid -> 0
    out[3] = 0.0f;
    return;
  }
  float f[3];
  int i0[3];
  for (int k = 0; k < 3; ++k) {
    const float x = dm::clamp(rgb[k] / m, 0.0f, 1.0f) * 32.0f;
    i0[k] = (int)x < 31 ? (int)x : 31;
    f[k] = x - (float)i0[k];
  }
  for (int c = 0; c < 3; ++c) {
    float v = 0.0f;
    for (int corner = 0; corner < 8; ++corner) {
      const int dr = corner & 1, dg = (corner >> 1) & 1, db = corner >> 2;
      const float w = (dr ? f[0] : 1.0f - f[0]) * (dg ? f[1] : 1.0f - f[1]) * (db ? f[2] : 1.0f - f[2]);
      v = v + w * tab[3 * (((i0[2] + db) * 33 + (i0[1] + dg)) * 33 + (i0[0] + dr)) + c];
    }
    out[c] = v;
  }
  out[3] = 2.0f * m * norm;
}

// XYZ of one path's spectral radiance (to_xyz) and linear sRGB.
SPHD V3 to_xyz(S4 L, const Wavelengths& w) {
  float x = 0.0f, y = 0.0f, z = 0.0f;
  for (int i = 0; i < 4; ++i) {
    float p = w.pdf.v[i];
    float li = p != 0.0f ? L.v[i] / p : 0.0f;
    x = x + li * cie_x(w.lambda.v[i]);
    y = y + li * cie_y(w.lambda.v[i]);
    z = z + li * cie_z(w.lambda.v[i]);
  }
  return v3(x, y, z) * (0.25f / kCieYIntegral);
}
SPHD V3 xyz_to_srgb(V3 c) {
  return v3(3.2404542f * c.x - 1.5371385f * c.y - 0.4985314f * c.z,
            -0.9692660f * c.x + 1.8760108f * c.y + 0.0415560f * c.z,
            0.0556434f * c.x - 0.2040259f * c.y + 1.0572252f * c.z);
}

// ---- materials and BSDFs ---------------------------------------------------

// Per material: albedo sigmoid coefficients (3), metallic; emission sigmoid
// coefficients (3), emission scale; transmission.
struct Material {
  float albedo[3], metallic;
  float emit[3], emit_scale;
  float transmission, pad0, pad1, pad2;
};

struct Frame {
  V3 t, b, n;
};
SPHD Frame frame_of(V3 n) {  // orthonormal basis (Duff et al. 2017)
  float sgn = n.z >= 0.0f ? 1.0f : -1.0f;
  float a = -1.0f / (sgn + n.z);
  float bb = n.x * n.y * a;
  Frame f;
  f.t = v3(1.0f + sgn * n.x * n.x * a, sgn * bb, -sgn * n.x);
  f.b = v3(bb, sgn + n.y * n.y * a, -n.y);
  f.n = n;
  return f;
}
SPHD V3 to_local(const Frame& f, V3 v) { return v3(dot(v, f.t), dot(v, f.b), dot(v, f.n)); }
SPHD V3 to_world(const Frame& f, V3 v) { return f.t * v.x + f.b * v.y + f.n * v.z; }

enum : uint32_t { BX_DIFFUSE = 0, BX_CONDUCTOR = 1, BX_DIELECTRIC = 2 };
constexpr float kConductorAlpha = 0.04f;  // ThrowbridgeReitzDistribution::new(0.04, 0.04)
constexpr float kDielectricEta = 1.5f;

struct Bsdf {
  uint32_t kind;
  S4 albedo;  // diffuse reflectance or conductor F0
  Frame fr;   // n faces the outgoing direction for diffuse and conductor
};

// Trowbridge-Reitz (GGX), isotropic alpha, local coordinates (z = normal).
SPHD float tr_d(V3 m, float a) {
  float c2 = m.z * m.z;
  if (!(c2 > 0.0f)) return 0.0f;
  float s2 = dm::fmax(0.0f, 1.0f - c2);
  float e = 1.0f + s2 / (c2 * a * a);
  return 1.0f / (kPi * a * a * c2 * c2 * e * e);
}
SPHD float tr_lambda(V3 w, float a) {
  float c2 = w.z * w.z, s2 = dm::fmax(0.0f, 1.0f - c2);
  if (c2 == 0.0f) return 0.0f;
  float t2 = s2 / c2;
  return (dm::sqrt_(1.0f + a * a * t2) - 1.0f) * 0.5f;
}
SPHD float tr_g(V3 wo, V3 wi, float a) { return 1.0f / (1.0f + tr_lambda(wo, a) + tr_lambda(wi, a)); }
SPHD float tr_g1(V3 w, float a) { return 1.0f / (1.0f + tr_lambda(w, a)); }
// Visible-normal sampling (Heitz 2018), wo in the upper hemisphere.
SPHD V3 tr_sample_wm(V3 wo, float a, float u0, float u1) {
  V3 wh = normalize(v3(a * wo.x, a * wo.y, wo.z));
  V3 t1 = wh.z < 0.99999f ? normalize(cross(v3(0.0f, 0.0f, 1.0f), wh)) : v3(1.0f, 0.0f, 0.0f);
  V3 t2 = cross(wh, t1);
  float r = dm::sqrt_(u0), phi = 2.0f * kPi * u1;
  float sp, cp;
  dm::sincos_(phi, &sp, &cp);
  float p1 = r * cp, p2 = r * sp;
  float s = 0.5f * (1.0f + wh.z);
  p2 = (1.0f - s) * dm::sqrt_(dm::fmax(0.0f, 1.0f - p1 * p1)) + s * p2;
  float p3 = dm::sqrt_(dm::fmax(0.0f, 1.0f - p1 * p1 - p2 * p2));
  V3 nh = t1 * p1 + t2 * p2 + wh * p3;
  return normalize(v3(a * nh.x, a * nh.y, dm::fmax(1e-6f, nh.z)));
}
SPHD float tr_pdf_wm(V3 wo, V3 wm, float a) {  // D_wo(wm)
  return tr_g1(wo, a) / dm::fabs_(wo.z) * tr_d(wm, a) * dm::fabs_(dot(wo, wm));
}
SPHD S4 schlick(S4 f0, float c) {
  float m = dm::fmax(0.0f, 1.0f - c), m5 = m * m * m * m * m;
  S4 r;
  for (int i = 0; i < 4; ++i) r.v[i] = f0.v[i] + (1.0f - f0.v[i]) * m5;
  return r;
}
SPHD float fresnel_dielectric(float ci, float eta) {
  ci = dm::clamp(ci, -1.0f, 1.0f);
  if (ci < 0.0f) {
    eta = 1.0f / eta;
    ci = -ci;
  }
  float s2i = 1.0f - ci * ci, s2t = s2i / (eta * eta);
  if (s2t >= 1.0f) return 1.0f;
  float ct = dm::sqrt_(1.0f - s2t);
  float rpar = (eta * ci - ct) / (eta * ci + ct), rperp = (ci - eta * ct) / (ci + eta * ct);
  return 0.5f * (rpar * rpar + rperp * rperp);
}

// f(wo, wi) for the non-specular lobes (diffuse, conductor), world directions.
SPHD S4 bsdf_f(const Bsdf& b, V3 wow, V3 wiw) {
  V3 wo = to_local(b.fr, wow), wi = to_local(b.fr, wiw);
  if (wo.z <= 0.0f || wi.z <= 0.0f) return s4(0.0f);
  if (b.kind == BX_DIFFUSE) return b.albedo * (1.0f / kPi);
  if (b.kind == BX_CONDUCTOR) {
    V3 wm = normalize(wo + wi);
    float a = kConductorAlpha;
    S4 F = schlick(b.albedo, dm::fabs_(dot(wo, wm)));
    return F * (tr_d(wm, a) * tr_g(wo, wi, a) / (4.0f * wo.z * wi.z));
  }
  return s4(0.0f);
}
SPHD float bsdf_pdf(const Bsdf& b, V3 wow, V3 wiw) {
  V3 wo = to_local(b.fr, wow), wi = to_local(b.fr, wiw);
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  if (b.kind == BX_DIFFUSE) return wi.z * (1.0f / kPi);
  if (b.kind == BX_CONDUCTOR) {
    V3 wm = normalize(wo + wi);
    return tr_pdf_wm(wo, wm, kConductorAlpha) / (4.0f * dm::fabs_(dot(wo, wm)));
  }
  return 0.0f;
}

struct BsdfSample {
  S4 f;
  V3 wi;
  float pdf, eta;
  bool specular, transmission, ok;
};
SPHD BsdfSample bsdf_sample(const Bsdf& b, V3 wow, float uc, float u0, float u1) {
  BsdfSample s;
  s.ok = false;
  s.specular = false;
  s.transmission = false;
  s.eta = 1.0f;
  s.pdf = 0.0f;
  s.f = s4(0.0f);
  s.wi = v3(0.0f, 0.0f, 0.0f);
  V3 wo = to_local(b.fr, wow);
  if (b.kind == BX_DIFFUSE) {
    if (wo.z <= 0.0f) return s;
    float r = dm::sqrt_(u0), phi = 2.0f * kPi * u1, sp, cp;
    dm::sincos_(phi, &sp, &cp);
    V3 wi = v3(r * cp, r * sp, dm::sqrt_(dm::fmax(0.0f, 1.0f - u0)));
    s.pdf = wi.z * (1.0f / kPi);
    if (!(s.pdf > 0.0f)) return s;
    s.f = b.albedo * (1.0f / kPi);
    s.wi = to_world(b.fr, wi);
    s.ok = true;
    return s;
  }
  if (b.kind == BX_CONDUCTOR) {
    if (wo.z <= 0.0f) return s;
    const float a = kConductorAlpha;
    V3 wm = tr_sample_wm(wo, a, u0, u1);
    V3 wi = wm * (2.0f * dot(wo, wm)) - wo;
    if (wi.z <= 0.0f) return s;
    s.pdf = tr_pdf_wm(wo, wm, a) / (4.0f * dm::fabs_(dot(wo, wm)));
    if (!(s.pdf > 0.0f)) return s;
    S4 F = schlick(b.albedo, dm::fabs_(dot(wo, wm)));
    s.f = F * (tr_d(wm, a) * tr_g(wo, wi, a) / (4.0f * wo.z * wi.z));
    s.wi = to_world(b.fr, wi);
    s.ok = true;
    return s;
  }
  // smooth dielectric (DielectricBxdf with alpha 0), normal from the surface
  const float eta = kDielectricEta;
  float R = fresnel_dielectric(wo.z, eta), T = 1.0f - R;
  if (uc < R / (R + T)) {
    V3 wi = v3(-wo.x, -wo.y, wo.z);
    s.pdf = R / (R + T);
    s.f = s4(R / dm::fabs_(wi.z));
    s.wi = to_world(b.fr, wi);
    s.specular = true;
    s.ok = true;
    return s;
  }
  float etap = wo.z > 0.0f ? eta : 1.0f / eta;
  V3 n = wo.z > 0.0f ? v3(0.0f, 0.0f, 1.0f) : v3(0.0f, 0.0f, -1.0f);
  float ci = dot(n, wo), s2i = dm::fmax(0.0f, 1.0f - ci * ci), s2t = s2i / (etap * etap);
  if (s2t >= 1.0f) return s;
  float ct = dm::sqrt_(1.0f - s2t);
  V3 wi = -wo * (1.0f / etap) + n * (ci / etap - ct);
  s.pdf = T / (R + T);
  s.f = s4(T / dm::fabs_(wi.z) / (etap * etap));
  s.wi = to_world(b.fr, wi);
  s.eta = etap;
  s.specular = true;
  s.transmission = true;
  s.ok = true;
  return s;
}

SPHD float power_heuristic(float f, float g) {
  float a = f * f, bb = g * g;
  return a + bb > 0.0f ? a / (a + bb) : 0.0f;
}

// ---- scene access and the integrator ----------------------------------------

// Sun (DistantLight, geometry_resources.rs:52-64): direction of travel,
// radiance sigmoid coefficients and scale; scene radius for the shadow ray.
struct Sun {
  float dir[3], scale;
  float coef[3], radius;
};

struct Hit {
  float t;
  uint32_t tri;
};

// Equirect lookup: u = (atan2(z, x) + pi) / 2pi, v = acos(y) / pi
// (sampling/mod.rs:65-70); the spectra of the four nearest texel centres are
// interpolated bilinearly (clamped).
template <class Geo>
SPHD S4 env_le(const Geo& g, V3 d, const S4& lambda) {
  if (g.env_w == 0) return s4(0.0f);
  float u = (dm::atan2_(d.z, d.x) + kPi) * (1.0f / (2.0f * kPi));
  float v = dm::acos_(dm::clamp(d.y, -1.0f, 1.0f)) * (1.0f / kPi);
  float x = u * (float)g.env_w - 0.5f, y = v * (float)g.env_h - 0.5f;
  float fx = dm::floor_(x), fy = dm::floor_(y);
  float ax = x - fx, ay = y - fy;
  int x0 = (int)fx, y0 = (int)fy;
  const S4 ill = illuminant4(lambda);
  S4 acc = s4(0.0f);
  for (int k = 0; k < 4; ++k) {
    int xi = x0 + (k & 1), yi = y0 + (k >> 1);
    xi = xi < 0 ? 0 : (xi >= (int)g.env_w ? (int)g.env_w - 1 : xi);
    yi = yi < 0 ? 0 : (yi >= (int)g.env_h ? (int)g.env_h - 1 : yi);
    float wgt = ((k & 1) ? ax : 1.0f - ax) * ((k >> 1) ? ay : 1.0f - ay);
    float c[4];
    g.env_texel((uint32_t)yi * g.env_w + (uint32_t)xi, c);
    acc = acc + emission4_ill(c, c[3], lambda, ill) * wgt;
  }
  return acc * g.env_scale;
}

// State of one path of PathIntegrator::li between vertices.
struct PathState {
  S4 L, beta;
  float eta_scale;
  int depth;
  Rng rng;
};
SPHD PathState path_start(Rng rng) { return PathState{s4(0.0f), s4(1.0f), 1.0f, 0, rng}; }

// Shadow ray of the distant light: its contribution c is added to L unless
// the segment (o, d, [0, tmax]) is occluded.
struct ShadowRay {
  V3 o, d;
  float tmax;
  S4 c;
};

// One vertex of PathIntegrator::li (path_integrator.rs:103-307): `hit` is the
// closest hit of the ray (o, d), or null when it escaped.  Adds emission (or
// the environment on escape), sets *shadow and fills sh for the light sample,
// samples the BSDF and applies Russian roulette.  Returns true when the path
// goes on along the updated (o, d).  li below runs it in a loop; the GPU runs
// it as one stage of a wavefront.
template <class Geo>
SPHD bool path_vertex(const Geo& g, V3& o, V3& d, const Hit* h, const S4& lambda, PathState& ps, int max_depth,
                      bool* shadow, ShadowRay* sh) {
  *shadow = false;
  if (!h) {  // escaped: the environment (not in the light sampler: weight 1)
    ps.L = ps.L + ps.beta * env_le(g, d, lambda);
    return false;
  }
  V3 p0, p1, p2;
  g.tri(h->tri, &p0, &p1, &p2);
  const Material& m = g.material(h->tri);
  V3 hit = o + d * h->t;
  V3 ng = normalize(cross(p1 - p0, p2 - p0));
  V3 wo = -d;
  if (m.emit_scale > 0.0f && dot(ng, wo) > 0.0f) ps.L = ps.L + ps.beta * emission4(m.emit, m.emit_scale, lambda);
  ps.depth += 1;
  if (ps.depth > max_depth) return false;
  Bsdf b;
  if (m.metallic > 0.9f) b.kind = BX_CONDUCTOR;
  else if (m.transmission > 0.0f) b.kind = BX_DIELECTRIC;
  else b.kind = BX_DIFFUSE;
  b.albedo = albedo4(m.albedo, lambda);
  V3 n = (b.kind != BX_DIELECTRIC && dot(ng, wo) < 0.0f) ? -ng : ng;
  b.fr = frame_of(n);
  if (b.kind != BX_DIELECTRIC && g.sun.scale > 0.0f) {  // sample_ld: the distant light (delta: no MIS)
    V3 wi = v3(-g.sun.dir[0], -g.sun.dir[1], -g.sun.dir[2]);
    S4 f = bsdf_f(b, wo, wi) * dm::fabs_(dot(wi, n));
    if (nonzero(f)) {
      V3 lp = hit + wi * (2.0f * g.sun.radius);
      sh->o = hit + wi * 0.0001f;
      sh->d = wi;
      sh->tmax = dist(hit, lp);
      sh->c = ps.beta * (f * emission4(g.sun.coef, g.sun.scale, lambda));
      *shadow = true;
    }
  }
  // three draws in a fixed order (argument evaluation order is unspecified)
  const float uc = ps.rng.next();
  const float u0 = ps.rng.next();
  const float u1 = ps.rng.next();
  BsdfSample s = bsdf_sample(b, wo, uc, u0, u1);
  if (!s.ok) return false;
  ps.beta = ps.beta * (s.f * (dm::fabs_(dot(s.wi, n)) / s.pdf));
  if (s.transmission) ps.eta_scale = ps.eta_scale * (s.eta * s.eta);
  o = hit + s.wi * 0.0001f;
  d = s.wi;
  S4 rr = ps.beta * ps.eta_scale;
  if (max4(rr) < 1.0f && ps.depth > 1) {
    float q = dm::fmax(1.0f - max4(rr), 0.0f);
    if (ps.rng.next() < q) return false;
    ps.beta = ps.beta * (1.0f / (1.0f - q));
  }
  return true;
}

// PathIntegrator::li for one camera ray: at most max_depth + 1 closest-hit
// rays, each followed by its vertex and the vertex's shadow ray.
template <class Geo>
SPHD S4 li(const Geo& g, V3 o, V3 d, const S4& lambda, Rng& rng, int max_depth) {
  PathState ps = path_start(rng);
  for (int k = 0; k <= max_depth; ++k) {
    Hit h;
    const bool hit = g.closest(o, d, 1e30f, h);
    bool shadow;
    ShadowRay sh = {};
    const bool more = path_vertex(g, o, d, hit ? &h : nullptr, lambda, ps, max_depth, &shadow, &sh);
    if (shadow && !g.occluded(sh.o, sh.d, sh.tmax)) ps.L = ps.L + sh.c;
    if (!more) break;
  }
  rng = ps.rng;
  return ps.L;
}

// Column-major 4x4 matrix times (x, y, z, w), summed in a fixed order.
SPHD void mul4(const float* m, float x, float y, float z, float w, float* o) {
  for (int r = 0; r < 4; ++r) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

// Camera ray through the centre of pixel (x, y): the uv of lib.rs:138-142 and
// the camera of path_tracer.rs:42-45 (direction normalised).
SPHD void camera_ray(const float* inv_view, const float* inv_proj, uint32_t x, uint32_t y, uint32_t W, uint32_t H,
                     V3* o, V3* d) {
  float ux = (((float)x + 0.5f) / (float)W) * 2.0f - 1.0f;
  float uy = (((float)y + 0.5f) / (float)H) * 2.0f - 1.0f;
  uy = -uy;
  float oo[4], t[4], dd[4];
  mul4(inv_view, 0.0f, 0.0f, 0.0f, 1.0f, oo);
  mul4(inv_proj, ux, uy, 1.0f, 1.0f, t);
  V3 tn = normalize(v3(t[0], t[1], t[2]));
  mul4(inv_view, tn.x, tn.y, tn.z, 0.0f, dd);
  *o = v3(oo[0], oo[1], oo[2]);
  *d = normalize(v3(dd[0], dd[1], dd[2]));
}

// Linear sRGB of one sample of pixel (x, y): the camera ray, the wavelengths
// from the sample's first random number (path_tracer.rs:59), li, the XYZ
// sensor and the sRGB matrix.
template <class Geo>
SPHD V3 pixel_sample(const Geo& g, const float* inv_view, const float* inv_proj, uint32_t x, uint32_t y, uint32_t W,
                     uint32_t H, uint32_t sample, uint32_t seed, int max_depth) {
  V3 o, d;
  camera_ray(inv_view, inv_proj, x, y, W, H, &o, &d);
  Rng rng = rng_for(y * W + x, sample, seed);
  Wavelengths w = sample_visible(rng.next());
  S4 L = li(g, o, d, w.lambda, rng, max_depth);
  return xyz_to_srgb(to_xyz(L, w));
}

}  // namespace spec
