// Spectral (hero-wavelength) path tracing: the estimator of the reference's
// CPU tracer, crates/appearance-path-tracer, restated for one path vertex at a
// time so that the CUDA wavefront (csrc/spectral.cu) can run it as a stage:
//
//   PathIntegrator::li and ::sample_ld      path_integrator.rs:34-307
//   ZSobolSampler (one 1-spp frame per sample, seed = frame index)
//                                           sampling/zsobol_sampler.rs:43-152,
//                                           math/sobol.rs:3-22, math/random.rs:69-152
//   SampledWavelengths::sample_visible      radiometry/spectrum.rs:117-160
//   Diffuse / conductor (gold) / smooth dielectric BxDFs, Trowbridge-Reitz
//                                           reflectance/*.rs
//   DistantLight, InfiniteLight::le / pdf_li (compensated distribution)
//                                           light_sources/*.rs, sampling/piecewise_constant.rs
//   interpolated shading normal             geometry_resources.rs:229-282
//   camera ray and sampler pixel            path_tracer.rs:28-68, lib.rs:138-142
//
// Substitutions, each because the reference's data or code cannot be used
// here: RGB upsampling uses sigmoid polynomials (Jakob and Hanika 2019)
// fitted by this library (spectral_fit.cpp; the reference's tables come from
// a crate missing from its repository) under a 6504 K blackbody standing in
// for D65; the output colour is the XYZ of the four wavelengths (CIE 1931
// analytic fit of Wyman, Sloan and Shirley, JCGT 2013) to linear sRGB in place
// of the film's Canon EOS 100D sensor model; wavelength sampling evaluates its
// analytic functions instead of lookup tables of them (and without the 470x
// factor those tables put on the pdf); emissive triangles, which the
// reference tracer lacks, add their emission when a path hits their front
// face.  Reference defects kept, because the contract is the reference's
// estimator: the concentric disk mapping with radius and angle exchanged,
// conductor Fresnel terms added as magnitudes, the x-major flattening of the
// environment's sampling distribution, and the escaped-path MIS weight
// against an environment the light sampler never samples.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define SPHD __host__ __device__ __forceinline__
#else
#define SPHD inline
#endif

namespace spec {

constexpr float kLambdaMin = 360.0f, kLambdaMax = 830.0f;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kPiOver2 = 1.57079632679489661923f;
constexpr float kPiOver4 = 0.785398163397448309616f;

struct V3 {
  float x, y, z;
};
SPHD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
SPHD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
SPHD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
SPHD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
SPHD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
SPHD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
SPHD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SPHD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
SPHD float length(V3 a) { return sqrtf(dot(a, a)); }
SPHD V3 normalize(V3 a) { return a * (1.0f / length(a)); }  // glam: v * (1 / |v|)

// Four wavelengths and their values (SampledWavelengths / SampledSpectrum).
struct S4 {
  float v[4];
};
SPHD S4 s4(float a) { return S4{{a, a, a, a}}; }
SPHD S4 operator*(S4 a, S4 b) { return S4{{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}}; }
SPHD S4 operator*(S4 a, float s) { return S4{{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
SPHD S4 operator/(S4 a, float s) { return S4{{a.v[0] / s, a.v[1] / s, a.v[2] / s, a.v[3] / s}}; }
SPHD S4 operator+(S4 a, S4 b) { return S4{{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}}; }
SPHD float fmax_nan(float a, float b) { return a > b ? a : (b == b ? b : a); }  // f32::max
SPHD float max4(S4 a) { return fmax_nan(fmax_nan(fmax_nan(a.v[0], a.v[1]), a.v[2]), a.v[3]); }
SPHD bool contributes(S4 a) {  // SampledSpectrum::has_contribution: |s|^2 > 0
  return a.v[0] * a.v[0] + a.v[1] * a.v[1] + a.v[2] * a.v[2] + a.v[3] * a.v[3] > 0.0f;
}
SPHD float sqr(float x) { return x * x; }
SPHD float safe_sqrt(float x) { return sqrtf(fmax_nan(x, 0.0f)); }
SPHD float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
SPHD uint32_t f2u_sat(float x) {  // `as u32`: saturating, NaN -> 0
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)x;
}

// ---- ZSobol sampler ----------------------------------------------------------

SPHD uint32_t rev32(uint32_t n) {
#ifdef __CUDA_ARCH__
  return __brev(n);
#else
  n = (n >> 16) | (n << 16);
  n = ((n & 0x00ff00ffu) << 8) | ((n & 0xff00ff00u) >> 8);
  n = ((n & 0x0f0f0f0fu) << 4) | ((n & 0xf0f0f0f0u) >> 4);
  n = ((n & 0x33333333u) << 2) | ((n & 0xccccccccu) >> 2);
  return ((n & 0x55555555u) << 1) | ((n & 0xaaaaaaaau) >> 1);
#endif
}
SPHD uint64_t mix_bits(uint64_t v) {  // math/random.rs:69-76
  v ^= v >> 31;
  v *= 0x7fb5d329728ea185ull;
  v ^= v >> 27;
  v *= 0x81dadef4bc2dd44dull;
  return v ^ (v >> 33);
}
SPHD uint32_t owen_scramble(uint32_t v, uint32_t seed) {  // FastOwenScrambler, math/random.rs:140-152
  v = rev32(v);
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return rev32(v);
}
// Sobol dimensions 0 and 1 (math/sobol.rs): dimension 0 reverses the index's
// bits; dimension 1 is the generator matrix of the primitive polynomial x + 1,
// column i = m_i << (31 - i) with m_0 = 1, m_i = m_{i-1} xor 2 m_{i-1}.
SPHD uint32_t sobol_bits(uint32_t a, int dim) {
  if (dim == 0) return rev32(a);
  uint32_t v = 0, m = 1;
  for (int i = 0; i < 32 && a; ++i, a >>= 1) {
    if (a & 1u) v ^= m << (31 - i);
    m ^= m << 1;
  }
  return v;
}
SPHD float sobol_sample(uint32_t a, int dim, uint32_t scramble) {
  return (float)owen_scramble(sobol_bits(a, dim), scramble) * 2.3283064e-10f;
}
SPHD uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
SPHD uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  return k ^ (k >> 33);
}
// h1 of MurmurHash3 x64_128 (seed 0) over the 12 bytes (dimension as u32,
// seed as u64), little-endian: the key ZSobolSampler hashes per draw.
SPHD uint64_t hash_dimension(uint32_t dim, uint64_t seed) {
  const uint64_t c1 = 0x87c37b91114253d5ull, c2 = 0x4cf5ad432745937full;
  uint64_t k1 = (uint64_t)dim | (seed << 32), k2 = seed >> 32;
  uint64_t h1 = 0, h2 = 0;
  k2 *= c2;
  k2 = rotl64(k2, 33);
  k2 *= c1;
  h2 ^= k2;
  k1 *= c1;
  k1 = rotl64(k1, 31);
  k1 *= c2;
  h1 ^= k1;
  h1 ^= 12u;
  h2 ^= 12u;
  h1 += h2;
  h2 += h1;
  h1 = fmix64(h1);
  h2 = fmix64(h2);
  return h1 + h2;
}
SPHD uint32_t spread2(uint32_t x) {  // left_shift_2 of a 16-bit value
  x &= 0xffffu;
  x = (x | (x << 8)) & 0x00ff00ffu;
  x = (x | (x << 4)) & 0x0f0f0f0fu;
  x = (x | (x << 2)) & 0x33333333u;
  return (x | (x << 1)) & 0x55555555u;
}
SPHD uint32_t morton2(uint32_t x, uint32_t y) { return (spread2(y) << 1) | spread2(x); }  // x, y < 65536
// The 24 permutations of four base-4 digits in ZSobolSampler's order, one per
// byte (digit d of permutation p at bits 2d of byte p).
SPHD uint32_t permuted_digit(uint32_t p, uint32_t d) {
  const uint64_t k0 = 0xb1e19c6c78d8b4e4ull, k1 = 0x72d236c68d2d39c9ull, k2 = 0x93634b1b87271e4eull;
  const uint64_t w = p < 8 ? k0 : (p < 16 ? k1 : k2);
  return (uint32_t)(w >> (8 * (p & 7) + 2 * d)) & 3u;
}
// Base-4 digits of a 1-spp ZSobol stream at resolution (W, H).
SPHD uint32_t zsobol_digits(uint32_t W, uint32_t H) {
  uint32_t r = (W > H ? W : H) - 1;
  r |= r >> 1;
  r |= r >> 2;
  r |= r >> 4;
  r |= r >> 8;
  r |= r >> 16;
  return (uint32_t)log2f((float)(r + 1));
}
// One path's stream: Morton index of its sampler pixel (1 spp: no sample
// bits), the frame seed, the next dimension.
struct ZSobol {
  uint32_t morton;
  uint32_t digits;
  uint64_t seed;
  uint32_t dim;

  SPHD uint32_t index() const {  // ZSobolSampler::get_sample_idx with log2 spp 0
    uint32_t idx = 0;
    for (int i = (int)digits - 1; i >= 0; --i) {
      const uint32_t shift = 2u * (uint32_t)i;
      const uint32_t digit = (morton >> shift) & 3u;
      const uint64_t higher = (uint64_t)(morton >> shift >> 2);
      const uint32_t p = (uint32_t)((mix_bits(higher ^ (0x55555555ull * (uint64_t)dim)) >> 24) % 24u);
      idx |= permuted_digit(p, digit) << shift;
    }
    return idx;
  }
  SPHD float get1d() {
    const uint32_t a = index();
    dim += 1;
    return sobol_sample(a, 0, (uint32_t)hash_dimension(dim, seed));
  }
  SPHD void get2d(float* u0, float* u1) {
    const uint32_t a = index();
    dim += 2;
    const uint64_t h = hash_dimension(dim, seed);
    *u0 = sobol_sample(a, 0, (uint32_t)h);
    *u1 = sobol_sample(a, 1, (uint32_t)(h >> 32));
  }
};
// The sampler pixel of image pixel (x, y): path_tracer.rs:52-56 maps the
// vertically flipped uv back to pixels.
SPHD void sampler_pixel(uint32_t x, uint32_t y, uint32_t W, uint32_t H, uint32_t* px, uint32_t* py) {
  const float ux = ((float)x + 0.5f) / (float)W * 2.0f - 1.0f;
  const float uy = -(((float)y + 0.5f) / (float)H * 2.0f - 1.0f);
  *px = f2u_sat((ux * 0.5f + 0.5f) * (float)W);
  *py = f2u_sat((uy * 0.5f + 0.5f) * (float)H);
}

// Independent PCG hash (training-batch selection of the cache mode).
SPHD uint32_t pcg(uint32_t v) {
  uint32_t state = v * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// ---- wavelengths ---------------------------------------------------------------

// Visible-wavelength importance sampling (spectrum.rs:134-166):
// lambda(u) = 538 - 138.888889 atanh(0.85691062 - 1.82750197 u),
// pdf(lambda) = 0.0039398042 / cosh^2(0.0072 (lambda - 538)) on [360, 830].
SPHD float sample_visible_wavelength(float u) {
  float x = 0.85691062f - 1.82750197f * u;
  return 538.0f - 138.888889f * (0.5f * logf((1.0f + x) / (1.0f - x)));
}
SPHD float visible_wavelength_pdf(float l) {
  if (!(l >= kLambdaMin && l <= kLambdaMax)) return 0.0f;
  float a = 0.0072f * (l - 538.0f);
  float c = 0.5f * (expf(a) + expf(-a));
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
  return expf(-0.5f * t * t);
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
  return 0.5f + t / (2.0f * sqrtf(1.0f + t * t));
}
// Blackbody radiance at 6504 K (Planck), normalised to 1 at 560 nm: the
// illuminant of the RGB upsampling (the reference uses D65).
// B(l) / B(560) = (560 / l)^5 (exp(x560) - 1) / (exp(x) - 1), x = c2 / (l T),
// c2 = hc/k = 1.4387769e7 nm K.
SPHD float illuminant(float l) {
  const float kC2T = 1.4387769e7f / 6504.0f;
  float r = 560.0f / l, r2 = r * r;
  return r2 * r2 * r * (expf(kC2T / 560.0f) - 1.0f) / (expf(kC2T / l) - 1.0f);
}
// An illuminant spectrum (RgbIlluminantSpectrum: scale x sigmoid x
// illuminant) at one wavelength; c = coefficients, c[3] = scale.
SPHD float illum_at(const float* c, float l) { return c[3] * sigmoid_poly(c, l) * illuminant(l); }

// Unbounded RGB (an emitter's radiance, an environment colour, a predicted
// radiance) as an illuminant spectrum: the sigmoid coefficients of
// rgb / (2 max) interpolated trilinearly in a 33^3 table over rgb / max
// (`tab`, 3 floats per entry, built by spectral_fit.cpp), and the scale
// 2 max(rgb) x norm (RgbIlluminantSpectrum).  out: 3 coefficients, scale.
SPHD void illum_lookup(const float* tab, float norm, const float rgb[3], float out[4]) {
  const float m = fmax_nan(rgb[0], fmax_nan(rgb[1], rgb[2]));
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
    const float x = clampf(rgb[k] / m, 0.0f, 1.0f) * 32.0f;
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

// XYZ of one path's spectral radiance (to_xyz, spectrum.rs:62-74) and linear sRGB.
SPHD V3 to_xyz(S4 L, const Wavelengths& w) {
  float xyz[3];
  for (int ch = 0; ch < 3; ++ch) {
    float sum = 0.0f;
    for (int i = 0; i < 4; ++i) {
      const float l = w.lambda.v[i];
      const float cmf = ch == 0 ? cie_x(l) : (ch == 1 ? cie_y(l) : cie_z(l));
      const float p = w.pdf.v[i];
      sum = sum + (p != 0.0f ? (cmf * L.v[i]) / p : 0.0f);
    }
    xyz[ch] = (sum / 4.0f) / kCieYIntegral;
  }
  return v3(xyz[0], xyz[1], xyz[2]);
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

struct Frame {  // CoordSystem::from_z (math/coord_system.rs:56-82)
  V3 x, y, z;
};
SPHD Frame frame_of(V3 f) {
  const float sign = signbit(f.z) ? -1.0f : 1.0f;  // f32::signum
  const float a = -1.0f / (sign + f.z);
  const float b = f.x * f.y * a;
  Frame c;
  c.x = v3(1.0f + sign * sqr(f.x) * a, sign * b, -sign * f.x);
  c.y = v3(b, sign + sqr(f.y) * a, -f.y);
  c.z = f;
  return c;
}
SPHD V3 to_local(const Frame& f, V3 v) { return v3(dot(v, f.x), dot(v, f.y), dot(v, f.z)); }
SPHD V3 to_world(const Frame& f, V3 v) { return v.x * f.x + v.y * f.y + v.z * f.z; }

SPHD bool same_hemisphere(V3 w, V3 wp) { return w.z * wp.z > 0.0f; }
SPHD float cos2(V3 w) { return sqr(w.z); }
SPHD float sin2(V3 w) { return fmax_nan(1.0f - cos2(w), 0.0f); }
SPHD float tan2(V3 w) { return sin2(w) / cos2(w); }
SPHD float cos_phi(V3 w) {
  const float s = sqrtf(sin2(w));
  return s == 0.0f ? 1.0f : clampf(w.x / s, -1.0f, 1.0f);
}
SPHD float sin_phi(V3 w) {
  const float s = sqrtf(sin2(w));
  return s == 0.0f ? 0.0f : clampf(w.y / s, -1.0f, 1.0f);
}

// Trowbridge-Reitz with alpha 0.04 on both axes (ThrowbridgeReitzDistribution
// of the conductor, microfacet.rs, path_integrator.rs:219).
constexpr float kTrAlpha = 0.04f;
SPHD float tr_d(V3 wm) {
  const float t2 = tan2(wm);
  if (isinf(t2)) return 0.0f;
  const float c4 = sqr(cos2(wm));
  const float e = t2 * (sqr(cos_phi(wm) / kTrAlpha) + sqr(sin_phi(wm) / kTrAlpha));
  return 1.0f / (kPi * kTrAlpha * kTrAlpha * c4 * sqr(1.0f + e));
}
SPHD float tr_lambda(V3 w) {
  const float t2 = tan2(w);
  if (isinf(t2)) return 0.0f;
  const float a2 = sqr(cos_phi(w) * kTrAlpha) + sqr(sin_phi(w) * kTrAlpha);
  return (sqrtf(1.0f + a2 * t2) - 1.0f) / 2.0f;
}
SPHD float tr_g1(V3 w) { return 1.0f / (1.0f + tr_lambda(w)); }
SPHD float tr_g(V3 wo, V3 wi) { return 1.0f / (1.0f + tr_lambda(wo) + tr_lambda(wi)); }
SPHD float tr_pdf(V3 w, V3 wm) { return tr_g1(w) / fabsf(w.z) * tr_d(wm) * fabsf(dot(w, wm)); }
SPHD V3 tr_sample_wm(V3 w, float u0, float u1) {
  V3 wh = normalize(v3(kTrAlpha * w.x, kTrAlpha * w.y, w.z));
  if (wh.z < 0.0f) wh = -wh;
  const V3 t1 = wh.z < 0.99999f ? normalize(cross(v3(0.0f, 0.0f, 1.0f), wh)) : v3(1.0f, 0.0f, 0.0f);
  const V3 t2 = cross(wh, t1);
  const float r = sqrtf(u0), th = 2.0f * kPi * u1;  // sample_uniform_disk_polar
  float sp, cp;
  sincosf(th, &sp, &cp);
  float px = r * cp, py = r * sp;
  const float h = sqrtf(1.0f - sqr(px));
  const float s = (1.0f + wh.z) / 2.0f;
  py = (1.0f - s) * h + s * py;  // lerp(s, h, p.y)
  const float pz = sqrtf(fmax_nan(1.0f - (px * px + py * py), 0.0f));
  const V3 nh = px * t1 + py * t2 + pz * wh;
  return normalize(v3(kTrAlpha * nh.x, kTrAlpha * nh.y, fmax_nan(nh.z, 1e-6f)));
}

// fresnel_complex (reflectance/mod.rs:281-294) with num-complex arithmetic;
// the two terms are combined as magnitudes, as the reference does.
struct Cx {
  float re, im;
};
SPHD Cx cmul(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
SPHD Cx cdiv(Cx a, Cx b) {
  const float n = b.re * b.re + b.im * b.im;
  return Cx{(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
SPHD Cx csqrt(Cx z) {
  if (z.im == 0.0f) return z.re >= 0.0f ? Cx{sqrtf(z.re), z.im} : Cx{0.0f, copysignf(sqrtf(-z.re), z.im)};
  const float r = hypotf(z.re, z.im);
  const float a = sqrtf(0.5f * (r + fabsf(z.re)));
  return z.re >= 0.0f ? Cx{a, z.im / (2.0f * a)} : Cx{fabsf(z.im) / (2.0f * a), copysignf(a, z.im)};
}
SPHD float fresnel_complex(float ci, float eta_re, float eta_im) {
  ci = clampf(ci, 0.0f, 1.0f);
  const Cx eta{eta_re, eta_im};
  const float s2i = 1.0f - sqr(ci);
  const Cx s2t = cdiv(Cx{s2i, 0.0f}, cmul(eta, eta));
  const Cx ct = csqrt(Cx{1.0f - s2t.re, 0.0f - s2t.im});
  const Cx ec{eta.re * ci, eta.im * ci};
  const Cx rpa = cdiv(Cx{ec.re - ct.re, ec.im - ct.im}, Cx{ec.re + ct.re, ec.im + ct.im});
  const Cx et = cmul(eta, ct);
  const Cx rpe = cdiv(Cx{ci - et.re, 0.0f - et.im}, Cx{ci + et.re, 0.0f + et.im});
  return (hypotf(rpa.re, rpa.im) + hypotf(rpe.re, rpe.im)) / 2.0f;
}
SPHD float fresnel_dielectric(float ci, float eta) {  // reflectance/mod.rs:260-279
  ci = clampf(ci, -1.0f, 1.0f);
  if (ci < 0.0f) {
    eta = 1.0f / eta;
    ci = -ci;
  }
  const float s2i = 1.0f - sqr(ci), s2t = s2i / sqr(eta);
  if (s2t >= 1.0f) return 1.0f;
  const float ct = safe_sqrt(1.0f - s2t);
  const float rpa = (eta * ci - ct) / (eta * ci + ct), rpe = (ci - eta * ct) / (ci + eta * ct);
  return (sqr(rpa) + sqr(rpe)) / 2.0f;
}

enum : uint32_t { BX_DIFFUSE = 0, BX_CONDUCTOR = 1, BX_DIELECTRIC = 2 };
constexpr float kDielectricEta = 1.5f;

struct Bsdf {
  uint32_t kind;
  S4 a;     // diffuse reflectance, or the conductor's eta
  S4 k;     // the conductor's k
  Frame fr; // shading frame around the (unflipped) shading normal
};

// Bsdf::f (reflectance/mod.rs:173-189) for the non-delta lobes.
SPHD S4 bsdf_f(const Bsdf& b, V3 wow, V3 wiw) {
  const V3 wi = to_local(b.fr, wiw), wo = to_local(b.fr, wow);
  if (wo.z == 0.0f) return s4(0.0f);
  if (b.kind == BX_DIFFUSE) return same_hemisphere(wo, wi) ? b.a * (1.0f / kPi) : s4(0.0f);
  if (b.kind == BX_CONDUCTOR) {  // conductor.rs:37-62
    if (!same_hemisphere(wo, wi)) return s4(0.0f);
    const float co = fabsf(wo.z), ci = fabsf(wi.z);
    if (ci == 0.0f || co == 0.0f) return s4(0.0f);
    V3 wm = wi + wo;
    if (dot(wm, wm) == 0.0f) return s4(0.0f);
    wm = normalize(wm);
    S4 F;
    for (int i = 0; i < 4; ++i) F.v[i] = fresnel_complex(fabsf(dot(wo, wm)), b.a.v[i], b.k.v[i]);
    return ((F * tr_d(wm)) * tr_g(wo, wi)) / (4.0f * ci * co);
  }
  return s4(0.0f);
}

struct BsdfSample {
  S4 f;
  V3 wi;
  float pdf, eta;
  bool specular, transmission;
};
// The reference's cosine hemisphere: its concentric disk mapping, whose
// radius and angle are exchanged (sampling/mod.rs:38-56,64-68).
SPHD V3 cosine_hemisphere(float u0, float u1) {
  const float ox = 2.0f * u0 - 1.0f, oy = 2.0f * u1 - 1.0f;
  float dx = ox, dy = oy;
  if (!(ox == 0.0f && oy == 0.0f)) {
    float th, r;
    if (fabsf(ox) > fabsf(oy)) {
      th = ox;
      r = kPiOver4 * (oy / ox);
    } else {
      th = oy;
      r = kPiOver2 - kPiOver4 * (ox / oy);
    }
    float s, c;
    sincosf(th, &s, &c);
    dx = c * r;
    dy = s * r;
  }
  return v3(dx, dy, safe_sqrt(1.0f - sqr(dx) - sqr(dy)));
}
// Bsdf::sample_f (reflectance/mod.rs:191-214) over the three BxDFs.
SPHD bool bsdf_sample(const Bsdf& b, V3 wow, float uc, float u0, float u1, BsdfSample* out) {
  const V3 wo = to_local(b.fr, wow);
  if (wo.z == 0.0f) return false;
  BsdfSample s;
  s.eta = 1.0f;
  s.specular = false;
  s.transmission = false;
  if (b.kind == BX_DIFFUSE) {  // diffuse.rs:34-60
    V3 wi = cosine_hemisphere(u0, u1);
    if (wo.z < 0.0f) wi.z *= -1.0f;
    s.pdf = fabsf(wi.z) * kInvPi;
    s.f = b.a * kInvPi;
    s.wi = wi;
  } else if (b.kind == BX_CONDUCTOR) {  // conductor.rs:64-119
    const V3 wm = tr_sample_wm(wo, u0, u1);
    const V3 wi = -wo + 2.0f * dot(wo, wm) * wm;
    if (!same_hemisphere(wo, wi)) return false;
    const float wo_wm = fabsf(dot(wo, wm));
    s.pdf = tr_pdf(wo, wm) / (4.0f * wo_wm);
    S4 F;
    for (int i = 0; i < 4; ++i) F.v[i] = fresnel_complex(wo_wm, b.a.v[i], b.k.v[i]);
    s.f = ((F * tr_d(wm)) * tr_g(wo, wi)) / (4.0f * fabsf(wi.z) * fabsf(wo.z));
    s.wi = wi;
  } else {  // dielectric.rs:83-139, smooth
    const float R = fresnel_dielectric(wo.z, kDielectricEta), T = 1.0f - R;
    if (R == 0.0f && T == 0.0f) return false;
    if (uc < R / (R + T)) {
      s.wi = v3(-wo.x, -wo.y, wo.z);
      s.f = s4(R / fabsf(s.wi.z));
      s.pdf = R / (R + T);
      s.specular = true;
    } else {  // refract(wo, +z, eta), reflectance/mod.rs:238-258
      V3 n = v3(0.0f, 0.0f, 1.0f);
      float eta = kDielectricEta;
      float ci = dot(n, wo);
      if (ci < 0.0f) {
        eta = 1.0f / eta;
        ci = -ci;
        n = -n;
      }
      const float s2i = fmax_nan(1.0f - sqr(ci), 0.0f), s2t = s2i / sqr(eta);
      if (s2t >= 1.0f) return false;
      const float ct = safe_sqrt(1.0f - s2t);
      const V3 wt = (-wo) * (1.0f / eta) + (ci / eta - ct) * n;
      s.f = s4(T / fabsf(wt.z)) / sqr(eta);
      s.wi = wt;
      s.pdf = T / (R + T);
      s.eta = eta;
      s.specular = true;
      s.transmission = true;
    }
  }
  if (!contributes(s.f) || s.pdf == 0.0f || s.wi.z == 0.0f) return false;
  s.wi = to_world(b.fr, s.wi);
  *out = s;
  return true;
}

SPHD float power_heuristic(float f, float g) { return sqr(f) / (sqr(f) + sqr(g)); }

// ---- scene access and the integrator ----------------------------------------

// Sun (DistantLight, geometry_resources.rs:52-64): direction of travel, the
// light's scale, the illuminant spectrum of its colour (sigmoid coefficients
// and their scale, as illum_at reads them), the scene radius for the shadow
// ray.
struct Sun {
  float dir[3], scale;
  float coef[4];
  float radius, pad0, pad1, pad2;
};

struct Hit {
  float t, u, v;
  uint32_t tri;
};

// A hit triangle's data as a Geo fetches it: world-space vertices, its vertex
// normals and, for an instance of a two-level scene, the 3x3 matrix that takes
// the (object-space) normals to world space (the transform's inverse
// transpose, geometry_resources.rs:258-261), row-major.
struct TriGeo {
  V3 p[3], n[3];
  float nm[9];
  bool xform;
};

// InfiniteLight::le (infinite_light.rs:69-82,145-148): the equirect uv of the
// direction (unit_vector_to_panorama_coords, sampling/mod.rs:70-75), the
// texture's clamped bilinear sample of its RGB (appearance-texture
// lib.rs:133-173), as an illuminant spectrum, times the light's scale.
SPHD void panorama_uv(V3 d, float* u, float* v) {
  *u = (atan2f(d.z, d.x) + kPi) / (2.0f * kPi);
  *v = acosf(d.y) * kInvPi;
}
template <class Geo>
SPHD S4 env_le(const Geo& g, V3 d, const S4& lambda) {
  if (g.env_w == 0) return s4(0.0f);
  float u, v;
  panorama_uv(d, &u, &v);
  const float x = fabsf(u * (float)g.env_w), y = fabsf(v * (float)g.env_h);
  const float tx = x - truncf(x), ty = y - truncf(y);
  const uint32_t xi = f2u_sat(x), yi = f2u_sat(y);
  const uint32_t x0 = xi < g.env_w - 1 ? xi : g.env_w - 1, x1 = xi + 1 < g.env_w - 1 ? xi + 1 : g.env_w - 1;
  const uint32_t y0 = yi < g.env_h - 1 ? yi : g.env_h - 1, y1 = yi + 1 < g.env_h - 1 ? yi + 1 : g.env_h - 1;
  float c00[3], c10[3], c01[3], c11[3], c[3];
  g.env_rgb(x0, y0, c00);
  g.env_rgb(x1, y0, c10);
  g.env_rgb(x0, y1, c01);
  g.env_rgb(x1, y1, c11);
  for (int k = 0; k < 3; ++k) {
    const float a = c00[k] * (1.0f - tx) + c10[k] * tx;
    const float b = c01[k] * (1.0f - tx) + c11[k] * tx;
    c[k] = a * (1.0f - ty) + b * ty;
  }
  float e[4];
  g.illum_coef(c, e);
  S4 r;
  for (int i = 0; i < 4; ++i) r.v[i] = illum_at(e, lambda.v[i]);
  return r * g.env_scale;
}
// InfiniteLight::pdf_li with the compensated distribution: its function value
// at the texel the uv falls in (rows of env_w in x-major order), over the
// distribution's integral, over 4 pi.
template <class Geo>
SPHD float env_pdf_li(const Geo& g, V3 d) {
  if (g.env_w == 0) return 0.0f;
  float u, v;
  panorama_uv(d, &u, &v);
  uint32_t iu = f2u_sat(u * (float)g.env_w), iv = f2u_sat(v * (float)g.env_h);
  iu = iu < g.env_w - 1 ? iu : g.env_w - 1;
  iv = iv < g.env_h - 1 ? iv : g.env_h - 1;
  return g.env_pdf_func((size_t)iv * g.env_w + iu) / g.env_pdf_integral / (4.0f * kPi);
}

// State of one path of PathIntegrator::li between vertices.
struct PathState {
  S4 L, beta;
  float eta_scale;
  float p_b;       // pdf of the last BSDF sample
  bool specular;   // the last BSDF sample was specular
  int depth;
  ZSobol smp;
};

// Shadow ray of the distant light: its contribution c is added to L unless
// the segment (o, d, [0, tmax]) is occluded.
struct ShadowRay {
  V3 o, d;
  float tmax;
  S4 c;
};

// One vertex of PathIntegrator::li (path_integrator.rs:103-307): `h` is the
// closest hit of the ray (o, d), or null when it escaped.  Adds the
// environment on escape (MIS-weighted after a non-specular bounce) or the
// emission of a front-facing emissive triangle, sets *shadow and fills sh for
// the light sample (sample_ld), samples the BSDF and applies Russian
// roulette.  Returns true when the path goes on along the updated (o, d).
template <class Geo>
SPHD bool path_vertex(const Geo& g, V3& o, V3& d, const Hit* h, const S4& lambda, PathState& ps, int max_depth,
                      bool* shadow, ShadowRay* sh) {
  *shadow = false;
  if (!h) {
    const S4 le = env_le(g, d, lambda);
    if (ps.depth == 0 || ps.specular) {
      ps.L = ps.L + ps.beta * le;
    } else {
      const float p_l = 1.0f * env_pdf_li(g, d);  // the uniform light sampler's pmf of its one light
      ps.L = ps.L + (ps.beta * power_heuristic(ps.p_b, p_l)) * le;
    }
    return false;
  }
  TriGeo tg;
  const Material& m = g.fetch(h->tri, &tg);
  const V3 p0 = tg.p[0], p1 = tg.p[1], p2 = tg.p[2];
  const float bx = 1.0f - h->u - h->v;
  V3 ni = tg.n[0] * bx + tg.n[1] * h->u + tg.n[2] * h->v;
  if (tg.xform)
    ni = v3(tg.nm[0] * ni.x + tg.nm[1] * ni.y + tg.nm[2] * ni.z, tg.nm[3] * ni.x + tg.nm[4] * ni.y + tg.nm[5] * ni.z,
            tg.nm[6] * ni.x + tg.nm[7] * ni.y + tg.nm[8] * ni.z);
  const V3 n = normalize(ni);
  const V3 hit = o + d * h->t;
  const V3 wo = -d;
  if (m.emit_scale > 0.0f && dot(cross(p1 - p0, p2 - p0), wo) > 0.0f) {
    S4 le;
    for (int i = 0; i < 4; ++i) le.v[i] = m.emit_scale * sigmoid_poly(m.emit, lambda.v[i]) * illuminant(lambda.v[i]);
    ps.L = ps.L + ps.beta * le;
  }
  ps.depth += 1;
  if (ps.depth > max_depth) return false;
  Bsdf b;
  b.fr = frame_of(n);
  if (m.metallic > 0.9f) {
    b.kind = BX_CONDUCTOR;  // gold (path_integrator.rs:216-221)
    for (int i = 0; i < 4; ++i) {
      b.a.v[i] = g.au_eta(lambda.v[i]);
      b.k.v[i] = g.au_k(lambda.v[i]);
    }
  } else if (m.transmission > 0.0f) {
    b.kind = BX_DIELECTRIC;
    b.a = s4(0.0f);
    b.k = s4(0.0f);
  } else {
    b.kind = BX_DIFFUSE;
    for (int i = 0; i < 4; ++i) b.a.v[i] = sigmoid_poly(m.albedo, lambda.v[i]);
    b.k = s4(0.0f);
  }
  if (b.kind != BX_DIELECTRIC) {  // sample_ld: the distant light (delta: no MIS)
    const V3 ctx = hit + (wo - hit) * 0.00001f;  // offset_ray_origin (reflection-only BSDF)
    float ul0, ul1;
    ps.smp.get2d(&ul0, &ul1);  // u_light
    (void)ps.smp.get1d();      // the light sampler's pick
    const V3 wi = v3(-g.sun.dir[0], -g.sun.dir[1], -g.sun.dir[2]);
    const V3 lp = ctx + wi * (2.0f * g.sun.radius);
    S4 ll;  // scale x the intensity sampled at 1 nm (DenselySampledSpectrum)
    for (int i = 0; i < 4; ++i) {
      const float lr = roundf(lambda.v[i]);
      const int idx = (int)lr - 360;
      ll.v[i] = (idx < 0 || idx >= 470) ? 0.0f : g.sun.scale * illum_at(g.sun.coef, lr);
    }
    if (contributes(ll)) {
      const S4 f = bsdf_f(b, wo, wi) * fabsf(dot(wi, n));
      if (contributes(f)) {
        sh->o = hit + wi * 0.0001f;
        sh->d = normalize(wi);
        sh->tmax = length(hit - lp);
        sh->c = ps.beta * ((ll * f) / 1.0f);
        *shadow = true;
      }
    }
  }
  const float uc = ps.smp.get1d();
  float u0, u1;
  ps.smp.get2d(&u0, &u1);
  BsdfSample s;
  if (!bsdf_sample(b, wo, uc, u0, u1, &s)) return false;
  ps.beta = ps.beta * ((s.f * fabsf(dot(s.wi, n))) / s.pdf);
  ps.p_b = s.pdf;
  ps.specular = s.specular;
  if (s.transmission) ps.eta_scale *= sqr(s.eta);
  o = hit + s.wi * 0.0001f;
  d = normalize(s.wi);
  const S4 rr = ps.beta * ps.eta_scale;
  if (max4(rr) < 1.0f && ps.depth > 1) {
    const float q = fmax_nan(1.0f - max4(rr), 0.0f);
    if (ps.smp.get1d() < q) return false;
    ps.beta = ps.beta / (1.0f - q);
  }
  return true;
}

// Column-major 4x4 matrix times (x, y, z, w), summed in a fixed order.
SPHD void mul4(const float* m, float x, float y, float z, float w, float* o) {
  for (int r = 0; r < 4; ++r) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

// Camera ray through the centre of pixel (x, y): the uv of lib.rs:138-142 and
// the camera of path_tracer.rs:42-45 (Ray::new normalises the direction).
SPHD void camera_ray(const float* inv_view, const float* inv_proj, uint32_t x, uint32_t y, uint32_t W, uint32_t H,
                     V3* o, V3* d) {
  float ux = ((float)x + 0.5f) / (float)W * 2.0f - 1.0f;
  float uy = ((float)y + 0.5f) / (float)H * 2.0f - 1.0f;
  uy = -uy;
  float oo[4], t[4], dd[4];
  mul4(inv_view, 0.0f, 0.0f, 0.0f, 1.0f, oo);
  mul4(inv_proj, ux, uy, 1.0f, 1.0f, t);
  V3 tn = normalize(v3(t[0], t[1], t[2]));
  mul4(inv_view, tn.x, tn.y, tn.z, 0.0f, dd);
  *o = v3(oo[0], oo[1], oo[2]);
  *d = normalize(v3(dd[0], dd[1], dd[2]));
}

}  // namespace spec
