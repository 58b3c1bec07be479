// Oracle (test infrastructure only): the reference's CPU spectral path tracer
// (crates/appearance-path-tracer), restated here on its own from the Rust
// source, for the GPU spectral mode's parity tests.  Nothing of the library's
// spectral integrator is used: this file follows the reference's functions
// one by one (file:line beside each), in the reference's evaluation order,
// over this oracle's own scene, watertight triangle test and binary BVH.
//
//   render loop      lib.rs:79-195, path_tracer.rs:28-68 (one 1-spp ZSobol
//                    frame per sample, seed = frame index)
//   sampler          sampling/zsobol_sampler.rs:43-152, math/sobol.rs:3-22
//                    (dimensions 0 and 1 only), math/random.rs:69-76,140-152
//                    (mix_bits, FastOwenScrambler), math/mod.rs:42-75
//   integrator       path_integrator.rs:34-307 (li, sample_ld)
//   lights           light_sources/distant_light.rs:47-67,
//                    light_sources/infinite_light.rs:30-149 (le, pdf_li with
//                    the compensated distribution), uniform_light_sampler.rs
//   distributions    sampling/piecewise_constant.rs:21-171
//   BxDFs            reflectance/{mod,diffuse,conductor,dielectric,microfacet}.rs
//   hit data         geometry_resources.rs:229-282 (interpolated normal)
//
// Substitutions, each because the reference's code or data cannot be used
// here (all shared with the library and stated in its documentation):
//   * RGB -> spectrum: the sigmoid coefficients come from the library's fit
//     (spectral_tables.h; the reference's tables are generated by a crate
//     missing from its repository), evaluated in x = (lambda - 360) / 470,
//     with a 6504 K blackbody standing in for the D65 illuminant;
//   * colour output: the XYZ of the four wavelengths (analytic CIE 1931 fit of
//     Wyman, Sloan and Shirley 2013) to linear sRGB, in place of the film's
//     Canon EOS 100D sensor model;
//   * wavelength sampling evaluates its analytic functions instead of the
//     reference's lookup tables of the same functions, without the 470x
//     factor those tables put on the pdf;
//   * MurmurHash3 x64_128 (the murmurhash3 0.0.5 crate, not vendored): the
//     published algorithm, pinned by its SMHasher verification value;
//   * BVH: closest hit by (t, triangle id) over a watertight test (tinybvh is
//     not vendored);
//   * the environment is the scene's RGB f32 equirect (the reference loads a
//     PNG); emissive triangles, which the reference tracer lacks, add their
//     emission when a path hits their front face.
// Data tables used as data: the reference's gold index of refraction
// (spectral_data.h, generated from its radiometry/data_tables/materials.rs).
// Reference defects reproduced as written, since parity is with the
// reference: the concentric disk mapping with radius and angle exchanged
// (sampling/mod.rs:38-56), conductor Fresnel terms combined as magnitudes
// rather than squared magnitudes (reflectance/mod.rs:286-294), the x-major
// flattening of the environment's sampling distribution
// (appearance-texture lib.rs:193-205 into piecewise_constant.rs:120-129), and
// the escaped-path MIS weight against a light the light sampler never picks.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <thread>
#include <vector>

#include "../appearance_b200/csrc/spectral_data.h"
#include "../appearance_b200/csrc/spectral_tables.h"
#include "oracle_scene.h"
#include "oracle_twolevel.h"

namespace {

constexpr float PI = 3.14159265358979323846f;
constexpr float FRAC_1_PI = 0.318309886183790671538f;
constexpr float FRAC_PI_2 = 1.57079632679489661923f;
constexpr float FRAC_PI_4 = 0.785398163397448309616f;
constexpr float LAMBDA_MIN = 360.0f, LAMBDA_MAX = 830.0f;

// ---- glam-style vectors (component-wise, left to right) -------------------

struct Vec2 {
  float x, y;
};
struct Vec3 {
  float x, y, z;
};
struct Vec4 {
  float v[4];
};
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
inline Vec3 operator*(Vec3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3 operator*(float s, Vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(Vec3 a, Vec3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline float length(Vec3 a) { return sqrtf(dot(a, a)); }
inline Vec3 normalize(Vec3 a) { return a * (1.0f / length(a)); }
inline float length_squared(Vec3 a) { return dot(a, a); }

inline Vec4 v4(float a) { return {{a, a, a, a}}; }
inline Vec4 operator*(Vec4 a, Vec4 b) { return {{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}}; }
inline Vec4 operator*(Vec4 a, float s) { return {{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
inline Vec4 operator*(float s, Vec4 a) { return {{s * a.v[0], s * a.v[1], s * a.v[2], s * a.v[3]}}; }
inline Vec4 operator/(Vec4 a, float s) { return {{a.v[0] / s, a.v[1] / s, a.v[2] / s, a.v[3] / s}}; }
inline Vec4 operator+(Vec4 a, Vec4 b) { return {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}}; }
inline float fmax_rs(float a, float b) { return a > b ? a : (b == b ? b : a); }  // f32::max: NaN-ignoring
inline float max_element(Vec4 a) { return fmax_rs(fmax_rs(fmax_rs(a.v[0], a.v[1]), a.v[2]), a.v[3]); }
inline bool has_contribution(Vec4 a) {  // spectrum.rs:58-60
  return a.v[0] * a.v[0] + a.v[1] * a.v[1] + a.v[2] * a.v[2] + a.v[3] * a.v[3] > 0.0f;
}
inline float sqr(float x) { return x * x; }
inline float safe_sqrt(float x) { return sqrtf(fmax_rs(x, 0.0f)); }
inline float signum(float x) { return signbit(x) ? -1.0f : 1.0f; }
inline float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
inline float fract_rs(float x) { return x - truncf(x); }
inline uint32_t f2u_sat(float x) {  // Rust `as u32`: saturating, NaN -> 0
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)x;
}

// ---- MurmurHash3 x64_128 (Austin Appleby's published algorithm) -----------

inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}
void murmur3_x64_128(const uint8_t* data, size_t len, uint64_t seed, uint64_t out[2]) {
  const uint64_t c1 = 0x87c37b91114253d5ull, c2 = 0x4cf5ad432745937full;
  uint64_t h1 = seed, h2 = seed;
  const size_t nblocks = len / 16;
  for (size_t i = 0; i < nblocks; ++i) {
    uint64_t k1 = 0, k2 = 0;
    for (int b = 7; b >= 0; --b) k1 = (k1 << 8) | data[16 * i + b];
    for (int b = 7; b >= 0; --b) k2 = (k2 << 8) | data[16 * i + 8 + b];
    k1 *= c1; k1 = rotl64(k1, 31); k1 *= c2; h1 ^= k1;
    h1 = rotl64(h1, 27); h1 += h2; h1 = h1 * 5 + 0x52dce729;
    k2 *= c2; k2 = rotl64(k2, 33); k2 *= c1; h2 ^= k2;
    h2 = rotl64(h2, 31); h2 += h1; h2 = h2 * 5 + 0x38495ab5;
  }
  const uint8_t* tail = data + nblocks * 16;
  const size_t rem = len & 15;
  uint64_t k1 = 0, k2 = 0;
  for (size_t b = rem; b > 8; --b) k2 = (k2 << 8) | tail[b - 1];
  if (rem > 8) {
    k2 *= c2; k2 = rotl64(k2, 33); k2 *= c1; h2 ^= k2;
  }
  for (size_t b = rem < 8 ? rem : 8; b > 0; --b) k1 = (k1 << 8) | tail[b - 1];
  if (rem > 0) {
    k1 *= c1; k1 = rotl64(k1, 31); k1 *= c2; h1 ^= k1;
  }
  h1 ^= (uint64_t)len;
  h2 ^= (uint64_t)len;
  h1 += h2;
  h2 += h1;
  h1 = fmix64(h1);
  h2 = fmix64(h2);
  h1 += h2;
  h2 += h1;
  out[0] = h1;
  out[1] = h2;
}

// ---- ZSobol sampler ---------------------------------------------------------

uint64_t mix_bits(uint64_t v) {  // math/random.rs:69-76
  v ^= v >> 31;
  v *= 0x7fb5d329728ea185ull;
  v ^= v >> 27;
  v *= 0x81dadef4bc2dd44dull;
  v ^= v >> 33;
  return v;
}
uint32_t reverse_bits_32(uint32_t n) {  // math/mod.rs:67-75
  n = (n >> 16) | (n << 16);
  n = ((n & 0x00ff00ffu) << 8) | ((n & 0xff00ff00u) >> 8);
  n = ((n & 0x0f0f0f0fu) << 4) | ((n & 0xf0f0f0f0u) >> 4);
  n = ((n & 0x33333333u) << 2) | ((n & 0xccccccccu) >> 2);
  n = ((n & 0x55555555u) << 1) | ((n & 0xaaaaaaaau) >> 1);
  return n;
}
uint32_t fast_owen_scramble(uint32_t v, uint32_t seed) {  // math/random.rs:140-152
  v = reverse_bits_32(v);
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return reverse_bits_32(v);
}
// Generator matrices of Sobol dimensions 0 and 1 (math/sobol.rs): dimension 0
// is the identity in reversed bit order, dimension 1 the matrix of the
// primitive polynomial x + 1 (direction numbers m_i = m_{i-1} xor 2 m_{i-1}).
struct SobolMatrices {
  uint32_t m[2][32];
  SobolMatrices() {
    uint32_t d = 1;
    for (int i = 0; i < 32; ++i) {
      m[0][i] = 0x80000000u >> i;
      m[1][i] = d << (31 - i);
      d ^= d << 1;
    }
  }
};
const SobolMatrices kSobol;
float sobol_sample(uint64_t a, int dim, uint32_t scramble_seed) {  // math/sobol.rs:3-22
  uint32_t v = 0;
  for (int i = 0; a != 0; ++i, a >>= 1)
    if (a & 1) v ^= i < 32 ? kSobol.m[dim][i] : 0u;
  v = fast_owen_scramble(v, scramble_seed);
  return (float)v * 2.3283064e-10f;
}
uint64_t left_shift_2(uint64_t x) {  // math/mod.rs:53-61
  x &= 0xffffffffull;
  x = (x ^ (x << 16)) & 0x0000ffff0000ffffull;
  x = (x ^ (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x ^ (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x ^ (x << 2)) & 0x3333333333333333ull;
  x = (x ^ (x << 1)) & 0x5555555555555555ull;
  return x;
}
uint64_t encode_morton_2(uint32_t x, uint32_t y) { return (left_shift_2(y) << 1) | left_shift_2(x); }
int32_t round_up_pow2(int32_t v) {
  v -= 1;
  v |= v >> 1;
  v |= v >> 2;
  v |= v >> 4;
  v |= v >> 8;
  v |= v >> 16;
  return v + 1;
}
const uint8_t PERMUTATIONS[24][4] = {
    {0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 1, 3}, {0, 2, 3, 1}, {0, 3, 2, 1}, {0, 3, 1, 2}, {1, 0, 2, 3}, {1, 0, 3, 2},
    {1, 2, 0, 3}, {1, 2, 3, 0}, {1, 3, 2, 0}, {1, 3, 0, 2}, {2, 1, 0, 3}, {2, 1, 3, 0}, {2, 0, 1, 3}, {2, 0, 3, 1},
    {2, 3, 0, 1}, {2, 3, 1, 0}, {3, 1, 2, 0}, {3, 1, 0, 2}, {3, 2, 1, 0}, {3, 2, 0, 1}, {3, 0, 2, 1}, {3, 0, 1, 2}};

struct ZSobolSampler {
  uint64_t seed;
  uint32_t log2_samples_per_pixel;
  uint32_t n_base_4_digits;
  uint64_t morton_idx = 0;
  uint32_t dimension = 0;

  ZSobolSampler(uint32_t samples_per_pixel, uint32_t res_x, uint32_t res_y, uint64_t seed_) : seed(seed_) {
    log2_samples_per_pixel = (uint32_t)log2f((float)samples_per_pixel);
    const int32_t res = round_up_pow2((int32_t)(res_x > res_y ? res_x : res_y));
    const uint32_t log4 = (log2_samples_per_pixel + 1) / 2;
    n_base_4_digits = (uint32_t)log2f((float)res) + log4;
  }
  uint64_t get_sample_idx() const {
    uint64_t sample_idx = 0;
    const bool pow_2_samples = (log2_samples_per_pixel & 1) != 0;
    const int last_digit = pow_2_samples ? 1 : 0;
    for (int i = (int)n_base_4_digits - 1; i >= last_digit; --i) {
      const int digit_shift = 2 * i - (pow_2_samples ? 1 : 0);
      const uint64_t digit = (morton_idx >> digit_shift) & 3;
      const uint64_t higher = morton_idx >> (digit_shift + 2);
      const uint64_t p = (mix_bits(higher ^ (0x55555555ull * (uint64_t)dimension)) >> 24) % 24;
      sample_idx |= (uint64_t)PERMUTATIONS[p][digit] << digit_shift;
    }
    if (pow_2_samples) {
      const uint64_t digit = morton_idx & 1;
      sample_idx |= digit ^ (mix_bits((morton_idx >> 1) ^ (0x55555555ull * (uint64_t)dimension)) & 1);
    }
    return sample_idx;
  }
  void start_pixel_sample(uint32_t px, uint32_t py, uint32_t sample_idx, uint32_t dim) {
    dimension = dim;
    morton_idx = (encode_morton_2(px, py) << log2_samples_per_pixel) | sample_idx;
  }
  uint64_t hash_dim() const {
    uint8_t key[12];
    memcpy(key, &dimension, 4);  // little-endian, as bytemuck::bytes_of
    memcpy(key + 4, &seed, 8);
    uint64_t h[2];
    murmur3_x64_128(key, 12, 0, h);
    return h[0];
  }
  float get_1d() {
    const uint64_t idx = get_sample_idx();
    dimension += 1;
    const uint64_t hash = hash_dim();
    return sobol_sample(idx, 0, (uint32_t)hash);
  }
  Vec2 get_2d() {
    const uint64_t idx = get_sample_idx();
    dimension += 2;
    const uint64_t hash = hash_dim();
    return {sobol_sample(idx, 0, (uint32_t)hash), sobol_sample(idx, 1, (uint32_t)(hash >> 32))};
  }
};

// ---- spectra (substitutions stated at the top) ---------------------------------

inline float lobe(float l, float mu, float s1, float s2) {
  const float t = (l - mu) / (l < mu ? s1 : s2);
  return expf(-0.5f * t * t);
}
inline float cie_x(float l) {
  return 1.056f * lobe(l, 599.8f, 37.9f, 31.0f) + 0.362f * lobe(l, 442.0f, 16.0f, 26.7f) -
         0.065f * lobe(l, 501.1f, 20.4f, 26.2f);
}
inline float cie_y(float l) { return 0.821f * lobe(l, 568.8f, 46.9f, 40.5f) + 0.286f * lobe(l, 530.9f, 16.3f, 31.1f); }
inline float cie_z(float l) { return 1.217f * lobe(l, 437.0f, 11.8f, 36.0f) + 0.681f * lobe(l, 459.0f, 26.0f, 13.8f); }
constexpr float CIE_Y_INTEGRAL = 106.922074f;  // of cie_y over 360-830 nm

inline float sigmoid_poly(const float c[3], float l) {
  const float x = (l - LAMBDA_MIN) * (1.0f / (LAMBDA_MAX - LAMBDA_MIN));
  const float t = (c[0] * x + c[1]) * x + c[2];
  return 0.5f + t / (2.0f * sqrtf(1.0f + t * t));
}
inline float planck_6504(float l) {  // normalised to 1 at 560 nm
  const float k = 1.4387769e7f / 6504.0f;
  const float r = 560.0f / l, r2 = r * r;
  return r2 * r2 * r * (expf(k / 560.0f) - 1.0f) / (expf(k / l) - 1.0f);
}

struct IllumCoef {
  float c[3], scale;
};
// RgbIlluminantSpectrum::new: the fitted table's trilinear lookup of
// rgb / max over a 33^3 grid, scale 2 max x the illuminant normaliser.
IllumCoef illum_coef(const std::vector<float>& tab, float norm, const float rgb[3]) {
  IllumCoef o;
  const float m = fmax_rs(rgb[0], fmax_rs(rgb[1], rgb[2]));
  if (!(m > 0.0f)) {
    o.c[0] = 0.0f;
    o.c[1] = 0.0f;
    o.c[2] = -1e4f;
    o.scale = 0.0f;
    return o;
  }
  int i0[3];
  float f[3];
  for (int k = 0; k < 3; ++k) {
    const float x = clampf(rgb[k] / m, 0.0f, 1.0f) * 32.0f;
    i0[k] = (int)x < 31 ? (int)x : 31;
    f[k] = x - (float)i0[k];
  }
  for (int ch = 0; ch < 3; ++ch) {
    float v = 0.0f;
    for (int corner = 0; corner < 8; ++corner) {
      const int dr = corner & 1, dg = (corner >> 1) & 1, db = corner >> 2;
      const float w = (dr ? f[0] : 1.0f - f[0]) * (dg ? f[1] : 1.0f - f[1]) * (db ? f[2] : 1.0f - f[2]);
      v = v + w * tab[3 * (((i0[2] + db) * 33 + (i0[1] + dg)) * 33 + (i0[0] + dr)) + ch];
    }
    o.c[ch] = v;
  }
  o.scale = 2.0f * m * norm;
  return o;
}
inline float illum_sample(const IllumCoef& e, float l) { return e.scale * sigmoid_poly(e.c, l) * planck_6504(l); }

struct Wavelengths {  // spectrum.rs:88-160
  Vec4 lambda, pdf;
};
inline float sample_visible_wavelengths(float u) {
  const float x = 0.85691062f - 1.82750197f * u;
  return 538.0f - 138.888889f * (0.5f * logf((1.0f + x) / (1.0f - x)));
}
inline float visible_wavelengths_pdf(float l) {
  if (!(l >= LAMBDA_MIN && l <= LAMBDA_MAX)) return 0.0f;
  const float a = 0.0072f * (l - 538.0f);
  const float c = 0.5f * (expf(a) + expf(-a));
  return 0.0039398042f / (c * c);
}
Wavelengths sample_visible(float u) {
  Wavelengths w;
  for (int i = 0; i < 4; ++i) {
    float up = u + (float)i / 4.0f;
    if (up > 1.0f) up -= 1.0f;
    w.lambda.v[i] = sample_visible_wavelengths(up);
    w.pdf.v[i] = visible_wavelengths_pdf(w.lambda.v[i]);
  }
  return w;
}

// Linear sRGB of a sample's spectral radiance: XYZ (to_xyz, spectrum.rs:62-74)
// through the sRGB matrix.
Vec3 to_srgb(Vec4 L, const Wavelengths& w) {
  float xyz[3] = {0.0f, 0.0f, 0.0f};
  for (int ch = 0; ch < 3; ++ch) {
    float sum = 0.0f;
    for (int i = 0; i < 4; ++i) {
      const float cmf = ch == 0 ? cie_x(w.lambda.v[i]) : (ch == 1 ? cie_y(w.lambda.v[i]) : cie_z(w.lambda.v[i]));
      const float p = w.pdf.v[i];
      sum = sum + (p != 0.0f ? (cmf * L.v[i]) / p : 0.0f);
    }
    xyz[ch] = (sum / 4.0f) / CIE_Y_INTEGRAL;
  }
  return {3.2404542f * xyz[0] - 1.5371385f * xyz[1] - 0.4985314f * xyz[2],
          -0.9692660f * xyz[0] + 1.8760108f * xyz[1] + 0.0415560f * xyz[2],
          0.0556434f * xyz[0] - 0.2040259f * xyz[1] + 1.0572252f * xyz[2]};
}

// ---- gold (radiometry/data_tables/materials.rs:89-129, spectral_data.h) -------

// PiecewiseLinearSpectrum::reflectance (spectrum.rs:552-566) over the gold
// tables, with find_interval_fast (math/mod.rs:97-113).
float au_sample(const float* vals, float lambda) {
  const int n = spec::kAuSamples;
  if (lambda < spec::kAuLambda[0] || lambda > spec::kAuLambda[n - 1]) return 0.0f;
  const int n_values = n - 2;
  int size = n_values, first = 1;
  while (size > 0) {
    const int half = size >> 1, middle = first + half;
    const bool pred = spec::kAuLambda[middle] <= lambda;
    first = pred ? middle + 1 : first;
    size = pred ? size - (half + 1) : half;
  }
  int o = first - 1;
  o = o < 0 ? 0 : (o > n_values ? n_values : o);
  const float t = (lambda - spec::kAuLambda[o]) / (spec::kAuLambda[o + 1] - spec::kAuLambda[o]);
  return vals[o] + (vals[o + 1] - vals[o]) * t;
}

// ---- BxDFs -----------------------------------------------------------------

struct CoordSystem {  // math/coord_system.rs:56-82 (from_z)
  Vec3 x, y, z;
  static CoordSystem from_z(Vec3 f) {
    const float sign = signum(f.z);
    const float a = -1.0f / (sign + f.z);
    const float b = f.x * f.y * a;
    CoordSystem c;
    c.x = {1.0f + sign * sqr(f.x) * a, sign * b, -sign * f.x};
    c.y = {b, sign + sqr(f.y) * a, -f.y};
    c.z = f;
    return c;
  }
  Vec3 ws_to_frame(Vec3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
  Vec3 frame_to_ws(Vec3 v) const { return v.x * x + v.y * y + v.z * z; }
};

inline bool same_hemisphere(Vec3 w, Vec3 wp) { return w.z * wp.z > 0.0f; }
inline float abs_cos_theta(Vec3 w) { return fabsf(w.z); }
inline float cos_2_theta(Vec3 w) { return sqr(w.z); }
inline float sin_2_theta(Vec3 w) { return fmax_rs(1.0f - cos_2_theta(w), 0.0f); }
inline float sin_theta(Vec3 w) { return sqrtf(sin_2_theta(w)); }
inline float tan_2_theta(Vec3 w) { return sin_2_theta(w) / cos_2_theta(w); }
inline float cos_phi(Vec3 w) {
  const float s = sin_theta(w);
  return s == 0.0f ? 1.0f : clampf(w.x / s, -1.0f, 1.0f);
}
inline float sin_phi(Vec3 w) {
  const float s = sin_theta(w);
  return s == 0.0f ? 0.0f : clampf(w.y / s, -1.0f, 1.0f);
}

struct TrowbridgeReitz {  // reflectance/microfacet.rs
  float ax, ay;
  float d(Vec3 wm) const {
    const float t2 = tan_2_theta(wm);
    if (isinf(t2)) return 0.0f;
    const float c4 = sqr(cos_2_theta(wm));
    const float e = t2 * (sqr(cos_phi(wm) / ax) + sqr(sin_phi(wm) / ay));
    return 1.0f / (PI * ax * ay * c4 * sqr(1.0f + e));
  }
  float lambda(Vec3 w) const {
    const float t2 = tan_2_theta(w);
    if (isinf(t2)) return 0.0f;
    const float a2 = sqr(cos_phi(w) * ax) + sqr(sin_phi(w) * ay);
    return (sqrtf(1.0f + a2 * t2) - 1.0f) / 2.0f;
  }
  float g1(Vec3 w) const { return 1.0f / (1.0f + lambda(w)); }
  float g(Vec3 wo, Vec3 wi) const { return 1.0f / (1.0f + lambda(wo) + lambda(wi)); }
  float pdf(Vec3 w, Vec3 wm) const { return g1(w) / abs_cos_theta(w) * d(wm) * fabsf(dot(w, wm)); }
  Vec3 sample_wm(Vec3 w, Vec2 u) const {
    Vec3 wh = normalize(Vec3{ax * w.x, ay * w.y, w.z});
    if (wh.z < 0.0f) wh = -wh;
    const Vec3 t1 = wh.z < 0.99999f ? normalize(cross(Vec3{0.0f, 0.0f, 1.0f}, wh)) : Vec3{1.0f, 0.0f, 0.0f};
    const Vec3 t2 = cross(wh, t1);
    // sample_uniform_disk_polar (sampling/mod.rs:58-62)
    const float r = sqrtf(u.x), theta = 2.0f * PI * u.y;
    Vec2 p{r * cosf(theta), r * sinf(theta)};
    const float h = sqrtf(1.0f - sqr(p.x));
    const float s = (1.0f + wh.z) / 2.0f;
    p.y = (1.0f - s) * h + s * p.y;  // lerp(s, h, p.y), math/mod.rs:38-40
    const float pz = sqrtf(fmax_rs(1.0f - (p.x * p.x + p.y * p.y), 0.0f));
    const Vec3 nh = p.x * t1 + p.y * t2 + pz * wh;
    return normalize(Vec3{ax * nh.x, ay * nh.y, fmax_rs(nh.z, 1e-6f)});
  }
};

// Complex arithmetic of num-complex's Complex32, as fresnel_complex uses it.
struct C32 {
  float re, im;
};
inline C32 cmul(C32 a, C32 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C32 cadd(C32 a, C32 b) { return {a.re + b.re, a.im + b.im}; }
inline C32 csub(C32 a, C32 b) { return {a.re - b.re, a.im - b.im}; }
inline C32 cscale(C32 a, float s) { return {a.re * s, a.im * s}; }
inline C32 cdiv(C32 a, C32 b) {
  const float n = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline C32 csqrt(C32 z) {  // principal square root
  if (z.im == 0.0f) {
    if (z.re >= 0.0f) return {sqrtf(z.re), z.im};
    return {0.0f, copysignf(sqrtf(-z.re), z.im)};
  }
  const float r = hypotf(z.re, z.im);
  const float a = sqrtf(0.5f * (r + fabsf(z.re)));
  if (z.re >= 0.0f) return {a, z.im / (2.0f * a)};
  return {fabsf(z.im) / (2.0f * a), copysignf(a, z.im)};
}
inline float cnorm(C32 z) { return hypotf(z.re, z.im); }  // num-complex norm(): |z|

float fresnel_complex(float cos_theta_i, C32 eta) {  // reflectance/mod.rs:281-294
  cos_theta_i = clampf(cos_theta_i, 0.0f, 1.0f);
  const float sin_2_theta_i = 1.0f - sqr(cos_theta_i);
  const C32 sin_2_theta_t = cdiv(C32{sin_2_theta_i, 0.0f}, cmul(eta, eta));
  const C32 cos_theta_t = csqrt(csub(C32{1.0f, 0.0f}, sin_2_theta_t));
  const C32 ec = cscale(eta, cos_theta_i);
  const C32 r_parl = cdiv(csub(ec, cos_theta_t), cadd(ec, cos_theta_t));
  const C32 etc = cmul(eta, cos_theta_t);
  const C32 r_perp = cdiv(csub(C32{cos_theta_i, 0.0f}, etc), cadd(C32{cos_theta_i, 0.0f}, etc));
  return (cnorm(r_parl) + cnorm(r_perp)) / 2.0f;
}

float fresnel_dielectric(float cos_theta_i, float eta) {  // reflectance/mod.rs:260-279
  cos_theta_i = clampf(cos_theta_i, -1.0f, 1.0f);
  if (cos_theta_i < 0.0f) {
    eta = 1.0f / eta;
    cos_theta_i = -cos_theta_i;
  }
  const float sin_2_theta_i = 1.0f - sqr(cos_theta_i);
  const float sin_2_theta_t = sin_2_theta_i / sqr(eta);
  if (sin_2_theta_t >= 1.0f) return 1.0f;
  const float cos_theta_t = safe_sqrt(1.0f - sin_2_theta_t);
  const float r_parl = (eta * cos_theta_i - cos_theta_t) / (eta * cos_theta_i + cos_theta_t);
  const float r_perp = (cos_theta_i - eta * cos_theta_t) / (cos_theta_i + eta * cos_theta_t);
  return (sqr(r_parl) + sqr(r_perp)) / 2.0f;
}

enum Kind { DIFFUSE, CONDUCTOR, DIELECTRIC };
struct BsdfSample {
  Vec4 f;
  Vec3 wi;
  float pdf, eta;
  bool specular, transmission;
};

// The reference's concentric mapping, with its radius and angle exchanged
// (sampling/mod.rs:38-56), then cosine_hemisphere (sampling/mod.rs:64-68).
Vec3 sample_cosine_hemisphere(Vec2 u) {
  const Vec2 o{2.0f * u.x - 1.0f, 2.0f * u.y - 1.0f};
  Vec2 d;
  if (o.x == 0.0f && o.y == 0.0f) {
    d = o;
  } else {
    float theta, r;
    if (fabsf(o.x) > fabsf(o.y)) {
      theta = o.x;
      r = FRAC_PI_4 * (o.y / o.x);
    } else {
      theta = o.y;
      r = FRAC_PI_2 - FRAC_PI_4 * (o.x / o.y);
    }
    d = {cosf(theta) * r, sinf(theta) * r};
  }
  const float z = safe_sqrt(1.0f - sqr(d.x) - sqr(d.y));
  return {d.x, d.y, z};
}

struct Bsdf {  // reflectance/mod.rs:160-232 over one of the three BxDFs
  Kind kind;
  Vec4 r;          // diffuse reflectance
  Vec4 eta, k;     // conductor index
  CoordSystem cs;
  TrowbridgeReitz mf{0.04f, 0.04f};

  bool reflection_only() const { return kind != DIELECTRIC; }
  Vec4 f(Vec3 wo_render, Vec3 wi_render) const {
    const Vec3 wi = cs.ws_to_frame(wi_render), wo = cs.ws_to_frame(wo_render);
    if (wo.z == 0.0f) return v4(0.0f);
    if (kind == DIFFUSE) return same_hemisphere(wo, wi) ? r * (1.0f / PI) : v4(0.0f);
    if (kind == CONDUCTOR) {  // conductor.rs:37-62 (alpha 0.04: not smooth)
      if (!same_hemisphere(wo, wi)) return v4(0.0f);
      const float cos_o = abs_cos_theta(wo), cos_i = abs_cos_theta(wi);
      if (cos_i == 0.0f || cos_o == 0.0f) return v4(0.0f);
      Vec3 wm = wi + wo;
      if (length_squared(wm) == 0.0f) return v4(0.0f);
      wm = normalize(wm);
      Vec4 F;
      for (int i = 0; i < 4; ++i) F.v[i] = fresnel_complex(fabsf(dot(wo, wm)), C32{eta.v[i], k.v[i]});
      return (mf.d(wm) * F * mf.g(wo, wi)) / (4.0f * cos_i * cos_o);
    }
    return v4(0.0f);  // smooth dielectric: no non-delta lobe
  }
  bool sample_f(Vec3 wo_render, float uc, Vec2 u, BsdfSample* out) const {
    const Vec3 wo = cs.ws_to_frame(wo_render);
    if (wo.z == 0.0f) return false;
    BsdfSample bs;
    bs.eta = 1.0f;
    bs.specular = false;
    bs.transmission = false;
    if (kind == DIFFUSE) {  // diffuse.rs:34-60
      Vec3 wi = sample_cosine_hemisphere(u);
      if (wo.z < 0.0f) wi.z *= -1.0f;
      bs.pdf = abs_cos_theta(wi) * FRAC_1_PI;
      bs.f = r * FRAC_1_PI;
      bs.wi = wi;
    } else if (kind == CONDUCTOR) {  // conductor.rs:64-119
      const Vec3 wm = mf.sample_wm(wo, u);
      const Vec3 wi = -wo + 2.0f * dot(wo, wm) * wm;  // reflect, reflectance/mod.rs:234-236
      if (!same_hemisphere(wo, wi)) return false;
      const float wo_dot_wm = fabsf(dot(wo, wm));
      bs.pdf = mf.pdf(wo, wm) / (4.0f * wo_dot_wm);
      const float cos_o = abs_cos_theta(wo), cos_i = abs_cos_theta(wi);
      Vec4 F;
      for (int i = 0; i < 4; ++i) F.v[i] = fresnel_complex(wo_dot_wm, C32{eta.v[i], k.v[i]});
      bs.f = (mf.d(wm) * F * mf.g(wo, wi)) / (4.0f * cos_i * cos_o);
      bs.wi = wi;
    } else {  // dielectric.rs:83-139, smooth, eta 1.5
      const float eta_d = 1.5f;
      const float R = fresnel_dielectric(wo.z, eta_d), T = 1.0f - R;
      const float pr = R, pt = T;
      if (pr == 0.0f && pt == 0.0f) return false;
      if (uc < pr / (pr + pt)) {
        bs.wi = {-wo.x, -wo.y, wo.z};
        bs.f = v4(R / abs_cos_theta(bs.wi));
        bs.pdf = pr / (pr + pt);
        bs.specular = true;
      } else {
        // refract(wo, (0, 0, 1), eta), reflectance/mod.rs:238-258
        Vec3 n{0.0f, 0.0f, 1.0f};
        float eta = eta_d;
        float cos_i = dot(n, wo);
        if (cos_i < 0.0f) {
          eta = 1.0f / eta;
          cos_i = -cos_i;
          n = -n;
        }
        const float sin_2_i = fmax_rs(1.0f - sqr(cos_i), 0.0f);
        const float sin_2_t = sin_2_i / sqr(eta);
        if (sin_2_t >= 1.0f) return false;
        const float cos_t = safe_sqrt(1.0f - sin_2_t);
        const Vec3 wt = (-wo) * (1.0f / eta) + (cos_i / eta - cos_t) * n;
        Vec4 ft = v4(T / abs_cos_theta(wt));
        ft = ft / sqr(eta);
        bs.f = ft;
        bs.wi = wt;
        bs.pdf = pt / (pr + pt);
        bs.eta = eta;
        bs.specular = true;
        bs.transmission = true;
      }
    }
    if (!has_contribution(bs.f) || bs.pdf == 0.0f || bs.wi.z == 0.0f) return false;
    bs.wi = cs.frame_to_ws(bs.wi);
    *out = bs;
    return true;
  }
};

// ---- the scene -------------------------------------------------------------

struct PiecewiseConstant1D {  // sampling/piecewise_constant.rs:21-49
  std::vector<float> func, cdf;
  float integral;
  void build(const float* f, size_t n) {
    func.assign(f, f + n);
    cdf.assign(n + 1, 0.0f);
    for (float& v : func) v = fabsf(v);
    for (size_t i = 1; i <= n; ++i) cdf[i] = cdf[i - 1] + func[i - 1] * (1.0f - 0.0f) / (float)n;
    integral = cdf[n];
  }
};

struct SpectralScene {
  const orc::Scene* scene;
  orc::OracleBvh bvh;
  // a world of instances: hits come from its two-level form (object-space
  // intersection, global triangle ids in the order of `scene`, the flattened
  // world, whose data shades them)
  const void* two_level = nullptr;
  std::vector<Vec3> normals;  // float vertex normals
  // per material: albedo coefficients, conductor and emission
  struct Mat {
    float albedo[3];
    float metallic, transmission;
    IllumCoef emit;
    float emit_max;
  };
  std::vector<Mat> mats;
  std::vector<float> illum_tab;
  float illum_norm = 1.0f;
  // environment (InfiniteLight, scale = env_scale) and its compensated
  // sampling distribution (x-major flattening, see the header)
  uint32_t env_w = 0, env_h = 0;
  float env_scale = 1.0f;
  std::vector<PiecewiseConstant1D> cond;
  PiecewiseConstant1D marginal;
  // distant light
  Vec3 sun_dir{0.0f, -1.0f, 0.0f};
  IllumCoef sun{};
  float sun_scale = 0.0f, scene_radius = 1000.0f;
};

// Conductor index: every metallic material is gold (path_integrator.rs:216-221).
inline void conductor_index(const Wavelengths& w, Vec4* eta, Vec4* k) {
  for (int i = 0; i < 4; ++i) {
    eta->v[i] = au_sample(spec::kAuEta, w.lambda.v[i]);
    k->v[i] = au_sample(spec::kAuK, w.lambda.v[i]);
  }
}

Vec3 texel(const SpectralScene& s, uint32_t x, uint32_t y) {
  const float* p = s.scene->env.data() + 3 * ((size_t)y * s.env_w + x);
  return {p[0], p[1], p[2]};
}

// InfiniteLight::le (infinite_light.rs:69-82,145-148): unit_vector_to_panorama_coords
// (sampling/mod.rs:70-75), the texture's bilinear sample with clamping
// (appearance-texture lib.rs:133-173,343-347), the RGB as an illuminant
// spectrum, times the light's scale.
Vec4 env_le(const SpectralScene& s, Vec3 d, const Wavelengths& w) {
  if (s.env_w == 0) return v4(0.0f);
  const float phi = atan2f(d.z, d.x) + PI;
  const float theta = acosf(d.y);
  const Vec2 uv{phi / (2.0f * PI), theta * FRAC_1_PI};
  const float x = fabsf(uv.x * (float)s.env_w), y = fabsf(uv.y * (float)s.env_h);
  const float tx = fract_rs(x), ty = fract_rs(y);
  const uint32_t xi = f2u_sat(x), yi = f2u_sat(y);
  auto cl = [](uint32_t v, uint32_t hi) { return v > hi ? hi : v; };
  const uint32_t x0 = cl(xi, s.env_w - 1), x1 = cl(xi + 1, s.env_w - 1);
  const uint32_t y0 = cl(yi, s.env_h - 1), y1 = cl(yi + 1, s.env_h - 1);
  const Vec3 c00 = texel(s, x0, y0), c10 = texel(s, x1, y0), c01 = texel(s, x0, y1), c11 = texel(s, x1, y1);
  const Vec3 a = c00 * (1.0f - tx) + c10 * tx;
  const Vec3 b = c01 * (1.0f - tx) + c11 * tx;
  const Vec3 c = a * (1.0f - ty) + b * ty;
  const float rgb[3] = {c.x, c.y, c.z};
  const IllumCoef e = illum_coef(s.illum_tab, s.illum_norm, rgb);
  Vec4 out;
  for (int i = 0; i < 4; ++i) out.v[i] = illum_sample(e, w.lambda.v[i]);
  return out * s.env_scale;
}

// InfiniteLight::pdf_li with the compensated distribution
// (infinite_light.rs:134-143, piecewise_constant.rs:142-170).
float env_pdf_li(const SpectralScene& s, Vec3 d) {
  if (s.env_w == 0) return 0.0f;
  const float phi = atan2f(d.z, d.x) + PI;
  const float theta = acosf(d.y);
  const Vec2 uv{phi / (2.0f * PI), theta * FRAC_1_PI};
  const uint32_t nu = (uint32_t)s.cond[0].func.size(), nv = (uint32_t)s.cond.size();
  uint32_t iu = f2u_sat(uv.x * (float)nu), iv = f2u_sat(uv.y * (float)nv);
  iu = iu > nu - 1 ? nu - 1 : iu;
  iv = iv > nv - 1 ? nv - 1 : iv;
  const float pdf = s.cond[iv].func[iu] / s.marginal.integral;
  return pdf / (4.0f * PI);
}

inline float power_heuristic(float f, float g) { return sqr(f) / (sqr(f) + sqr(g)); }

// PathIntegrator::li (path_integrator.rs:103-307) with sample_ld (:34-101).
Vec4 li(const SpectralScene& s, Vec3 ray_o, Vec3 ray_d, const Wavelengths& w, ZSobolSampler& sampler,
        uint32_t max_bounces) {
  const orc::Scene& sc = *s.scene;
  Vec4 l = v4(0.0f), throughput = v4(1.0f);
  float p_b = 1.0f, eta_scale = 1.0f;
  bool specular_bounce = false;
  uint32_t depth = 0;
  while (true) {
    const orc::V3 ro = orc::v3(ray_o.x, ray_o.y, ray_o.z), rd = orc::v3(ray_d.x, ray_d.y, ray_d.z);
    const orc::Hit hit = s.two_level ? orc::two_level_closest(s.two_level, ro, rd, 1e30f)
                                     : s.bvh.closest(sc, ro, rd, 0.0f, 1e30f, nullptr, nullptr);
    if (hit.tri == 0xFFFFFFFFu) {
      const Vec4 le = env_le(s, ray_d, w);
      if (depth == 0 || specular_bounce) {
        l = l + throughput * le;
      } else {
        const float p_l = 1.0f * env_pdf_li(s, ray_d);  // pmf of the one-light sampler
        const float w_b = power_heuristic(p_b, p_l);
        l = l + (throughput * w_b) * le;
      }
      break;
    }
    // geometry_resources.rs:229-282
    const orc::Instance& in = sc.instances[sc.tri_instance[hit.tri]];
    const uint32_t loc = hit.tri - in.first_global_tri;
    const uint32_t i0 = in.first_vertex + sc.indices[in.first_index + 3 * loc + 0];
    const uint32_t i1 = in.first_vertex + sc.indices[in.first_index + 3 * loc + 1];
    const uint32_t i2 = in.first_vertex + sc.indices[in.first_index + 3 * loc + 2];
    const float bx = 1.0f - hit.u - hit.v, by = hit.u, bz = hit.v;
    const Vec3 n = normalize(s.normals[i0] * bx + s.normals[i1] * by + s.normals[i2] * bz);
    const SpectralScene::Mat& m = s.mats[in.material_idx + sc.tri_material[in.first_index / 3 + loc]];
    const Vec3 hit_point = ray_o + ray_d * hit.t;
    const Vec3 wo = -ray_d;
    if (m.emit_max > 0.0f) {  // emissive triangles: added on a front-face hit
      const orc::V3 a = sc.positions[i0], b = sc.positions[i1], c = sc.positions[i2];
      const Vec3 e1{b.x - a.x, b.y - a.y, b.z - a.z}, e2{c.x - a.x, c.y - a.y, c.z - a.z};
      if (dot(cross(e1, e2), wo) > 0.0f) {
        Vec4 le;
        for (int i = 0; i < 4; ++i) le.v[i] = illum_sample(m.emit, w.lambda.v[i]);
        l = l + throughput * le;
      }
    }
    depth += 1;
    if (depth > max_bounces) break;
    Bsdf bsdf;
    bsdf.cs = CoordSystem::from_z(n);
    if (m.metallic > 0.9f) {
      bsdf.kind = CONDUCTOR;
      conductor_index(w, &bsdf.eta, &bsdf.k);
    } else if (m.transmission > 0.0f) {
      bsdf.kind = DIELECTRIC;
    } else {
      bsdf.kind = DIFFUSE;
      for (int i = 0; i < 4; ++i) bsdf.r.v[i] = sigmoid_poly(m.albedo, w.lambda.v[i]);
    }
    if (bsdf.kind != DIELECTRIC) {  // flags().is_non_specular(): sample_ld
      Vec3 ctx_point = hit_point;
      if (bsdf.reflection_only()) ctx_point = ctx_point + (wo - ctx_point) * 0.00001f;
      (void)sampler.get_2d();  // u_light (unused by the distant light)
      (void)sampler.get_1d();  // the light sampler's pick of its one light
      const Vec3 wi = -s.sun_dir;
      const Vec3 p = ctx_point + wi * (2.0f * s.scene_radius);
      Vec4 li_l;  // DistantLight: scale x the intensity sampled at 1 nm (DenselySampledSpectrum)
      for (int i = 0; i < 4; ++i) {
        const float lr = roundf(w.lambda.v[i]);
        const int idx = (int)lr - 360;
        li_l.v[i] = (idx < 0 || idx >= 470) ? 0.0f : s.sun_scale * illum_sample(s.sun, lr);
      }
      if (has_contribution(li_l)) {
        const Vec4 f = bsdf.f(wo, wi) * fabsf(dot(wi, n));
        if (has_contribution(f)) {
          const Vec3 so = hit_point + wi * 0.0001f;
          const Vec3 sd = normalize(wi);
          const Vec3 dd = hit_point - p;
          const float tmax = length(dd);
          const orc::V3 qo = orc::v3(so.x, so.y, so.z), qd = orc::v3(sd.x, sd.y, sd.z);
          if (!(s.two_level ? orc::two_level_any(s.two_level, qo, qd, tmax) : s.bvh.any(sc, qo, qd, 0.0f, tmax))) {
            const Vec4 ld = (li_l * f) / 1.0f;
            l = l + throughput * ld;
          }
        }
      }
    }
    const float u = sampler.get_1d();
    const Vec2 u2 = sampler.get_2d();
    BsdfSample bs;
    if (!bsdf.sample_f(wo, u, u2, &bs)) break;
    throughput = throughput * ((bs.f * fabsf(dot(bs.wi, n))) / bs.pdf);
    p_b = bs.pdf;
    specular_bounce = bs.specular;
    if (bs.transmission) eta_scale *= sqr(bs.eta);
    ray_o = hit_point + bs.wi * 0.0001f;
    ray_d = normalize(bs.wi);
    const Vec4 rr = throughput * eta_scale;
    if (max_element(rr) < 1.0f && depth > 1) {
      const float r = fmax_rs(1.0f - max_element(rr), 0.0f);
      if (sampler.get_1d() < r) break;
      throughput = throughput / (1.0f - r);
    }
  }
  return l;
}

inline void mul4(const float* m, float x, float y, float z, float w, float* o) {
  for (int r = 0; r < 4; ++r) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

// One sample of pixel (x, y): path_tracer.rs:28-68 with the uv of lib.rs:138-142.
Vec3 pixel_sample(const SpectralScene& s, const float* inv_view, const float* inv_proj, uint32_t x, uint32_t y,
                  uint32_t W, uint32_t H, uint64_t frame_seed, uint32_t max_bounces) {
  const float uvx = ((float)x + 0.5f) / (float)W * 2.0f - 1.0f;
  const float uvy = ((float)y + 0.5f) / (float)H * 2.0f - 1.0f;
  const float cx = uvx, cy = -uvy;
  float o4[4], t4[4], d4[4];
  mul4(inv_view, 0.0f, 0.0f, 0.0f, 1.0f, o4);
  mul4(inv_proj, cx, cy, 1.0f, 1.0f, t4);
  const Vec3 tn = normalize(Vec3{t4[0], t4[1], t4[2]});
  mul4(inv_view, tn.x, tn.y, tn.z, 0.0f, d4);
  const Vec3 o{o4[0], o4[1], o4[2]};
  const Vec3 d = normalize(Vec3{d4[0], d4[1], d4[2]});  // Ray::new normalises
  ZSobolSampler sampler(1, W, H, frame_seed);
  const uint32_t px = f2u_sat((cx * 0.5f + 0.5f) * (float)W), py = f2u_sat((cy * 0.5f + 0.5f) * (float)H);
  sampler.start_pixel_sample(px, py, 0, 0);
  const Wavelengths w = sample_visible(sampler.get_1d());
  const Vec4 L = li(s, o, d, w, sampler, max_bounces);
  return to_srgb(L, w);
}

}  // namespace

extern "C" {

// Spectral scene of an oracle scene (orc_scene_new) for the parameters of
// ap_spectral_setup.  `normals` are the scene's float vertex normals.  With
// `two_level` (orc_two_level_new, its instances in the order of the flattened
// `scene`) rays are traced through the two-level form.
void* orc_spectral_new(void* scene, const float* normals, const float* sun_dir3, const float* sun_rgb3, float sun_scale,
                       float scene_radius, float env_scale, const void* two_level) {
  const orc::Scene* sc = (const orc::Scene*)scene;
  SpectralScene* s = new SpectralScene();
  s->scene = sc;
  s->two_level = two_level;
  if (!two_level) s->bvh.build(*sc);
  s->normals.resize(sc->positions.size());
  for (size_t i = 0; i < s->normals.size(); ++i)
    s->normals[i] = {normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]};
  const spec::IlluminantTable& tab = spec::illuminant_table();
  s->illum_tab = tab.coef;
  s->illum_norm = (float)spec::illuminant_norm();
  s->mats.resize(sc->materials.size());
  for (size_t i = 0; i < sc->materials.size(); ++i) {
    const orc::Material& om = sc->materials[i];
    SpectralScene::Mat& m = s->mats[i];
    spec::fit_albedo(om.color, m.albedo);
    m.metallic = om.metallic;
    m.transmission = om.transmission;
    m.emit = illum_coef(s->illum_tab, s->illum_norm, om.emission);
    m.emit_max = fmax_rs(om.emission[0], fmax_rs(om.emission[1], om.emission[2]));
  }
  s->env_w = sc->env_w;
  s->env_h = sc->env_h;
  s->env_scale = env_scale;
  if (s->env_w && s->env_h) {
    // Texture::get_sampling_distribution (x-major) with the compensation of
    // InfiniteLight::new, flattened and cut into rows of env_w as
    // PiecewiseConstant2D::new does.
    const uint32_t W = s->env_w, H = s->env_h;
    std::vector<float> dist((size_t)W * H);
    for (uint32_t y = 0; y < H; ++y)
      for (uint32_t x = 0; x < W; ++x) {
        const float* p = sc->env.data() + 3 * ((size_t)y * W + x);
        dist[(size_t)x * H + y] = (p[0] + p[1] + p[2]) / 3.0f;
      }
    float average = 0.0f;
    for (float v : dist) average += v;
    average /= (float)((size_t)W * H);
    for (float& v : dist) v = fmax_rs(v - average, 0.0f);
    s->cond.resize(H);
    std::vector<float> marg(H);
    for (uint32_t v = 0; v < H; ++v) {
      s->cond[v].build(dist.data() + (size_t)v * W, W);
      marg[v] = s->cond[v].integral;
    }
    s->marginal.build(marg.data(), H);
  }
  const float len = sqrtf(sun_dir3[0] * sun_dir3[0] + sun_dir3[1] * sun_dir3[1] + sun_dir3[2] * sun_dir3[2]);
  s->sun_dir = Vec3{sun_dir3[0], sun_dir3[1], sun_dir3[2]} * (1.0f / len);
  s->sun = illum_coef(s->illum_tab, s->illum_norm, sun_rgb3);
  s->sun_scale = sun_scale;
  s->scene_radius = scene_radius;
  return s;
}

void orc_spectral_free(void* p) { delete (SpectralScene*)p; }

// Rows [row0, row1) of a W x H image, spp samples per pixel (sample k is the
// reference's 1-spp frame with seed `seed + k`), out 3 floats per pixel
// (linear sRGB, mean over samples).  inv_view / inv_proj: column-major.
void orc_spectral_render(void* p, const float* inv_view, const float* inv_proj, uint32_t W, uint32_t H, uint32_t row0,
                         uint32_t row1, uint32_t spp, int max_depth, uint32_t seed, uint32_t threads, float* out) {
  const SpectralScene& s = *(const SpectralScene*)p;
  std::atomic<uint32_t> next{row0};
  auto work = [&]() {
    for (uint32_t y = next.fetch_add(1); y < row1; y = next.fetch_add(1))
      for (uint32_t x = 0; x < W; ++x) {
        Vec3 acc{0.0f, 0.0f, 0.0f};
        for (uint32_t k = 0; k < spp; ++k)
          acc = acc + pixel_sample(s, inv_view, inv_proj, x, y, W, H, (uint64_t)seed + k, (uint32_t)max_depth);
        const float inv = 1.0f / (float)spp;
        float* q = out + 3 * ((size_t)(y - row0) * W + x);
        q[0] = acc.x * inv;
        q[1] = acc.y * inv;
        q[2] = acc.z * inv;
      }
  };
  if (threads <= 1) {
    work();
    return;
  }
  std::vector<std::thread> ts;
  for (uint32_t t = 0; t < threads; ++t) ts.emplace_back(work);
  for (auto& t : ts) t.join();
}

// Building blocks for the CPU tests.
// The analytic CIE functions and the 6504 K illuminant at one wavelength.
void orc_spectral_cmf(float lambda, float* out4) {
  out4[0] = cie_x(lambda);
  out4[1] = cie_y(lambda);
  out4[2] = cie_z(lambda);
  out4[3] = planck_6504(lambda);
}
void orc_spectral_fit(const float* rgb, float* coef3) { spec::fit_albedo(rgb, coef3); }
void orc_spectral_sigmoid(const float* coef3, float lambda, float* out) { *out = sigmoid_poly(coef3, lambda); }
void orc_spectral_wavelength(float u, float* out2) {
  out2[0] = sample_visible_wavelengths(u);
  out2[1] = visible_wavelengths_pdf(out2[0]);
}
double orc_spectral_illuminant_norm() { return spec::illuminant_norm(); }

// MurmurHash3 x64_128 of `len` bytes.
void orc_murmur3_x64_128(const uint8_t* data, size_t len, uint64_t seed, uint64_t* out2) {
  murmur3_x64_128(data, len, seed, out2);
}
// The first n samples of a ZSobol stream: pixel (px, py), sample index, frame
// seed, image resolution; per sample the sequence of draws `kinds` (1: get_1d,
// 2: get_2d), written to out in order.
void orc_zsobol(uint32_t res_x, uint32_t res_y, uint32_t spp, uint64_t seed, uint32_t px, uint32_t py,
                uint32_t sample_idx, const uint8_t* kinds, uint32_t n_kinds, float* out) {
  ZSobolSampler z(spp, res_x, res_y, seed);
  z.start_pixel_sample(px, py, sample_idx, 0);
  size_t o = 0;
  for (uint32_t i = 0; i < n_kinds; ++i) {
    if (kinds[i] == 1) {
      out[o++] = z.get_1d();
    } else {
      const Vec2 v = z.get_2d();
      out[o++] = v.x;
      out[o++] = v.y;
    }
  }
}

}  // extern "C"
