// Host-side RGB upsampling for the spectral mode (csrc/spectral.h): sigmoid
// polynomial coefficients (Jakob and Hanika, "A Low-Dimensional Function Space
// for Efficient Spectral Upsampling", 2019) fitted by damped Gauss-Newton so
// that the reflectance, integrated against the analytic CIE matching
// functions under the 6504 K illuminant, reproduces the XYZ of a linear sRGB
// colour.  Albedos are fitted per colour; emission and environment texels use
// a 33^3 table over rgb / max(rgb), interpolated trilinearly.
#include "spectral_fit.h"

#include <cmath>
#include <vector>

#include "spectral.h"

namespace spec {
namespace {

constexpr int kSamples = 94;  // 362.5 ... 827.5 nm, 5 nm

struct Weights {
  float lambda[kSamples];
  double wx[kSamples], wy[kSamples], wz[kSamples];  // E(l) cmf(l) dl / integral(E y dl)
  double k_illum;                                   // CIE_Y_integral / integral(E y dl)
  Weights() {
    double norm = 0.0;
    for (int i = 0; i < kSamples; ++i) {
      lambda[i] = 362.5f + 5.0f * (float)i;
      double e = illuminant(lambda[i]);
      wx[i] = e * cie_x(lambda[i]) * 5.0;
      wy[i] = e * cie_y(lambda[i]) * 5.0;
      wz[i] = e * cie_z(lambda[i]) * 5.0;
      norm += wy[i];
    }
    for (int i = 0; i < kSamples; ++i) {
      wx[i] /= norm;
      wy[i] /= norm;
      wz[i] /= norm;
    }
    k_illum = (double)kCieYIntegral / norm;
  }
};
const Weights& weights() {
  static const Weights w;
  return w;
}

void xyz_of(const double c[3], double out[3]) {
  const Weights& w = weights();
  float cf[3] = {(float)c[0], (float)c[1], (float)c[2]};
  out[0] = out[1] = out[2] = 0.0;
  for (int i = 0; i < kSamples; ++i) {
    double s = sigmoid_poly(cf, w.lambda[i]);
    out[0] += s * w.wx[i];
    out[1] += s * w.wy[i];
    out[2] += s * w.wz[i];
  }
}

void rgb_to_xyz(const float rgb[3], double xyz[3]) {
  const double r = rgb[0], g = rgb[1], b = rgb[2];
  xyz[0] = 0.4124564 * r + 0.3575761 * g + 0.1804375 * b;
  xyz[1] = 0.2126729 * r + 0.7151522 * g + 0.0721750 * b;
  xyz[2] = 0.0193339 * r + 0.1191920 * g + 0.9503041 * b;
}

bool solve3(double A[3][3], double b[3], double x[3]) {
  double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
               A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (std::fabs(det) < 1e-300) return false;
  for (int k = 0; k < 3; ++k) {
    double M[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i][j] = j == k ? b[i] : A[i][j];
    x[k] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
            M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) /
           det;
  }
  return true;
}

}  // namespace

void fit_albedo(const float rgb_in[3], float coef[3]) {
  float rgb[3];
  for (int i = 0; i < 3; ++i) rgb[i] = std::fmin(std::fmax(rgb_in[i], 0.0f), 1.0f);
  double target[3];
  rgb_to_xyz(rgb, target);
  // start from the constant reflectance with the target's luminance
  double v = std::fmin(std::fmax(target[1], 1e-4), 1.0 - 1e-4);
  double c[3] = {0.0, 0.0, (2.0 * v - 1.0) / (2.0 * std::sqrt(v * (1.0 - v)))};
  double mu = 1e-3;
  double cur[3];
  xyz_of(c, cur);
  double err = 0.0;
  for (int i = 0; i < 3; ++i) err += (cur[i] - target[i]) * (cur[i] - target[i]);
  for (int it = 0; it < 100 && err > 1e-12; ++it) {
    double J[3][3];
    for (int j = 0; j < 3; ++j) {
      double cp[3] = {c[0], c[1], c[2]}, xp[3];
      const double h = 1e-3 * std::fmax(1.0, std::fabs(c[j]));
      cp[j] += h;
      xyz_of(cp, xp);
      for (int i = 0; i < 3; ++i) J[i][j] = (xp[i] - cur[i]) / h;
    }
    double JtJ[3][3], g[3];
    for (int a = 0; a < 3; ++a) {
      g[a] = 0.0;
      for (int i = 0; i < 3; ++i) g[a] += J[i][a] * (target[i] - cur[i]);
      for (int b = 0; b < 3; ++b) {
        JtJ[a][b] = 0.0;
        for (int i = 0; i < 3; ++i) JtJ[a][b] += J[i][a] * J[i][b];
      }
    }
    bool improved = false;
    for (int tries = 0; tries < 12 && !improved; ++tries) {
      double A[3][3], dx[3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) A[a][b] = JtJ[a][b] + (a == b ? mu * (JtJ[a][a] + 1e-9) : 0.0);
      if (!solve3(A, g, dx)) {
        mu *= 10.0;
        continue;
      }
      double cn[3] = {c[0] + dx[0], c[1] + dx[1], c[2] + dx[2]}, xn[3];
      xyz_of(cn, xn);
      double en = 0.0;
      for (int i = 0; i < 3; ++i) en += (xn[i] - target[i]) * (xn[i] - target[i]);
      if (en < err) {
        for (int i = 0; i < 3; ++i) {
          c[i] = cn[i];
          cur[i] = xn[i];
        }
        err = en;
        mu = std::fmax(mu * 0.3, 1e-9);
        improved = true;
      } else {
        mu *= 10.0;
      }
    }
    if (!improved) break;
  }
  for (int i = 0; i < 3; ++i) coef[i] = (float)c[i];
}

double illuminant_norm() { return weights().k_illum; }

IlluminantTable::IlluminantTable() : coef(33 * 33 * 33 * 3) {
  for (int b = 0; b < 33; ++b)
    for (int g = 0; g < 33; ++g)
      for (int r = 0; r < 33; ++r) {
        float rgb[3] = {0.5f * (float)r / 32.0f, 0.5f * (float)g / 32.0f, 0.5f * (float)b / 32.0f};
        fit_albedo(rgb, &coef[3 * ((b * 33 + g) * 33 + r)]);
      }
}

void IlluminantTable::lookup(const float rgb[3], float out[4]) const {
  illum_lookup(coef.data(), (float)illuminant_norm(), rgb, out);
}

const IlluminantTable& illuminant_table() {
  static const IlluminantTable t;
  return t;
}

void upsample_materials(const float* mats26, uint32_t n, Material* out) {
  const IlluminantTable& tab = illuminant_table();
  for (uint32_t i = 0; i < n; ++i) {
    const float* m = mats26 + 26 * (size_t)i;
    Material& o = out[i];
    fit_albedo(m, o.albedo);
    o.metallic = m[3];
    float e[4];
    tab.lookup(m + 5, e);
    o.emit[0] = e[0];
    o.emit[1] = e[1];
    o.emit[2] = e[2];
    o.emit_scale = e[3];
    o.transmission = m[8];
    o.pad0 = o.pad1 = o.pad2 = 0.0f;
  }
}

Sun make_sun(const float dir[3], const float rgb[3], float scale, float radius) {
  Sun s;
  V3 d = normalize(v3(dir[0], dir[1], dir[2]));
  s.dir[0] = d.x;
  s.dir[1] = d.y;
  s.dir[2] = d.z;
  s.scale = scale;
  illuminant_table().lookup(rgb, s.coef);
  s.radius = radius;
  s.pad0 = s.pad1 = s.pad2 = 0.0f;
  return s;
}

}  // namespace spec
