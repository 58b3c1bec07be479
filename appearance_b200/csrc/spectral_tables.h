// RGB-to-spectrum data of the spectral mode, fitted by spectral_fit.cpp.
//
// The reference's 64^3 sigmoid-coefficient tables come from a crate that is
// not in its repository (appearance-color-spaces), so this library fits its
// own (Jakob and Hanika 2019 sigmoid polynomials in x = (lambda - 360) / 470,
// damped Gauss-Newton against the CIE matching functions under a 6504 K
// blackbody).  This header exposes only the fitted numbers, so that a user of
// the data needs none of the integrator's code.
#pragma once

#include <vector>

namespace spec {

// Sigmoid coefficients (c0, c1, c2: sigmoid(c0 x^2 + c1 x + c2)) of the
// reflectance reproducing linear sRGB `rgb` (components clamped to [0, 1]).
void fit_albedo(const float rgb[3], float coef[3]);
// Factor that makes the 6504 K illuminant integrate, against cie_y, to the
// CIE-Y normaliser of to_xyz.
double illuminant_norm();

// Emission / environment upsampling: coefficients of rgb / (2 max) on a 33^3
// grid over rgb / max (entry (r, g, b) at 3 * ((b * 33 + g) * 33 + r)),
// interpolated trilinearly; out[3] = 2 max(rgb) x illuminant_norm().
struct IlluminantTable {
  std::vector<float> coef;
  IlluminantTable();
  void lookup(const float rgb[3], float out[4]) const;
};
// The table, built once per process (about half a second) on first use.
const IlluminantTable& illuminant_table();

}  // namespace spec
