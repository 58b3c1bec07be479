// Host-side RGB upsampling for the spectral mode (spectral_fit.cpp).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "spectral.h"

namespace spec {

// Sigmoid coefficients of the reflectance reproducing linear sRGB `rgb`
// (components clamped to [0, 1]).
void fit_albedo(const float rgb[3], float coef[3]);
// Factor that makes the 6504 K illuminant integrate, against cie_y, to the
// CIE-Y normaliser of to_xyz.
double illuminant_norm();

// Emission / environment upsampling: coefficients of rgb / (2 max) on a 33^3
// grid over rgb / max, interpolated; out[3] = 2 max(rgb) x illuminant_norm().
struct IlluminantTable {
  std::vector<float> coef;
  IlluminantTable();
  void lookup(const float rgb[3], float out[4]) const;
};
// The table, built once per process (about half a second) on first use.
const IlluminantTable& illuminant_table();

// Spectral tables of an RGB scene.  Materials are read in the 26-float
// MaterialDescriptor order (color 0-2, metallic 3, emission 5-7,
// transmission 8); environment texels are linear RGB triples; the distant
// light travels along `dir` (normalised here) with radiance scale x the
// illuminant spectrum of `rgb` (DistantLight::new, geometry_resources.rs:52-64).
void upsample_materials(const float* mats26, uint32_t n, Material* out);
void upsample_env(const float* rgb, size_t texels, float* out4);
Sun make_sun(const float dir[3], const float rgb[3], float scale, float radius);

}  // namespace spec
