// Host-side RGB upsampling for the spectral mode (spectral_fit.cpp).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "spectral.h"
#include "spectral_tables.h"

namespace spec {

// Spectral tables of an RGB scene.  Materials are read in the 26-float
// MaterialDescriptor order (color 0-2, metallic 3, emission 5-7,
// transmission 8); the distant light travels along `dir` (normalised here)
// with radiance scale x the illuminant spectrum of `rgb` (DistantLight::new,
// geometry_resources.rs:52-64).
void upsample_materials(const float* mats26, uint32_t n, Material* out);
Sun make_sun(const float dir[3], const float rgb[3], float scale, float radius);

}  // namespace spec
