// Host interface of the spectral kernel (spectral.cu).
#pragma once

#include <cuda_runtime.h>

#include "scene_layout.h"
#include "spectral.h"

namespace ap {

// Device tables of the spectral mode: the upsampled material table (one per
// scene material) and environment texels {sigmoid coefficients, scale}.
struct SpectralView {
  const spec::Material* mats;
  const float4* env;  // env_w x env_h, or null with env_w = 0
  uint32_t env_w, env_h;
  float env_scale;
  spec::Sun sun;
};

struct SpectralCamera {
  float inv_view[16], inv_proj[16];
};

// Renders rows [row0, row1) of a W x H image at `spp` samples per pixel into
// out (3 floats per pixel, row row0 first); asynchronous on `st`.  With
// ray_count non-null the rays traced are added to it (a slower kernel form).
void launch_spectral(const DevScene& s, const SpectralView& v, const SpectralCamera& cam, uint32_t W, uint32_t H,
                     uint32_t row0, uint32_t row1, uint32_t spp, int max_depth, uint32_t seed, float* out,
                     unsigned long long* ray_count, cudaStream_t st);

}  // namespace ap
