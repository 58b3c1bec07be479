// Host interface of the spectral kernel (spectral.cu).
#pragma once

#include <cuda_runtime.h>

#include "scene_layout.h"
#include "spectral.h"
#include "traverse2.cuh"

namespace ap {

// Device tables of the spectral mode: the upsampled material table (one per
// scene material), the environment's scale and compensated sampling
// distribution (InfiniteLight, infinite_light.rs:30-67: the function values
// in the reference's x-major flattening, rows of env_w, and its integral; the
// environment's RGB texels are the scene's), the distant light, and the
// illuminant upsampling table.
// The models of a two-level world, for shading (World::build_two_level):
// model-space vertices (x, y, z, 0) and normals (3 floats), per model
// triangle its vertex indices and its material, each model's first triangle,
// and per global triangle id its instance.
struct ModelGeo {
  const float4* positions;
  const float* normals;
  const uint32_t* indices;
  const uint32_t* tri_mat;
  const uint32_t* model_tri0;
  const uint32_t* tri_inst;
};

struct SpectralView {
  const spec::Material* mats;
  // a two-level world (instances): traversal over tl, shading from mg; the
  // DevScene passed with the view then holds the BLAS pool
  int two_level;
  TwoLevel tl;
  ModelGeo mg;
  const float* env_pdf;  // env_w x env_h, or null with env_w = 0
  float env_pdf_integral;
  uint32_t env_w, env_h;
  float env_scale;
  spec::Sun sun;
  const float* illum_tab;  // 33^3 x 3 illuminant upsampling coefficients (spec::illum_lookup)
  float illum_norm;
};

// The compensated environment distribution of the reference's InfiniteLight
// (texture.get_sampling_distribution, then minus its average, clamped at
// zero), flattened x-major and cut into rows of env_w as PiecewiseConstant2D
// reads it, with the integral of that distribution (float sums in the
// reference's order).  rgb: env_w x env_h texels, row-major.
void spectral_env_distribution(const float* rgb, uint32_t env_w, uint32_t env_h, float* func, float* integral);

// Radiance-cache mode of the spectral render (the cache of ap_rc_attach):
// paths are retired at their prefix-th hit into the cache's RGB prediction,
// upsampled to the path's wavelengths; a rotating 1/stride of the pixels trace
// full paths and, per sample pass, a batch of their suffix vertices trains
// the cache (RGB targets from the spectral estimates).
struct SpectralCache {
  void* cache;
  uint32_t prefix, stride, batch;
  float lr;
  int train;
};

struct SpectralCamera {
  float inv_view[16], inv_proj[16];
};

constexpr int kSpectralMaxDepth = 1000;

// Device bytes of the work area for P = W x rows paths (and the cache mode's
// buffers when rc is non-null).
size_t spectral_work_bytes(uint32_t P, const SpectralCache* rc);
// Counters of the last launch_spectral on `work` (device): closest-hit rays,
// nodes, triangles; any-hit rays, nodes, triangles (nodes and triangles only
// when it ran with count_visits).
const unsigned long long* spectral_stats(void* work, uint32_t P, const SpectralCache* rc);

// Renders rows [row0, row1) of a W x H image at `spp` samples per pixel into
// out (3 floats per pixel, row row0 first), with `work` of
// spectral_work_bytes(W * (row1 - row0)) bytes; asynchronous on `st`.
// With count_visits the traversal kernels run in their instrumented form
// (slower).  With `fs` (more streams, not used with count_visits): without
// the cache and with spp > 1, four sample passes are in flight, sample k on
// the k % 4-th of `st`, fs->side, fs->side2, fs->side3, each with its own path state in
// `work`, adding to the shared accumulator in sample order; otherwise each round's
// shadow rays are traced on fs->side beside the next round's extension, which
// reads none of their results.  The streams have joined into `st` when the
// last launch on `st` has run.  Returns the number of kernels launched.
int launch_spectral(const DevScene& s, const SpectralView& v, const SpectralCamera& cam, uint32_t W, uint32_t H,
                    uint32_t row0, uint32_t row1, uint32_t spp, int max_depth, uint32_t seed, float* out, void* work,
                    int num_sms, bool count_visits, const SpectralCache* rc, cudaStream_t st,
                    const FrameStreams* fs = nullptr);

}  // namespace ap
