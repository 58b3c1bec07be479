// Spectral (hero-wavelength) rendering on sm_100a: one thread per pixel runs
// spec::pixel_sample (spectral.h) for each of its samples, tracing through the
// compressed 8-wide BVH with the shared closest-hit and any-hit traversals
// (traverse.cuh).  Output is linear sRGB, the mean over the pixel's samples.
// Rays traced are summed per warp and added to a 64-bit counter.
#include "spectral.cuh"
#include "traverse.cuh"

namespace ap {

namespace {

struct GpuGeo {
  const DevScene& s;
  const spec::Material* mats;
  const float4* env;
  uint32_t env_w, env_h;
  float env_scale;
  spec::Sun sun;
  uint32_t* rays;  // rays traced by this thread

  APD bool closest(spec::V3 o, spec::V3 d, float tmax, spec::Hit& h) const {
    *rays += 1;
    Hit r;
    bool hit = trace_closest(s, f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), tmax, r);
    h.t = r.t;
    h.tri = r.tri;
    return hit;
  }
  APD bool occluded(spec::V3 o, spec::V3 d, float tmax) const {
    *rays += 1;
    return trace_any(s, f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), tmax);
  }
  APD void tri(uint32_t g, spec::V3* p0, spec::V3* p1, spec::V3* p2) const {
    const InstanceDev& in = s.instances[s.tri_instance[g]];
    uint32_t fi = in.first_index + (g - in.first_global_tri) * 3;
    float4 a = s.positions[in.first_vertex + s.indices[fi + 0]];
    float4 b = s.positions[in.first_vertex + s.indices[fi + 1]];
    float4 c = s.positions[in.first_vertex + s.indices[fi + 2]];
    *p0 = spec::v3(a.x, a.y, a.z);
    *p1 = spec::v3(b.x, b.y, b.z);
    *p2 = spec::v3(c.x, c.y, c.z);
  }
  APD const spec::Material& material(uint32_t g) const {
    const InstanceDev& in = s.instances[s.tri_instance[g]];
    return mats[in.material_idx + s.tri_material[in.first_index / 3 + (g - in.first_global_tri)]];
  }
  APD void env_texel(uint32_t idx, float c[4]) const {
    float4 v = __ldg(env + idx);
    c[0] = v.x;
    c[1] = v.y;
    c[2] = v.z;
    c[3] = v.w;
  }
};

__global__ void __launch_bounds__(128) k_spectral(DevScene s, SpectralView v, SpectralCamera cam, uint32_t W,
                                                  uint32_t H, uint32_t row0, uint32_t row1, uint32_t spp,
                                                  int max_depth, uint32_t seed, float* out,
                                                  unsigned long long* ray_count) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= row1) return;
  uint32_t rays = 0;
  GpuGeo g{s, v.mats, v.env, v.env_w, v.env_h, v.env_scale, v.sun, &rays};
  spec::V3 acc = spec::v3(0.0f, 0.0f, 0.0f);
  for (uint32_t k = 0; k < spp; ++k)
    acc = acc + spec::pixel_sample(g, cam.inv_view, cam.inv_proj, x, y, W, H, k, seed, max_depth);
  const float inv = 1.0f / (float)spp;
  float* o = out + 3 * ((size_t)(y - row0) * W + x);
  o[0] = acc.x * inv;
  o[1] = acc.y * inv;
  o[2] = acc.z * inv;
  const uint32_t mask = __activemask();
  const uint32_t warp_rays = __reduce_add_sync(mask, rays);
  uint32_t lane;
  asm("mov.u32 %0, %%laneid;" : "=r"(lane));
  if (ray_count && __ffs(mask) - 1 == (int)lane) atomicAdd(ray_count, (unsigned long long)warp_rays);
}

}  // namespace

void launch_spectral(const DevScene& s, const SpectralView& v, const SpectralCamera& cam, uint32_t W, uint32_t H,
                     uint32_t row0, uint32_t row1, uint32_t spp, int max_depth, uint32_t seed, float* out,
                     unsigned long long* ray_count, cudaStream_t st) {
  dim3 block(16, 8);
  dim3 grid((W + block.x - 1) / block.x, (row1 - row0 + block.y - 1) / block.y);
  k_spectral<<<grid, block, 0, st>>>(s, v, cam, W, H, row0, row1, spp, max_depth, seed, out, ray_count);
}

}  // namespace ap
