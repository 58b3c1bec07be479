// Oracle (test infrastructure only): the spectral mode on the CPU.
//
// The integrator is PathIntegrator::li of the reference's CPU tracer
// (crates/appearance-path-tracer/src/path_integrator.rs:103-307) with the
// camera of path_tracer.rs:42-45 and the pixel-centre uv of lib.rs:138-142,
// as written once in the library's spectral.h and compiled here against this
// oracle's own scene and binned-SAH BVH (oracle_bvh.cpp) instead of the
// device's compressed 8-wide BVH.  Closest hits agree bit for bit between the
// two traversals (minimum of (t, triangle id)), so the renders agree bit for
// bit.  The RGB-to-spectrum tables come from the library's spectral_fit.cpp,
// a host precomputation checked on its own by the CPU tests (round-trip
// colour error).  Parity of the reference's own numbers is unpinned: the
// reference crate does not build (missing build dependency and BVH crate), so
// no output of it exists to compare against.
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <thread>
#include <vector>

#include "../appearance_b200/csrc/spectral.h"
#include "../appearance_b200/csrc/spectral_fit.h"
#include "oracle_scene.h"

namespace {

using orc::OracleBvh;
using orc::Scene;

struct SpectralOracle {
  const Scene* scene;
  OracleBvh bvh;
  std::vector<spec::Material> mats;
  std::vector<float> env4;
  uint32_t env_w = 0, env_h = 0;
  float env_scale = 1.0f;
  spec::Sun sun{};
};

struct CpuGeo {
  const SpectralOracle& o;
  uint32_t env_w, env_h;
  float env_scale;
  spec::Sun sun;

  bool closest(spec::V3 p, spec::V3 d, float tmax, spec::Hit& h) const {
    orc::Hit r = o.bvh.closest(*o.scene, orc::v3(p.x, p.y, p.z), orc::v3(d.x, d.y, d.z), 0.0f, tmax, nullptr, nullptr);
    h.t = r.t;
    h.tri = r.tri;
    return r.tri != 0xFFFFFFFFu;
  }
  bool occluded(spec::V3 p, spec::V3 d, float tmax) const {
    return o.bvh.any(*o.scene, orc::v3(p.x, p.y, p.z), orc::v3(d.x, d.y, d.z), 0.0f, tmax);
  }
  void tri(uint32_t g, spec::V3* p0, spec::V3* p1, spec::V3* p2) const {
    orc::V3 a, b, c;
    o.scene->tri_verts(g, a, b, c);
    *p0 = spec::v3(a.x, a.y, a.z);
    *p1 = spec::v3(b.x, b.y, b.z);
    *p2 = spec::v3(c.x, c.y, c.z);
  }
  const spec::Material& material(uint32_t g) const {
    const orc::Instance& in = o.scene->instances[o.scene->tri_instance[g]];
    return o.mats[in.material_idx + o.scene->tri_material[in.first_index / 3 + (g - in.first_global_tri)]];
  }
  void env_texel(uint32_t idx, float c[4]) const {
    for (int k = 0; k < 4; ++k) c[k] = o.env4[4 * (size_t)idx + k];
  }
};

}  // namespace

extern "C" {

// Spectral tables and BVH for an oracle scene (orc_scene_new); the light and
// environment parameters mean what they mean in ap_spectral_setup.
void* orc_spectral_new(void* scene, const float* sun_dir3, const float* sun_rgb3, float sun_scale, float scene_radius,
                       float env_scale) {
  const Scene* s = (const Scene*)scene;
  SpectralOracle* o = new SpectralOracle();
  o->scene = s;
  o->bvh.build(*s);
  o->mats.resize(s->materials.size());
  spec::upsample_materials(reinterpret_cast<const float*>(s->materials.data()), (uint32_t)s->materials.size(),
                           o->mats.data());
  if (s->env_w && s->env_h) {
    o->env4.resize(4 * (size_t)s->env_w * s->env_h);
    spec::upsample_env(s->env.data(), (size_t)s->env_w * s->env_h, o->env4.data());
    o->env_w = s->env_w;
    o->env_h = s->env_h;
  }
  o->env_scale = env_scale;
  o->sun = spec::make_sun(sun_dir3, sun_rgb3, sun_scale, scene_radius);
  return o;
}

void orc_spectral_free(void* p) { delete (SpectralOracle*)p; }

// Rows [row0, row1) of a W x H image, spp samples per pixel, out 3 floats per
// pixel (linear sRGB, mean over samples).  inv_view / inv_proj: column-major.
void orc_spectral_render(void* p, const float* inv_view, const float* inv_proj, uint32_t W, uint32_t H, uint32_t row0,
                         uint32_t row1, uint32_t spp, int max_depth, uint32_t seed, uint32_t threads, float* out) {
  const SpectralOracle& o = *(const SpectralOracle*)p;
  CpuGeo g{o, o.env_w, o.env_h, o.env_scale, o.sun};
  std::atomic<uint32_t> next{row0};
  auto work = [&]() {
    for (uint32_t y = next.fetch_add(1); y < row1; y = next.fetch_add(1))
      for (uint32_t x = 0; x < W; ++x) {
        spec::V3 acc = spec::v3(0.0f, 0.0f, 0.0f);
        for (uint32_t k = 0; k < spp; ++k)
          acc = acc + spec::pixel_sample(g, inv_view, inv_proj, x, y, W, H, k, seed, max_depth);
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

// The upsampled material table (12 floats per material) and environment
// texels (4 floats each), for the tests of the tables.
void orc_spectral_tables(void* p, float* mats_out, float* env_out) {
  const SpectralOracle& o = *(const SpectralOracle*)p;
  if (mats_out) memcpy(mats_out, o.mats.data(), sizeof(spec::Material) * o.mats.size());
  if (env_out && !o.env4.empty()) memcpy(env_out, o.env4.data(), sizeof(float) * o.env4.size());
}

// Spectral building blocks, for the CPU tests: the analytic CIE functions
// and the 6504 K illuminant at one wavelength (out: x, y, z, illuminant);
// the albedo fit of one colour; wavelength sampling (lambda, pdf) of u.
void orc_spectral_cmf(float lambda, float* out4) {
  out4[0] = spec::cie_x(lambda);
  out4[1] = spec::cie_y(lambda);
  out4[2] = spec::cie_z(lambda);
  out4[3] = spec::illuminant(lambda);
}
void orc_spectral_fit(const float* rgb, float* coef3) { spec::fit_albedo(rgb, coef3); }
void orc_spectral_sigmoid(const float* coef3, float lambda, float* out) { *out = spec::sigmoid_poly(coef3, lambda); }
void orc_spectral_wavelength(float u, float* out2) {
  out2[0] = spec::sample_visible_wavelength(u);
  out2[1] = spec::visible_wavelength_pdf(out2[0]);
}
double orc_spectral_illuminant_norm() { return spec::illuminant_norm(); }

}  // extern "C"
