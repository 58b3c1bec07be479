// Spectral (hero-wavelength) rendering on sm_100a as a wavefront.
//
// One pass per sample index renders that sample for every pixel of the rows:
// the camera rays of all pixels, then up to max_depth + 1 rounds of
//   extend: persistent closest-hit traversal of the compacted ray queue;
//   shade:  spec::path_vertex (spectral.h) per live path -- emission or the
//           environment, the light sample's shadow ray, BSDF sampling and
//           Russian roulette -- pushing surviving paths and shadow rays into
//           the next queues (warp ballot + one atomic per warp);
//   shadow: persistent any-hit traversal of the shadow queue, adding the
//           light sample's contribution of unoccluded rays;
// then the pass's radiance goes through the XYZ sensor into the pixel sums.
// Each path runs exactly the vertex sequence of spec::li, so the image equals
// the per-pixel loop of the CPU restatement bit for bit.
//
// Radiance-cache mode (SpectralCache): after each extension round, k_svertex
// retires the paths reaching their prefix-th hit (query stored, path ended)
// and records the suffix vertices of a rotating 1/stride of the pixels; after
// the rounds the cache infers the retired queries (tensor-core MLP, mlp.cu),
// k_sapply adds throughput x the prediction upsampled to the path's
// wavelengths, and a batch of recorded vertices, with RGB targets from their
// spectral suffix radiance, trains it.
#include <algorithm>

#include "frame.cuh"
#include "persistent.cuh"
#include "spectral.cuh"
#include "spectral_data.h"

namespace ap {

namespace {

constexpr int kBlock = 128;

// The gold tables (spectral_data.h) in device memory, read through the
// read-only cache.
__device__ const float g_au_lambda[spec::kAuSamples] = {SPEC_AU_LAMBDA};
__device__ const float g_au_eta[spec::kAuSamples] = {SPEC_AU_ETA};
__device__ const float g_au_k[spec::kAuSamples] = {SPEC_AU_K};

// PiecewiseLinearSpectrum::reflectance over a gold table (spectrum.rs:552-566,
// find_interval_fast, math/mod.rs:97-113).
APD float au_sample(const float* vals, float l) {
  constexpr int n = spec::kAuSamples;
  if (l < __ldg(&g_au_lambda[0]) || l > __ldg(&g_au_lambda[n - 1])) return 0.0f;
  int size = n - 2, first = 1;
  while (size > 0) {
    const int half = size >> 1, middle = first + half;
    const bool pred = __ldg(&g_au_lambda[middle]) <= l;
    first = pred ? middle + 1 : first;
    size = pred ? size - (half + 1) : half;
  }
  const int o = min(max(first - 1, 0), n - 2);
  const float l0 = __ldg(&g_au_lambda[o]), l1 = __ldg(&g_au_lambda[o + 1]);
  const float a = __ldg(&vals[o]), b = __ldg(&vals[o + 1]);
  return a + (b - a) * ((l - l0) / (l1 - l0));
}

// Scene access of the spectral integrator (spectral.h's Geo): the flat scene,
// or (kTwo) a two-level world, whose shading data is the hit's instance (the
// last whose first global triangle id is at most g), its model's triangle,
// the vertices mapped to world space by the instance transform, and the
// normals with the transform's inverse transpose (the transpose of the
// world-to-object rows).
template <bool kTwo>
struct GpuGeo {
  const DevScene& s;
  const SpectralView& v;
  uint32_t env_w, env_h;
  float env_scale, env_pdf_integral;
  spec::Sun sun;

  APD void tri_index(uint32_t g, uint32_t* i0, uint32_t* i1, uint32_t* i2) const {
    const InstanceDev& in = s.instances[s.tri_instance[g]];
    const uint32_t fi = in.first_index + (g - in.first_global_tri) * 3;
    *i0 = in.first_vertex + s.indices[fi + 0];
    *i1 = in.first_vertex + s.indices[fi + 1];
    *i2 = in.first_vertex + s.indices[fi + 2];
  }
  // world-space vertices and normals of triangle g, and its material
  APD const spec::Material& fetch(uint32_t g, spec::TriGeo* tg) const {
    if (kTwo) return fetch2(g, tg);
    uint32_t vi[3];
    tri_index(g, &vi[0], &vi[1], &vi[2]);
    const float* n = s.normals_f;
    for (int k = 0; k < 3; ++k) {
      const float4 p = s.positions[vi[k]];
      tg->p[k] = spec::v3(p.x, p.y, p.z);
      tg->n[k] = spec::v3(n[3 * (size_t)vi[k]], n[3 * (size_t)vi[k] + 1], n[3 * (size_t)vi[k] + 2]);
    }
    tg->xform = false;
    const InstanceDev& in = s.instances[s.tri_instance[g]];
    return v.mats[in.material_idx + s.tri_material[in.first_index / 3 + (g - in.first_global_tri)]];
  }
  APD const spec::Material& fetch2(uint32_t g, spec::TriGeo* tg) const {
    const InstRec& in = v.tl.insts[__ldg(&v.mg.tri_inst[g])];
    const uint32_t t = __ldg(&v.mg.model_tri0[in.model]) + (g - in.tri_base);
    const float* m = in.o2w;
    for (int k = 0; k < 3; ++k) {
      const uint32_t vi = __ldg(&v.mg.indices[3 * (size_t)t + k]);
      const float4 p = v.mg.positions[vi];
      tg->p[k] = spec::v3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
                          m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
      const float* n = v.mg.normals + 3 * (size_t)vi;
      tg->n[k] = spec::v3(n[0], n[1], n[2]);
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) tg->nm[3 * r + c] = in.w2o[4 * c + r];
    tg->xform = true;
    return v.mats[__ldg(&v.mg.tri_mat[t])];
  }
  APD void env_rgb(uint32_t x, uint32_t y, float c[3]) const {
    const float* p = s.env + 3 * ((size_t)y * env_w + x);
    c[0] = __ldg(p);
    c[1] = __ldg(p + 1);
    c[2] = __ldg(p + 2);
  }
  APD void illum_coef(const float rgb[3], float out[4]) const {
    spec::illum_lookup(v.illum_tab, v.illum_norm, rgb, out);
  }
  APD float env_pdf_func(size_t i) const { return __ldg(v.env_pdf + i); }
  APD float au_eta(float l) const { return au_sample(g_au_eta, l); }
  APD float au_k(float l) const { return au_sample(g_au_k, l); }
};

// Per-path state and queues of P paths (one per pixel of the rows).
struct SpecBuffers {
  float4* rq_o[2];  // extension ray queue (by bounce parity): origin
  float4* rq_d[2];  //   direction, w = owning path (bits)
  uint4* hits;      // per extension queue slot: t, u, v (bits), triangle
  float4* sq_o;     // shadow ray queue: origin, w = tmax
  float4* sq_d;     //   direction, w = owning path (bits)
  float4* L;        // spectral radiance of the path (4 wavelengths)
  float4* beta;     // path throughput
  float4* lambda;   // the path's wavelengths
  float4* shc;      // contribution of the pending shadow ray
  float4* acc;      // linear sRGB sum over the samples so far (xyz)
  uint4* misc;      // sampler dimension, depth | specular << 16, eta_scale, p_b (bits)
  uint32_t* morton; // Morton index of the path's sampler pixel
  uint32_t* counters;  // per round: extension size, cursor, shadow size, cursor
  // closest-hit rays, nodes, triangles; any-hit rays, nodes, triangles (nodes
  // and triangles only in the counting form)
  unsigned long long* stats;
  // cache mode only
  float4* cq;       // per retired path (compacted): query of its last vertex (4 float4)
  float4* cT;       //   throughput at that vertex
  uint32_t* cown;   //   the path
  float* cout;      //   predicted RGB
  float4* rec;      // per training pixel and round: query (4), throughput, radiance so far, tag
  float4* bq;       // training batch queries
  float* bt;        // training batch targets (RGB)
  uint32_t* ccount; // [0] candidate records, [1] batch entries, [2] retired paths of the pass
  uint32_t* cbcount;  // per 256 record slots: records kept for the batch, then their first batch slot
};

constexpr uint32_t kSpecRecord = 7;  // float4 per recorded vertex

constexpr size_t kAlign = 256;

size_t carve(void* base, uint32_t P, const SpectralCache* rc, SpecBuffers* b) {
  char* p = static_cast<char*>(base);
  size_t off = 0;
  auto take = [&](size_t bytes) -> void* {
    void* r = p ? p + off : nullptr;
    off += (bytes + kAlign - 1) & ~(kAlign - 1);
    return r;
  };
  const size_t f4 = sizeof(float4) * (size_t)P;
  for (int q = 0; q < 2; ++q) {
    b->rq_o[q] = static_cast<float4*>(take(f4));
    b->rq_d[q] = static_cast<float4*>(take(f4));
  }
  b->hits = static_cast<uint4*>(take(sizeof(uint4) * (size_t)P));
  b->sq_o = static_cast<float4*>(take(f4));
  b->sq_d = static_cast<float4*>(take(f4));
  b->L = static_cast<float4*>(take(f4));
  b->beta = static_cast<float4*>(take(f4));
  b->lambda = static_cast<float4*>(take(f4));
  b->shc = static_cast<float4*>(take(f4));
  b->acc = static_cast<float4*>(take(f4));
  b->misc = static_cast<uint4*>(take(sizeof(uint4) * (size_t)P));
  b->morton = static_cast<uint32_t*>(take(sizeof(uint32_t) * (size_t)P));
  b->counters = static_cast<uint32_t*>(take(sizeof(uint32_t) * 4 * (kSpectralMaxDepth + 2)));
  b->stats = static_cast<unsigned long long*>(take(6 * sizeof(unsigned long long)));
  b->cq = b->cT = b->rec = b->bq = nullptr;
  b->cout = b->bt = nullptr;
  b->ccount = b->cown = b->cbcount = nullptr;
  if (rc) {
    const size_t slots = ((size_t)P / rc->stride + 1) * kRcMaxBounces;
    b->cq = static_cast<float4*>(take(4 * f4));
    b->cT = static_cast<float4*>(take(f4));
    b->cown = static_cast<uint32_t*>(take(sizeof(uint32_t) * (size_t)P));
    b->cout = static_cast<float*>(take(3 * sizeof(float) * (size_t)P));
    b->rec = static_cast<float4*>(take(sizeof(float4) * kSpecRecord * slots));
    b->bq = static_cast<float4*>(take(sizeof(float4) * 4 * (size_t)rc->batch));
    b->bt = static_cast<float*>(take(sizeof(float) * 3 * (size_t)rc->batch));
    b->ccount = static_cast<uint32_t*>(take(3 * sizeof(uint32_t)));
    b->cbcount = static_cast<uint32_t*>(take(sizeof(uint32_t) * ((slots + 255) / 256)));
  }
  return off;
}

APD float4 f4(spec::S4 a) { return make_float4(a.v[0], a.v[1], a.v[2], a.v[3]); }
APD spec::S4 s4of(float4 a) { return spec::S4{{a.x, a.y, a.z, a.w}}; }

// Appends (o, w0), (d, owner) to a queue with one atomic per warp.
APD void push(bool want, uint32_t* size, float4* qo, float4* qd, spec::V3 o, float w0, spec::V3 d, uint32_t owner) {
  const unsigned active = __activemask();
  const unsigned bal = __ballot_sync(active, want);
  if (!want) return;
  const int lane = (int)lane_id();
  const int leader = __ffs(bal) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(size, (uint32_t)__popc(bal));
  base = __shfl_sync(bal, base, leader);
  const uint32_t slot = base + __popc(bal & ((1u << lane) - 1u));
  qo[slot] = make_float4(o.x, o.y, o.z, w0);
  qd[slot] = make_float4(d.x, d.y, d.z, __uint_as_float(owner));
}

// Camera rays of one sample pass: the sample is the reference's 1-spp frame
// with seed `frame_seed`; the sampler starts at dimension 0 of the path's
// sampler pixel and gives the wavelengths their first draw.
__global__ void __launch_bounds__(kBlock) k_sgen(SpecBuffers b, SpectralCamera cam, uint32_t W, uint32_t H,
                                                 uint32_t row0, uint32_t P, uint32_t sample, uint32_t digits,
                                                 uint64_t frame_seed) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const uint32_t x = p % W, y = row0 + p / W;
  spec::V3 o, d;
  spec::camera_ray(cam.inv_view, cam.inv_proj, x, y, W, H, &o, &d);
  uint32_t px, py;
  spec::sampler_pixel(x, y, W, H, &px, &py);
  spec::ZSobol z{spec::morton2(px, py), digits, frame_seed, 0u};
  const spec::Wavelengths w = spec::sample_visible(z.get1d());
  b.rq_o[0][p] = make_float4(o.x, o.y, o.z, 0.0f);
  b.rq_d[0][p] = make_float4(d.x, d.y, d.z, __uint_as_float(p));
  b.lambda[p] = f4(w.lambda);
  b.L[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  b.beta[p] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  b.misc[p] = make_uint4(z.dim, 0u, __float_as_uint(1.0f), __float_as_uint(1.0f));
  b.morton[p] = z.morton;
  if (sample == 0) b.acc[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// The traversal loop of a scene: flat, or two-level when `tl` is given.
template <bool kAny, bool kCount, bool kTwo, class Load, class Store>
APD void trace_loop(const DevScene& s, const TwoLevel& tl, uint32_t count, uint32_t* cursor, Load load, Store store) {
  if (kTwo) persistent_trace2<kAny, kCount>(s, tl, count, cursor, load, store);
  else persistent_trace<kAny, kCount>(s, count, cursor, load, store);
}

template <bool kCount, bool kTwo>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_sextend(DevScene s, TwoLevel tl, SpecBuffers b,
                                                                     uint32_t round, uint32_t P) {
  const uint32_t count = round == 0 ? P : min(b.counters[4 * round], P);
  if (blockIdx.x == 0 && threadIdx.x == 0 && count) atomicAdd(&b.stats[0], (unsigned long long)count);
  const float4* qo = b.rq_o[round & 1];
  const float4* qd = b.rq_d[round & 1];
  trace_loop<false, kCount, kTwo>(
      s, tl, count, &b.counters[4 * round + 1],
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const float4 a = qo[i], c = qd[i];
        o = f3(a.x, a.y, a.z);
        d = f3(c.x, c.y, c.z);
        tmax = 1e30f;
      },
      [&](uint32_t i, const Trav& t, const Visits& vc) {
        b.hits[i] = make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v),
                               t.hit.tri);
        if (kCount) {
          atomicAdd(&b.stats[1], (unsigned long long)vc.nodes);
          atomicAdd(&b.stats[2], (unsigned long long)vc.tris);
        }
      });
}

#ifndef AP_SSHADE_MIN_BLOCKS
#define AP_SSHADE_MIN_BLOCKS 8  // resident blocks per SM the shading kernel is register-capped for (measured)
#endif
template <bool kTwo>
__global__ void __launch_bounds__(kBlock, AP_SSHADE_MIN_BLOCKS) k_sshade(DevScene s, SpectralView v, SpecBuffers b,
                                                                     uint32_t round, uint32_t P, int max_depth,
                                                                     uint32_t digits, uint64_t frame_seed) {
  const uint32_t count = round == 0 ? P : min(b.counters[4 * round], P);
  const float4* qo = b.rq_o[round & 1];
  const float4* qd = b.rq_d[round & 1];
  float4* no = b.rq_o[(round + 1) & 1];
  float4* nd = b.rq_d[(round + 1) & 1];
  const GpuGeo<kTwo> g{s, v, v.env_w, v.env_h, v.env_scale, v.env_pdf_integral, v.sun};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float4 ro = qo[i], rd = qd[i];
    const uint32_t owner = __float_as_uint(rd.w);
    const uint4 hh = b.hits[i];
    if (hh.w == kRcRetired) continue;  // ended in the radiance cache at this vertex
    spec::V3 o = spec::v3(ro.x, ro.y, ro.z), d = spec::v3(rd.x, rd.y, rd.z);
    const spec::Hit h{__uint_as_float(hh.x), __uint_as_float(hh.y), __uint_as_float(hh.z), hh.w};
    const uint4 m = b.misc[owner];
    spec::PathState ps{s4of(b.L[owner]), s4of(b.beta[owner]), __uint_as_float(m.z), __uint_as_float(m.w),
                       (m.y >> 16) != 0u, (int)(m.y & 0xffffu),
                       spec::ZSobol{b.morton[owner], digits, frame_seed, m.x}};
    const spec::S4 lam = s4of(b.lambda[owner]);
    bool shadow;
    spec::ShadowRay sh = {};
    const bool more = spec::path_vertex(g, o, d, hh.w != kNoHit ? &h : nullptr, lam, ps, max_depth, &shadow, &sh);
    b.L[owner] = f4(ps.L);
    if (more) {
      b.beta[owner] = f4(ps.beta);
      b.misc[owner] = make_uint4(ps.smp.dim, (uint32_t)ps.depth | (ps.specular ? 1u << 16 : 0u),
                                 __float_as_uint(ps.eta_scale), __float_as_uint(ps.p_b));
    }
    if (shadow) b.shc[owner] = f4(sh.c);
    push(shadow, &b.counters[4 * round + 2], b.sq_o, b.sq_d, sh.o, sh.tmax, sh.d, owner);
    push(more, &b.counters[4 * (round + 1)], no, nd, o, 0.0f, d, owner);
  }
}

template <bool kCount, bool kTwo>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_sshadow(DevScene s, TwoLevel tl, SpecBuffers b,
                                                                     uint32_t round, uint32_t P) {
  const uint32_t count = min(b.counters[4 * round + 2], P);
  if (blockIdx.x == 0 && threadIdx.x == 0 && count) atomicAdd(&b.stats[3], (unsigned long long)count);
  trace_loop<true, kCount, kTwo>(
      s, tl, count, &b.counters[4 * round + 3],
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const float4 a = b.sq_o[i], c = b.sq_d[i];
        o = f3(a.x, a.y, a.z);
        d = f3(c.x, c.y, c.z);
        tmax = a.w;
      },
      [&](uint32_t i, const Trav& t, const Visits& vc) {
        if (kCount) {
          atomicAdd(&b.stats[4], (unsigned long long)vc.nodes);
          atomicAdd(&b.stats[5], (unsigned long long)vc.tris);
        }
        if (t.hit.tri != kNoHit) return;  // occluded
        const uint32_t owner = __float_as_uint(b.sq_d[i].w);
        b.L[owner] = f4(s4of(b.L[owner]) + s4of(b.shc[owner]));
      });
}

// ---- radiance-cache mode ----

APD bool training_path(uint32_t p, uint32_t pass, uint32_t seed, uint32_t stride) {
  return p % stride == (pass * 7u + 3u + seed) % stride;
}

// The cache's query at a hit (position, roughness, outgoing direction, diffuse
// albedo, specular albedo) from the scene's RGB material, as the RGB frame
// builds it.
APD void spec_query(const DevScene& s, uint32_t tri, spec::V3 p, spec::V3 wo, float4* q) {
  const InstanceDev& in = s.instances[s.tri_instance[tri]];
  const MaterialDev* m = s.materials + in.material_idx + s.tri_material[in.first_index / 3 + (tri - in.first_global_tri)];
  const float3 col = f3(m->color[0], m->color[1], m->color[2]);
  const float kd = (1.0f - m->metallic) * (1.0f - m->transmission);
  const float3 spec = f3s(0.08f * m->specular) * (1.0f - m->metallic) + col * m->metallic;
  q[0] = make_float4(p.x, p.y, p.z, m->roughness);
  q[1] = make_float4(wo.x, wo.y, wo.z, 0.0f);
  q[2] = make_float4(col.x * kd, col.y * kd, col.z * kd, spec.x);
  q[3] = make_float4(spec.y, spec.z, 0.0f, 0.0f);
}

__global__ void __launch_bounds__(kBlock) k_svertex(DevScene s, SpecBuffers b, SpectralCache rc, uint32_t round,
                                                    uint32_t P, uint32_t pass, uint32_t seed) {
  const uint32_t count = round == 0 ? P : min(b.counters[4 * round], P);
  const float4* qo = b.rq_o[round & 1];
  const float4* qd = b.rq_d[round & 1];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint4 hh = b.hits[i];
    if (hh.w == kNoHit) continue;
    const float4 rd = qd[i];
    const uint32_t p = __float_as_uint(rd.w);
    const bool tp = training_path(p, pass, seed, rc.stride);
    if (!tp && round != rc.prefix) continue;
    if (tp && (round == 0 || round >= kRcMaxBounces)) continue;
    const float4 ro = qo[i];
    const float t = __uint_as_float(hh.x);
    const spec::V3 o = spec::v3(ro.x, ro.y, ro.z), d = spec::v3(rd.x, rd.y, rd.z);
    float4 q[4];
    spec_query(s, hh.w, o + d * t, -d, q);
    if (tp) {
      float4* r = b.rec + ((size_t)(p / rc.stride) * kRcMaxBounces + round) * kSpecRecord;
      r[0] = q[0]; r[1] = q[1]; r[2] = q[2]; r[3] = q[3];
      r[4] = b.beta[p];
      r[5] = b.L[p];
      r[6] = make_float4((float)(pass + 1), 0.0f, 0.0f, 0.0f);  // tag: the pass that wrote it
    } else {  // retired: its query goes to the next compact slot (one atomic per warp)
      const unsigned m = __activemask();
      const int lane = (int)lane_id(), leader = __ffs(m) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(&b.ccount[2], (uint32_t)__popc(m));
      const uint32_t j = __shfl_sync(m, base, leader) + __popc(m & ((1u << lane) - 1u));
      float4* dst = b.cq + 4 * (size_t)j;
      dst[0] = q[0]; dst[1] = q[1]; dst[2] = q[2]; dst[3] = q[3];
      b.cT[j] = b.beta[p];
      b.cown[j] = p;
      b.hits[i].w = kRcRetired;
    }
  }
}

// For each retired path: L += throughput x the prediction, upsampled to the
// path's wavelengths.
__global__ void __launch_bounds__(kBlock) k_sapply(SpectralView v, SpecBuffers b, uint32_t P) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= min(b.ccount[2], P)) return;
  const uint32_t p = b.cown[j];
  float rgb[3] = {b.cout[3 * (size_t)j], b.cout[3 * (size_t)j + 1], b.cout[3 * (size_t)j + 2]};
  float c[4];
  spec::illum_lookup(v.illum_tab, v.illum_norm, rgb, c);
  const spec::S4 lam = s4of(b.lambda[p]);
  spec::S4 Lc;
  for (int i = 0; i < 4; ++i) Lc.v[i] = spec::illum_at(c, lam.v[i]);
  b.L[p] = f4(s4of(b.L[p]) + s4of(b.cT[j]) * Lc);
}

__global__ void k_scount(SpecBuffers b, SpectralCache rc, uint32_t slots, float tag) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = k < slots && b.rec[(size_t)k * kSpecRecord + 6].x == tag;
  const unsigned bal = __ballot_sync(0xffffffffu, ok);
  if ((threadIdx.x & 31) == 0 && bal) atomicAdd(&b.ccount[0], (uint32_t)__popc(bal));
}

// Keeps each of this pass's records with probability batch / count; its
// target is the RGB of the path's radiance after the vertex divided by the
// throughput at the vertex, per wavelength (clamped at 0).
APD bool s_kept(const SpecBuffers& b, const SpectralCache& rc, uint32_t k, uint32_t slots, float tag, uint32_t pass,
                uint32_t seed, uint32_t P) {
  if (k >= slots || b.rec[(size_t)k * kSpecRecord + 6].x != tag) return false;
  const uint32_t cand = b.ccount[0];
  const float keep = cand <= rc.batch ? 1.0f : (float)rc.batch / (float)cand;
  const float u = (float)(spec::pcg(k * 2654435761u ^ spec::pcg(pass + seed * 7919u)) >> 8) * (1.0f / 16777216.0f);
  return u < keep && (k / kRcMaxBounces) * rc.stride + (pass * 7u + 3u + seed) % rc.stride < P;
}

// Records kept per block of 256 slots (count_scan turns them into the blocks'
// first batch slots, so the batch is in record order).
__global__ void k_skeep(SpecBuffers b, SpectralCache rc, uint32_t slots, float tag, uint32_t pass, uint32_t seed,
                        uint32_t P) {
  uint32_t tot;
  block_prefix(s_kept(b, rc, blockIdx.x * blockDim.x + threadIdx.x, slots, tag, pass, seed, P), &tot);
  if (threadIdx.x == 0) b.cbcount[blockIdx.x] = tot;
}

__global__ void k_sbatch(SpecBuffers b, SpectralCache rc, uint32_t slots, float tag, uint32_t pass, uint32_t seed,
                         uint32_t P) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool kept = s_kept(b, rc, k, slots, tag, pass, seed, P);
  uint32_t tot;
  const uint32_t slot = b.cbcount[blockIdx.x] + block_prefix(kept, &tot);
  if (!kept || slot >= rc.batch) return;
  const float4* r = b.rec + (size_t)k * kSpecRecord;
  const uint32_t p = (k / kRcMaxBounces) * rc.stride + (pass * 7u + 3u + seed) % rc.stride;
  const spec::S4 Lend = s4of(b.L[p]), Lv = s4of(r[5]), T = s4of(r[4]);
  spec::S4 dl;
  for (int j = 0; j < 4; ++j) dl.v[j] = T.v[j] > 0.0f ? dm::fmax(Lend.v[j] - Lv.v[j], 0.0f) / T.v[j] : 0.0f;
  spec::Wavelengths w;
  w.lambda = s4of(b.lambda[p]);
  for (int j = 0; j < 4; ++j) w.pdf.v[j] = spec::visible_wavelength_pdf(w.lambda.v[j]);
  const spec::V3 rgb = spec::xyz_to_srgb(spec::to_xyz(dl, w));
  float4* q = b.bq + 4 * (size_t)slot;
  q[0] = r[0]; q[1] = r[1]; q[2] = r[2]; q[3] = r[3];
  b.bt[3 * (size_t)slot + 0] = dm::fmax(rgb.x, 0.0f);
  b.bt[3 * (size_t)slot + 1] = dm::fmax(rgb.y, 0.0f);
  b.bt[3 * (size_t)slot + 2] = dm::fmax(rgb.z, 0.0f);
}

__global__ void __launch_bounds__(kBlock) k_saccum(SpecBuffers b, uint32_t P, bool last, float inv, float* out) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  spec::Wavelengths w;
  w.lambda = s4of(b.lambda[p]);
  for (int k = 0; k < 4; ++k) w.pdf.v[k] = spec::visible_wavelength_pdf(w.lambda.v[k]);
  const spec::V3 rgb = spec::xyz_to_srgb(spec::to_xyz(s4of(b.L[p]), w));
  const float4 a = b.acc[p];
  const spec::V3 acc = spec::v3(a.x, a.y, a.z) + rgb;
  if (last) {
    out[3 * (size_t)p + 0] = acc.x * inv;
    out[3 * (size_t)p + 1] = acc.y * inv;
    out[3 * (size_t)p + 2] = acc.z * inv;
  } else {
    b.acc[p] = make_float4(acc.x, acc.y, acc.z, 0.0f);
  }
}

}  // namespace

void spectral_env_distribution(const float* rgb, uint32_t W, uint32_t H, float* func, float* integral) {
  // Texture::get_sampling_distribution (appearance-texture lib.rs:193-205):
  // the texel's channel mean, stored x-major
  const size_t n = (size_t)W * H;
  for (uint32_t y = 0; y < H; ++y)
    for (uint32_t x = 0; x < W; ++x) {
      const float* p = rgb + 3 * ((size_t)y * W + x);
      func[(size_t)x * H + y] = (p[0] + p[1] + p[2]) / 3.0f;
    }
  // InfiniteLight::new (infinite_light.rs:41-54): minus the mean, clamped at 0
  float average = 0.0f;
  for (size_t i = 0; i < n; ++i) average += func[i];
  average /= (float)n;
  for (size_t i = 0; i < n; ++i) func[i] = spec::fmax_nan(func[i] - average, 0.0f);
  // PiecewiseConstant2D::new (piecewise_constant.rs:101-125) over rows of W
  // of that x-major array, and PiecewiseConstant1D's integrals (:21-49)
  float marginal = 0.0f;
  for (uint32_t v = 0; v < H; ++v) {
    float row = 0.0f;
    for (uint32_t u = 0; u < W; ++u) row = row + func[(size_t)v * W + u] * 1.0f / (float)W;
    marginal = marginal + row * 1.0f / (float)H;
  }
  *integral = marginal;
}

// Sample passes in flight at once without the cache (launch_spectral).  On a
// 2048^2 x 16 spp city image (Msamples/s): one pass with its shadow rays beside
// the next extension 448, two passes 476, three 490, four 503.
#ifndef AP_SPEC_PASSES
#define AP_SPEC_PASSES 4
#endif
constexpr int kSpecPasses = AP_SPEC_PASSES;
static_assert(kSpecPasses >= 2 && kSpecPasses <= 4, "two to four sample passes in flight");

// Without the cache the work area holds kSpecPasses sets of path state.
size_t spectral_work_bytes(uint32_t P, const SpectralCache* rc) {
  SpecBuffers b;
  const size_t one = carve(nullptr, P, rc, &b);
  return rc ? one : kSpecPasses * one;
}

const unsigned long long* spectral_stats(void* work, uint32_t P, const SpectralCache* rc) {
  SpecBuffers b;
  carve(work, P, rc, &b);
  return b.stats;
}

int launch_spectral(const DevScene& s, const SpectralView& v, const SpectralCamera& cam, uint32_t W, uint32_t H,
                    uint32_t row0, uint32_t row1, uint32_t spp, int max_depth, uint32_t seed, float* out, void* work,
                    int num_sms, bool count_visits, const SpectralCache* rc, cudaStream_t st,
                    const FrameStreams* fs) {
  const uint32_t P = W * (row1 - row0);
  const bool overlap = fs && fs->side && fs->fork && fs->join && !count_visits;
  // kSpecPasses sample passes in flight: sample k on stream k % kSpecPasses
  // (`st`, fs->side, fs->side2, fs->side3), each with its own path state; the
  // accumulator and the counters are shared, and every pass adds to the
  // accumulator after the previous pass did (an event between the streams), so
  // the sum's order is unchanged.
  const bool pipe = overlap && !rc && spp > 1 && (kSpecPasses < 3 || fs->side2) && (kSpecPasses < 4 || fs->side3);
  bool shadow_pending = false;  // a shadow pass in flight on fs->side
  SpecBuffers bufs[kSpecPasses];
  const size_t set_bytes = carve(work, P, rc, &bufs[0]);
  if (pipe) {
    for (int h = 1; h < kSpecPasses; ++h) {
      carve(static_cast<char*>(work) + h * set_bytes, P, nullptr, &bufs[h]);
      bufs[h].acc = bufs[0].acc;
      bufs[h].stats = bufs[0].stats;
    }
  }
  SpecBuffers& b = bufs[0];
  const uint32_t slots = rc ? (P / rc->stride + 1) * kRcMaxBounces : 0u;
  if (rc) cudaMemsetAsync(b.rec, 0, sizeof(float4) * kSpecRecord * slots, st);  // no tags from an earlier call
  const uint32_t rounds = (uint32_t)max_depth + 1;
  const uint32_t digits = spec::zsobol_digits(W, H);
  const bool two = v.two_level != 0;
  const int linear = (int)((P + kBlock - 1) / kBlock);
  const int persistent = num_sms * kTraceMinBlocks;
  const int shade = std::min(linear, num_sms * 16);
  int launches = 0;
  cudaMemsetAsync(b.stats, 0, 6 * sizeof(unsigned long long), st);
  if (pipe) {
    const cudaStream_t streams[4] = {st, fs->side, fs->side2, fs->side3};
    cudaEventRecord(fs->fork, st);
    for (int h = 1; h < kSpecPasses; ++h) cudaStreamWaitEvent(streams[h], fs->fork, 0);
    for (uint32_t k = 0; k < spp; ++k) {
      const int h = (int)(k % (uint32_t)kSpecPasses);
      const cudaStream_t sk = streams[h];
      const SpecBuffers& bk = bufs[h];
      cudaMemsetAsync(bk.counters, 0, sizeof(uint32_t) * 4 * (rounds + 1), sk);
      k_sgen<<<linear, kBlock, 0, sk>>>(bk, cam, W, H, row0, P, k, digits, (uint64_t)seed + k);
      ++launches;
      for (uint32_t r = 0; r < rounds; ++r) {
        if (two) {
          k_sextend<false, true><<<persistent, kBlock, 0, sk>>>(s, v.tl, bk, r, P);
          k_sshade<true><<<shade, kBlock, 0, sk>>>(s, v, bk, r, P, max_depth, digits, (uint64_t)seed + k);
          k_sshadow<false, true><<<persistent, kBlock, 0, sk>>>(s, v.tl, bk, r, P);
        } else {
          k_sextend<false, false><<<persistent, kBlock, 0, sk>>>(s, v.tl, bk, r, P);
          k_sshade<false><<<shade, kBlock, 0, sk>>>(s, v, bk, r, P, max_depth, digits, (uint64_t)seed + k);
          k_sshadow<false, false><<<persistent, kBlock, 0, sk>>>(s, v.tl, bk, r, P);
        }
        launches += 3;
      }
      if (k > 0) cudaStreamWaitEvent(sk, fs->join, 0);  // the previous pass's accumulation
      k_saccum<<<linear, kBlock, 0, sk>>>(bk, P, k + 1 == spp, 1.0f / (float)spp, out);
      cudaEventRecord(fs->join, sk);
      ++launches;
    }
    // the last pass recorded fs->join after its accumulation, which followed every other pass's
    cudaStreamWaitEvent(st, fs->join, 0);
    return launches;
  }
  for (uint32_t k = 0; k < spp; ++k) {
    cudaMemsetAsync(b.counters, 0, sizeof(uint32_t) * 4 * (rounds + 1), st);
    if (rc) cudaMemsetAsync(b.ccount + 2, 0, sizeof(uint32_t), st);
    k_sgen<<<linear, kBlock, 0, st>>>(b, cam, W, H, row0, P, k, digits, (uint64_t)seed + k);
    ++launches;
    for (uint32_t r = 0; r < rounds; ++r) {
      if (two) {
        if (count_visits) k_sextend<true, true><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
        else k_sextend<false, true><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
      } else {
        if (count_visits) k_sextend<true, false><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
        else k_sextend<false, false><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
      }
      if (shadow_pending) {  // the previous round's shadow rays, traced beside this extension
        cudaEventRecord(fs->join, fs->side);
        cudaStreamWaitEvent(st, fs->join, 0);
        shadow_pending = false;
      }
      if (rc) {
        k_svertex<<<shade, kBlock, 0, st>>>(s, b, *rc, r, P, k, seed);
        ++launches;
      }
      if (two) k_sshade<true><<<shade, kBlock, 0, st>>>(s, v, b, r, P, max_depth, digits, (uint64_t)seed + k);
      else k_sshade<false><<<shade, kBlock, 0, st>>>(s, v, b, r, P, max_depth, digits, (uint64_t)seed + k);
      if (overlap && r + 1 < rounds) {
        // only the next shading pass reads what these rays add to L
        cudaEventRecord(fs->fork, st);
        cudaStreamWaitEvent(fs->side, fs->fork, 0);
        if (two) k_sshadow<false, true><<<persistent, kBlock, 0, fs->side>>>(s, v.tl, b, r, P);
        else k_sshadow<false, false><<<persistent, kBlock, 0, fs->side>>>(s, v.tl, b, r, P);
        shadow_pending = true;
      } else if (count_visits) {
        if (two) k_sshadow<true, true><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
        else k_sshadow<true, false><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
      } else {
        if (two) k_sshadow<false, true><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
        else k_sshadow<false, false><<<persistent, kBlock, 0, st>>>(s, v.tl, b, r, P);
      }
      launches += 3;
    }
    if (rc) {
      rc_infer_device(rc->cache, b.cq, P, b.cout, st, b.ccount + 2);  // the retired queries only
      k_sapply<<<linear, kBlock, 0, st>>>(v, b, P);
      launches += 2;
      if (rc->train) {
        const float tag = (float)(k + 1);
        const int sb = (int)((slots + 255) / 256);
        cudaMemsetAsync(b.ccount, 0, 2 * sizeof(uint32_t), st);
        k_scount<<<sb, 256, 0, st>>>(b, *rc, slots, tag);
        k_skeep<<<sb, 256, 0, st>>>(b, *rc, slots, tag, k, seed, P);
        count_scan(b.cbcount, (uint32_t)sb, b.ccount + 1, rc->batch, st);
        k_sbatch<<<sb, 256, 0, st>>>(b, *rc, slots, tag, k, seed, P);
        rc_train_device(rc->cache, b.bq, b.bt, b.ccount + 1, rc->batch, rc->lr, 1, st);
        launches += 6;
      }
    }
    k_saccum<<<linear, kBlock, 0, st>>>(b, P, k + 1 == spp, 1.0f / (float)spp, out);
    ++launches;
  }
  return launches;
}

}  // namespace ap
