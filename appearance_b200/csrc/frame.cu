// Wavefront path-tracing frame for sm_100a.
//
// Pass structure and per-pixel arithmetic follow PathTracerGpu::render
// (crates/appearance-path-tracer-gpu/src/lib.rs:314-615) and its WGSL passes;
// the data layout and scheduling are this library's own:
//   * per-pixel state in 16-byte SoA records (frame.cuh);
//   * the path-extension ray of every bounce is traced by a persistent kernel
//     that fetches 32 rays per warp from a compacted queue of live paths;
//   * live paths are re-queued by warp ballot + popc + one atomic per warp;
//   * shading, next-event estimation, the GI candidate path and ReSTIR
//     resampling trace their short rays inline (traverse.cuh);
//   * the a-trous filter stages each 16x16 tile with its 2*2^i halo through
//     shared memory.
#include <algorithm>

#include "dev_shade.cuh"
#include "frame.cuh"
#include "persistent.cuh"
#include "traverse.cuh"
#include "traverse2.cuh"

namespace ap {

namespace {

constexpr int kBlock = 128;

struct Consts {
  uint32_t W, H, P;
  uint32_t bounce, seed, frame_idx, qin, qout;
  uint32_t sample;
  FrameConfig cfg;
};

APD float3 ray_dir(const float4 r) { return unpack_oct30(__float_as_uint(r.w)); }
APD float3 ray_org(const float4 r) { return f3(r.x, r.y, r.z); }

// ---- hit attributes (trace.wgsl:101-201) ----
struct Surface {
  uint32_t material_idx;
  float3 hit_point, n;
  bool back_face;
  Frame frame;
};
APD Surface surface(const DevScene& s, const Hit& h, float3 origin, float3 direction, const MaterialDev** mat) {
  Surface sf;
  uint32_t inst_idx = s.tri_instance[h.tri];
  const InstanceDev in = s.instances[inst_idx];
  uint32_t prim = h.tri - in.first_global_tri;
  float bx = 1.0f - h.u - h.v;
  uint32_t fi = in.first_index + prim * 3;
  float3 n0 = unpack_oct30(s.normals[in.first_vertex + s.indices[fi + 0]]);
  float3 n1 = unpack_oct30(s.normals[in.first_vertex + s.indices[fi + 1]]);
  float3 n2 = unpack_oct30(s.normals[in.first_vertex + s.indices[fi + 2]]);
  sf.material_idx = in.material_idx + s.tri_material[in.first_index / 3 + prim];
  *mat = s.materials + sf.material_idx;
  float3 hit_n = normalize(n0 * bx + n1 * h.u + n2 * h.v);
  sf.hit_point = origin + direction * h.t;
  float3 w_out = -direction;
  sf.back_face = dot(w_out, hit_n) < 0.0f;
  float3 ff = sf.back_face ? hit_n * -1.0f : hit_n;
  sf.n = ff;
  sf.frame.n = ff;
  sf.frame.t2w = onb(ff);
  if ((*mat)->clearcoat > 0.0f) {
    sf.frame.cc_t2w = onb(ff);
  } else {
    sf.frame.cc_t2w.c0 = f3s(0.0f);
    sf.frame.cc_t2w.c1 = f3s(0.0f);
    sf.frame.cc_t2w.c2 = f3s(0.0f);
  }
  return sf;
}

APD bool shadow_ray(const DevScene& s, float3 origin, float3 dir, float d, float3 n) {
  return !trace_any(s, origin + n * 1e-4f, dir, d - 1e-4f * 2.0f);
}

// ---- InlinePathTracer::trace with the approx() config (inline_path_tracer.wgsl:51-256) ----
APD float3 inline_trace(const DevScene& s, float3 origin, float3 direction, float3 throughput, float3* first_hit,
                        uint32_t& rng) {
  float3 acc = f3s(0.0f);
  Hit h;
  if (trace_closest(s, origin + direction * 1e-4f, direction, 1000.0f - 1e-4f * 2.0f, h)) {
    const MaterialDev* m;
    Surface sf = surface(s, h, origin, direction, &m);
    Bsdf b = load_bsdf(m);
    float3 wo = -direction;
    float pdf = 0.0f;
    float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng), r3 = rnd(rng), r4 = rnd(rng);
    LightSample ls = sample_uniform(s, r0, r1, r2, make_float2(r3, r4), &pdf);
    float W = 1.0f / pdf;
    if (W > 0.0f) {
      LightEval ev = load_eval(s, ls, sf.hit_point);
      float3 sdir = normalize(ev.point - sf.hit_point);
      float sd = dist(ev.point, sf.hit_point);
      float ndl = dot(sdir, sf.n);
      if (ndl > 0.0f && shadow_ray(s, sf.hit_point, sdir, sd, sf.n)) {
        float sp = 0.0f;
        float3 refl = disney_eval(b, sf.frame, wo, sdir, &sp);
        acc = acc + throughput * refl * ev.emission * ndl * W;
      }
    }
    *first_hit = sf.hit_point;
    return acc;
  }
  *first_hit = origin + direction * 1000.0f;
  return acc + throughput * sky_radiance(s, direction, true);
}

APD Frame ctx_frame(const uint4 c) {
  Frame fr;
  fr.n = unpack_oct30(c.z);
  fr.t2w = onb(fr.n);
  fr.cc_t2w = onb(unpack_oct30(c.w));
  return fr;
}

// GiReservoir::phat (inline_path_tracer.wgsl:299-331)
APD float gi_phat(const DevScene& s, const GiRes& r, const uint4 c, float3 T, float3 hit, float3 wo) {
  Bsdf b = load_bsdf(s.materials + c.x);
  Frame fr = ctx_frame(c);
  float3 wi = normalize(r.point - hit);
  float sp = 0.0f;
  float3 refl = disney_eval(b, fr, wo, wi, &sp);
  float cos_in = dm::fabs_(dot(wi, fr.n));
  float3 local = cos_in * refl;
  float3 gi_origin = hit + wi * 0.0001f;
  float3 tr = T * local;
  uint32_t prng = r.phat_rng;
  float3 pt;
  return luma(inline_trace(s, gi_origin, wi, tr, &pt, prng));
}

// LightSample::phat (di_reservoir.wgsl:58-97)
APD float ls_phat(const DevScene& s, const LightSample& l, const uint4 c, float3 hit, float3 wo, bool vis) {
  LightEval ev = load_eval(s, l, hit);
  Bsdf b = load_bsdf(s.materials + c.x);
  Frame fr = ctx_frame(c);
  float3 wi = normalize(ev.point - hit);
  float wdn = dot(wi, fr.n);
  if (wdn > 0.0f) {
    bool visible = true;
    if (vis) visible = shadow_ray(s, hit, wi, dist(ev.point, hit), fr.n);
    if (visible) {
      float sp = 0.0f;
      float3 refl = disney_eval(b, fr, wo, wi, &sp);
      return luma(refl * wdn * ev.emission);
    }
  }
  return 0.0f;
}

APD DiRes di_new() {
  DiRes r;
  r.M = r.W = r.wsum = r.phat = 0.0f;
  r.s = ls_empty();
  return r;
}
APD GiRes gi_new() {
  GiRes r;
  r.M = r.W = r.wsum = r.phat = 0.0f;
  r.point = f3s(0.0f);
  r.phat_rng = 0u;
  return r;
}

// ---- kernels ----------------------------------------------------------------

// Lane of the calling thread within its warp, for any block shape (a 2-D
// block's warps span several rows, so threadIdx.x alone does not give it).
APD void mul4(const float* m, float v0, float v1, float v2, float v3, float out[4]) {
#pragma unroll
  for (int r = 0; r < 4; ++r) out[r] = m[r] * v0 + m[4 + r] * v1 + m[8 + r] * v2 + m[12 + r] * v3;
}

// raygen.wgsl:21-39
__global__ void k_raygen(FrameBuffers fb, uint32_t W, uint32_t H, Mats mats) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  float ux = (((float)x + 0.5f) / (float)W) * 2.0f - 1.0f;
  float uy = (((float)y + 0.5f) / (float)H) * 2.0f - 1.0f;
  uy = -uy;
  float o[4], t[4], d[4];
  mul4(mats.inv_view, 0.0f, 0.0f, 0.0f, 1.0f, o);
  mul4(mats.inv_proj, ux, uy, 1.0f, 1.0f, t);
  float3 tn = normalize(f3(t[0], t[1], t[2]));
  mul4(mats.inv_view, tn.x, tn.y, tn.z, 0.0f, d);
  fb.rays[y * W + x] = make_float4(o[0], o[1], o[2], __uint_as_float(pack_oct30(f3(d[0], d[1], d[2]))));
}

// Persistent closest-hit kernel for the path-extension rays: each warp takes
// 32 consecutive queue entries per atomic.  Bounce 0 traces every pixel.
template <bool kCount>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_extend(DevScene s, FrameBuffers fb, Consts c) {
  const uint32_t count = c.bounce == 0 ? c.P : min(fb.counters[c.qin], c.P);
  const uint32_t* q = fb.queue[c.qin];
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&fb.counters[3], count);  // rays traced this frame
  const bool all = c.bounce == 0;
  persistent_trace<false, kCount>(
      s, count, &fb.counters[2],
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const uint32_t id = all ? i : q[i];
        const float4 r = fb.rays[id];
        d = ray_dir(r);
        o = ray_org(r) + d * 1e-4f;
        tmax = 1000.0f;
      },
      [&](uint32_t i, const Trav& t, const Visits& vc) {
        const uint32_t id = all ? i : q[i];
        fb.hits[id] = make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
        if (kCount) {
          atomicAdd(&fb.visits[3 * K_EXTEND + 0], 1ull);
          atomicAdd(&fb.visits[3 * K_EXTEND + 1], (unsigned long long)vc.nodes);
          atomicAdd(&fb.visits[3 * K_EXTEND + 2], (unsigned long long)vc.tris);
        }
      });
}

APD float2 velocity_of(const Mats& m, float3 p) {
  float cs[4], ps[4];
  mul4(m.view_proj, p.x, p.y, p.z, 1.0f, cs);
  mul4(m.prev_view_proj, p.x, p.y, p.z, 1.0f, ps);
  float px = (ps[0] / ps[3] + 1.0f) / 2.0f, py = 1.0f - (ps[1] / ps[3] + 1.0f) / 2.0f;
  float cx = (cs[0] / cs[3] + 1.0f) / 2.0f, cy = 1.0f - (cs[1] / cs[3] + 1.0f) / 2.0f;
  return make_float2(cx - px, cy - py);
}

// ---- secondary-ray queues -------------------------------------------------

// Appends one ray per requesting lane with one atomic per warp (ballot + popc).
APD void push_ray(const FrameBuffers& fb, int q, bool want, float3 o, float tmax, float3 d, uint32_t owner) {
  const unsigned active = __activemask();
  const unsigned b = __ballot_sync(active, want);
  if (!want) return;
  const int lane = (int)lane_id();
  const int leader = __ffs(b) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&fb.counters[kCounterQueueSize + q], (uint32_t)__popc(b));
  base = __shfl_sync(b, base, leader);
  uint32_t slot = base + __popc(b & ((1u << lane) - 1u));
  fb.rq_o[q][slot] = make_float4(o.x, o.y, o.z, tmax);
  fb.rq_d[q][slot] = make_float4(d.x, d.y, d.z, __uint_as_float(owner));
}

// Persistent traversal of one ray queue (per-lane refill).
template <bool kAny, bool kCount>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_queue(DevScene s, FrameBuffers fb, int q, uint32_t cap,
                                                                         uint4* hits, uint8_t* vis) {
  // a queue holds at most one ray per pixel
  const uint32_t count = min(fb.counters[kCounterQueueSize + q], cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&fb.counters[3], count);
  const float4* qo = fb.rq_o[q];
  const float4* qd = fb.rq_d[q];
  persistent_trace<kAny, kCount>(
      s, count, &fb.counters[kCounterQueueCursor + q],
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const float4 a = qo[i], b = qd[i];
        o = f3(a.x, a.y, a.z);
        d = f3(b.x, b.y, b.z);
        tmax = a.w;
      },
      [&](uint32_t i, const Trav& t, const Visits& vc) {
        const uint32_t owner = __float_as_uint(qd[i].w);
        if (kAny) {
          vis[owner] = t.hit.tri != kNoHit ? 0 : 1;
        } else {
          hits[owner] = make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
        }
        if (kCount) {
          const int k = kAny ? K_TRACE_ANY : K_TRACE_CLOSEST;
          atomicAdd(&fb.visits[3 * k + 0], 1ull);
          atomicAdd(&fb.visits[3 * k + 1], (unsigned long long)vc.nodes);
          atomicAdd(&fb.visits[3 * k + 2], (unsigned long long)vc.tris);
        }
      });
}

// Persistent any-hit traversal of two ray queues in one launch: rays [0, n0)
// of the combined range come from queue Q0, the rest from Q1, each result
// going to its own queue's visibility array.  One launch instead of two
// saves a launch and the second drain tail; every ray's result is the same.
template <int Q0, int Q1, bool kCount>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_pair(DevScene s, FrameBuffers fb, uint32_t cap) {
  const uint32_t n0 = min(fb.counters[kCounterQueueSize + Q0], cap);
  const uint32_t count = n0 + min(fb.counters[kCounterQueueSize + Q1], cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&fb.counters[3], count);
  const float4 *o0 = fb.rq_o[Q0], *d0 = fb.rq_d[Q0], *o1 = fb.rq_o[Q1], *d1 = fb.rq_d[Q1];
  uint8_t *v0 = fb.vis[Q0], *v1 = fb.vis[Q1];
  persistent_trace<true, kCount>(
      s, count, &fb.counters[kCounterQueueCursor + Q0],
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const bool first = i < n0;
        const uint32_t j = first ? i : i - n0;
        const float4 a = (first ? o0 : o1)[j], b = (first ? d0 : d1)[j];
        o = f3(a.x, a.y, a.z);
        d = f3(b.x, b.y, b.z);
        tmax = a.w;
      },
      [&](uint32_t i, const Trav& t, const Visits& vc) {
        const bool first = i < n0;
        const uint32_t j = first ? i : i - n0;
        const uint32_t owner = __float_as_uint((first ? d0 : d1)[j].w);
        (first ? v0 : v1)[owner] = t.hit.tri != kNoHit ? 0 : 1;
        if (kCount) {
          atomicAdd(&fb.visits[3 * K_TRACE_ANY + 0], 1ull);
          atomicAdd(&fb.visits[3 * K_TRACE_ANY + 1], (unsigned long long)vc.nodes);
          atomicAdd(&fb.visits[3 * K_TRACE_ANY + 2], (unsigned long long)vc.tris);
        }
      });
}

// Persistent closest-hit traversal of two ray queues in one launch, each hit
// going to its own queue's hit array (the closest-hit form of k_trace_pair).
template <int Q0, int Q1, bool kCount>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_pair_closest(DevScene s, FrameBuffers fb, uint32_t cap,
                                                                                uint4* h0, uint4* h1) {
  const uint32_t n0 = min(fb.counters[kCounterQueueSize + Q0], cap);
  const uint32_t count = n0 + min(fb.counters[kCounterQueueSize + Q1], cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&fb.counters[3], count);
  const float4 *o0 = fb.rq_o[Q0], *d0 = fb.rq_d[Q0], *o1 = fb.rq_o[Q1], *d1 = fb.rq_d[Q1];
  persistent_trace<false, kCount>(
      s, count, &fb.counters[kCounterQueueCursor + Q0],
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const bool first = i < n0;
        const uint32_t j = first ? i : i - n0;
        const float4 a = (first ? o0 : o1)[j], b = (first ? d0 : d1)[j];
        o = f3(a.x, a.y, a.z);
        d = f3(b.x, b.y, b.z);
        tmax = a.w;
      },
      [&](uint32_t i, const Trav& t, const Visits& vc) {
        const bool first = i < n0;
        const uint32_t j = first ? i : i - n0;
        const uint32_t owner = __float_as_uint((first ? d0 : d1)[j].w);
        (first ? h0 : h1)[owner] =
            make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
        if (kCount) {
          atomicAdd(&fb.visits[3 * K_TRACE_CLOSEST + 0], 1ull);
          atomicAdd(&fb.visits[3 * K_TRACE_CLOSEST + 1], (unsigned long long)vc.nodes);
          atomicAdd(&fb.visits[3 * K_TRACE_CLOSEST + 2], (unsigned long long)vc.tris);
        }
      });
}

// ---- batches of frames: shared traversal launches (serving) -----------------

// Block prologue of a batch traversal kernel: the frames' first ray indices
// (start[nj] = the batch's ray count) and their BVHs, in shared memory.
template <class CountOf>
APD uint32_t batch_setup(const JobTrace* jobs, int nj, CountOf count_of, uint32_t* s_start, BvhView* s_bvh) {
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int j = 0; j < nj; ++j) {
      s_start[j] = acc;
      acc += count_of(jobs[j]);
    }
    s_start[nj] = acc;
  }
  if ((int)threadIdx.x < nj) s_bvh[threadIdx.x] = BvhView{jobs[threadIdx.x].nodes, jobs[threadIdx.x].tris};
  __syncthreads();
  return s_start[nj];
}

// k_extend over a batch: each frame's path queue (all its pixels at bounce 0).
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_extend_batch(const JobTrace* jobs, int nj, uint32_t bounce,
                                                                          uint32_t qin) {
  __shared__ uint32_t s_start[kMaxBatch + 1];
  __shared__ BvhView s_bvh[kMaxBatch];
  const uint32_t count = batch_setup(
      jobs, nj, [&](const JobTrace& b) { return bounce == 0 ? b.P : min(b.counters[qin], b.P); }, s_start, s_bvh);
  if (blockIdx.x == 0 && (int)threadIdx.x < nj)
    atomicAdd(&jobs[threadIdx.x].counters[3], s_start[threadIdx.x + 1] - s_start[threadIdx.x]);
  persistent_trace_batch<false>(
      s_bvh, nj, s_start, count, &jobs[0].counters[2],
      [&](int j, uint32_t i, float3& o, float3& d, float& tmax) {
        const JobTrace& b = jobs[j];
        const uint32_t id = bounce == 0 ? i : b.queue[qin][i];
        const float4 r = b.rays[id];
        d = ray_dir(r);
        o = ray_org(r) + d * 1e-4f;
        tmax = 1000.0f;
      },
      [&](int j, uint32_t i, const Trav& t) {
        const JobTrace& b = jobs[j];
        const uint32_t id = bounce == 0 ? i : b.queue[qin][i];
        b.hits[id] = make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
      });
}

// k_trace_queue over a batch: queue q of every frame (closest hits of the
// candidate queues to hit_bsdf / hit_gi, visibility of the shadow queues).
template <bool kAny>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_queue_batch(const JobTrace* jobs, int nj, int q) {
  __shared__ uint32_t s_start[kMaxBatch + 1];
  __shared__ BvhView s_bvh[kMaxBatch];
  const uint32_t count = batch_setup(
      jobs, nj, [&](const JobTrace& b) { return min(b.counters[kCounterQueueSize + q], b.P); }, s_start, s_bvh);
  if (blockIdx.x == 0 && (int)threadIdx.x < nj)
    atomicAdd(&jobs[threadIdx.x].counters[3], s_start[threadIdx.x + 1] - s_start[threadIdx.x]);
  persistent_trace_batch<kAny>(
      s_bvh, nj, s_start, count, &jobs[0].counters[kCounterQueueCursor + q],
      [&](int j, uint32_t i, float3& o, float3& d, float& tmax) {
        const float4 a = jobs[j].rq_o[q][i], b = jobs[j].rq_d[q][i];
        o = f3(a.x, a.y, a.z);
        d = f3(b.x, b.y, b.z);
        tmax = a.w;
      },
      [&](int j, uint32_t i, const Trav& t) {
        const JobTrace& b = jobs[j];
        const uint32_t owner = __float_as_uint(b.rq_d[q][i].w);
        if (kAny) {
          b.vis[q][owner] = t.hit.tri != kNoHit ? 0 : 1;
        } else {
          (q == Q_BSDF_CAND ? b.hit_bsdf : b.hit_gi)[owner] =
              make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
        }
      });
}

// k_trace_pair over a batch: the any-hit queues Q0 and Q1 of every frame.
template <int Q0, int Q1>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_pair_batch(const JobTrace* jobs, int nj) {
  __shared__ uint32_t s_start[kMaxBatch + 1];
  __shared__ BvhView s_bvh[kMaxBatch];
  const uint32_t count = batch_setup(
      jobs, nj,
      [&](const JobTrace& b) {
        return min(b.counters[kCounterQueueSize + Q0], b.P) + min(b.counters[kCounterQueueSize + Q1], b.P);
      },
      s_start, s_bvh);
  if (blockIdx.x == 0 && (int)threadIdx.x < nj)
    atomicAdd(&jobs[threadIdx.x].counters[3], s_start[threadIdx.x + 1] - s_start[threadIdx.x]);
  persistent_trace_batch<true>(
      s_bvh, nj, s_start, count, &jobs[0].counters[kCounterQueueCursor + Q0],
      [&](int j, uint32_t i, float3& o, float3& d, float& tmax) {
        const JobTrace& b = jobs[j];
        const uint32_t n0 = min(b.counters[kCounterQueueSize + Q0], b.P);
        const bool first = i < n0;
        const float4 a = (first ? b.rq_o[Q0] : b.rq_o[Q1])[first ? i : i - n0];
        const float4 e = (first ? b.rq_d[Q0] : b.rq_d[Q1])[first ? i : i - n0];
        o = f3(a.x, a.y, a.z);
        d = f3(e.x, e.y, e.z);
        tmax = a.w;
      },
      [&](int j, uint32_t i, const Trav& t) {
        const JobTrace& b = jobs[j];
        const uint32_t n0 = min(b.counters[kCounterQueueSize + Q0], b.P);
        const bool first = i < n0;
        const uint32_t owner = __float_as_uint((first ? b.rq_d[Q0] : b.rq_d[Q1])[first ? i : i - n0].w);
        (first ? b.vis[Q0] : b.vis[Q1])[owner] = t.hit.tri != kNoHit ? 0 : 1;
      });
}

// ---- trace.wgsl:62-262 as four stages around the secondary rays -------------
//   A: hit attributes, emission, G-buffer, first NEE candidates (area + BSDF);
//      queues the BSDF candidate ray            (Nee::sample_ris, nee.wgsl:131-197)
//   B: finishes resampled NEE, queues its shadow ray; Russian roulette; samples
//      the GI direction and queues the GI candidate ray (inline_path_tracer.wgsl:258-283)
//   C: sets the DI contribution weight from the shadow ray; shades the GI
//      candidate's hit and queues its light-sample shadow ray (inline_path_tracer.wgsl:51-256)
//   D: finishes the GI reservoir
// The per-path RNG stream is consumed in exactly the reference's order.

constexpr uint32_t F_SHADED = 1u, F_BSDF_RAY = 2u;  // stage A -> B1
constexpr uint32_t F_B_SHADOW = 4u;                  // stage B1 -> B2
constexpr uint32_t F_RIS_SHADOW = 1u, F_GI_RAY = 2u, F_GI_SHADOW = 4u;  // B -> C -> D

APD uint32_t bounce_count(const FrameBuffers& fb, const Consts& c) { return c.bounce == 0 ? c.P : min(fb.counters[c.qin], c.P); }
APD uint32_t bounce_path(const FrameBuffers& fb, const Consts& c, uint32_t i) {
  return c.bounce == 0 ? i : fb.queue[c.qin][i];
}

// Area light candidate (nee.wgsl:136-155).
// Shared-memory copy of the light table (emissive_info) for the kernels that
// sample many light candidates per path; scenes with more emissive instances
// than fit read the table from global memory.
constexpr uint32_t kSmemLights = 512;
// All threads of the block must call this (it synchronises the block when it stages).
APD const uint4* stage_lights(const DevScene& s, uint4* sm) {
  if (s.num_emissive_instances > kSmemLights) return s.emissive_info;
  for (uint32_t i = threadIdx.x; i < s.num_emissive_instances; i += blockDim.x) sm[i] = s.emissive_info[i];
  __syncthreads();
  return sm;
}

// The full evaluation kept out of line in the RIS candidate loop, where only
// transmissive materials take it, so the loop's code stays small (the first
// candidate, evaluated without a context, keeps it inline); same arithmetic.
__device__ __noinline__ float3 disney_eval_outlined(const Bsdf& b, const Frame& fr, float3 wo, float3 wi, float* sp) {
  return disney_eval(b, fr, wo, wi, sp);
}

// `ctx` (the shading point's DisneyCtx, or null) saves the per-candidate
// evaluation its wo-only terms; transmissive materials evaluate in full.
APD void area_candidate(const DevScene& s, float3 hit, float3 wo, const Frame& fr, const Bsdf& b, uint32_t& rng,
                        LightSample* ls, float* pdf, LightEval* ev, float* phat, const uint4* lights,
                        const DisneyCtx* ctx = nullptr) {
  float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng), r3 = rnd(rng), r4 = rnd(rng);
  *ls = sample_uniform(s, r0, r1, r2, make_float2(r3, r4), pdf, lights);
  *ev = load_eval(s, *ls, hit, lights);
  *phat = 0.0f;
  float3 wi = normalize(ev->point - hit);
  float wdn = dot(wi, fr.n);
  // a light sample without emission (a sun of intensity 0) has target +0 whatever
  // the BSDF value: skip its evaluation (the oracle skips it too)
  const bool lit = ev->emission.x != 0.0f || ev->emission.y != 0.0f || ev->emission.z != 0.0f;
  if (wdn > 0.0f && *pdf > 0.0f && lit) {
    float sp = 0.0f;
    float3 refl = !ctx ? disney_eval(b, fr, wo, wi, &sp)
                       : (b.transmission <= 0.5f ? disney_eval_ctx(b, *ctx, fr, wo, wi, &sp)
                                                 : disney_eval_outlined(b, fr, wo, wi, &sp));
    if (sp > 0.0f) *phat = luma(refl * wdn * ev->emission);
  }
}

#ifndef AP_SHADE_A_MIN_BLOCKS
#define AP_SHADE_A_MIN_BLOCKS 10  // resident blocks per SM the kernel is register-capped for (measured)
#endif
__global__ void __launch_bounds__(kBlock, AP_SHADE_A_MIN_BLOCKS) k_shade_a(DevScene s, FrameBuffers fb, Consts c, Mats mats) {
  __shared__ uint4 s_lights[kSmemLights];
  const uint4* lights = stage_lights(s, s_lights);
  const uint32_t count = bounce_count(fb, c);
  const uint32_t cur = c.frame_idx & 1u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    float4 ray = fb.rays[id];
    float3 origin = ray_org(ray), direction = ray_dir(ray);
    uint4 pl = fb.payload[id];
    if (c.bounce == 0) {
      pl.x = pack_rgb9e5(f3s(1.0f));
      pl.y = pcg_hash(id ^ xor_shift(c.seed));
      pl.z = __float_as_uint(0.0f);
    }
    float3 acc = unpack_rgb9e5(fb.radiance[id]);
    float3 T = unpack_rgb9e5(pl.x);
    uint32_t rng = pl.y;
    float3 g_pos = f3s(0.0f), g_n = f3s(0.0f), g_alb = f3s(0.0f);
    float g_depth = 0.0f;
    float2 vel = make_float2(0.0f, 0.0f);
    uint4 hr = fb.hits[id];
    Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
    float t_out;
    uint32_t flags = 0;
    bool want_ray = false;
    float3 ray_o = f3s(0.0f), wi = f3s(0.0f);
    if (h.tri == kRcRetired) {  // ended in the radiance cache at this vertex
      t_out = -1.0f;
      fb.st_a[id] = make_uint4(0u, 0u, 0u, 0u);
    } else if (h.tri != kNoHit) {
      float depth_ws = 0.0f + h.t;
      const MaterialDev* m;
      Surface sf = surface(s, h, origin, direction, &m);
      float3 emission = ld3(m->emission);
      if (c.bounce == 0) acc = acc + T * emission;
      float3 wo = -direction;
      Bsdf b = load_bsdf(m);
      if (c.bounce == 0) {
        g_pos = sf.hit_point;
        g_depth = depth_ws;
        g_n = sf.n;
        g_alb = ld3(m->color) + emission;
        vel = velocity_of(mats, sf.hit_point);
      }
      fb.ctx[id] = make_uint4(sf.material_idx, pack_rgb9e5(T), pack_oct30(sf.n), pack_oct30(sf.frame.cc_t2w.c2));
      float area_pdf = 0.0f, area_phat = 0.0f, bsdf_pdf = 0.0f;
      LightSample area_s{make_float2(0.0f, 0.0f), 0u, 0u};
      if (c.cfg.di_area_samples > 0) {
        LightEval ev;
        area_candidate(s, sf.hit_point, wo, sf.frame, b, rng, &area_s, &area_pdf, &ev, &area_phat, lights);
      }
      float3 contribution = f3s(0.0f);
      if (c.cfg.di_bsdf_samples > 0) {
        float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng);
        float3 refl = disney_sample(b, sf.frame, wo, h.t, sf.back_face, r0, r1, r2, &wi, &bsdf_pdf);
        float wdn = dm::fabs_(dot(wi, sf.n));
        contribution = wdn * refl;
        if (dot(contribution, contribution) > 0.0f) {
          want_ray = true;
          ray_o = sf.hit_point + sf.n * 1e-4f;
        }
      }
      flags = F_SHADED | (want_ray ? F_BSDF_RAY : 0u);
      fb.st_a[id] = make_uint4(__float_as_uint(area_pdf), __float_as_uint(area_phat), __float_as_uint(bsdf_pdf), flags);
      fb.st_b[id] = make_uint4(__float_as_uint(area_s.uv.x), __float_as_uint(area_s.uv.y), area_s.inst, area_s.tri);
      fb.st_c[id] = make_uint4(__float_as_uint(contribution.x), __float_as_uint(contribution.y),
                               __float_as_uint(contribution.z), 0u);
      fb.st_d[id] = make_uint4(__float_as_uint(wi.x), __float_as_uint(wi.y), __float_as_uint(wi.z), 0u);
      t_out = depth_ws;
    } else {
      g_alb = f3s(1.0f);
      acc = acc + T * sky_radiance(s, direction, true);
      t_out = -1.0f;
      fb.st_a[id] = make_uint4(0u, 0u, 0u, 0u);
    }
    push_ray(fb, Q_BSDF_CAND, want_ray, ray_o, 1000.0f, wi, id);
    fb.radiance[id] = pack_rgb9e5(acc);
    fb.payload[id] = make_uint4(pack_rgb9e5(T), rng, __float_as_uint(t_out), 0u);
    if (c.bounce == 0) {
      fb.gb_a[cur][id] = make_uint4(__float_as_uint(g_pos.x), __float_as_uint(g_pos.y), __float_as_uint(g_pos.z),
                                    __float_as_uint(g_depth));
      fb.gb_b[cur][id] = make_uint4(pack_oct30(g_n), pack_rgb9e5(g_alb), __float_as_uint(vel.x), __float_as_uint(vel.y));
    }
  }
}

// Stage B1: resampled importance sampling of the direct light (Nee::sample_ris,
// nee.wgsl:122-237) and its shadow ray.
#ifndef AP_SHADE_B_MIN_BLOCKS
#define AP_SHADE_B_MIN_BLOCKS 8  // resident blocks per SM the RIS stage is register-capped for (measured)
#endif
__global__ void __launch_bounds__(kBlock, AP_SHADE_B_MIN_BLOCKS) k_shade_b(DevScene s, FrameBuffers fb, Consts c) {
  __shared__ uint4 s_lights[kSmemLights];
  const uint4* lights = stage_lights(s, s_lights);
  const uint32_t count = bounce_count(fb, c);
  const uint32_t NA = c.cfg.di_area_samples, NB = c.cfg.di_bsdf_samples;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    uint4 sa = fb.st_a[id];
    bool active = (sa.w & F_SHADED) != 0;
    bool want_shadow = false;
    float3 sh_o = f3s(0.0f), sh_d = f3s(0.0f);
    float sh_t = 0.0f;
    if (active) {
      uint4 pl = fb.payload[id];
      float4 ray = fb.rays[id];
      float3 origin = ray_org(ray), direction = ray_dir(ray);
      float3 T = unpack_rgb9e5(pl.x);
      uint32_t rng = pl.y;
      uint4 hr = fb.hits[id];
      Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
      const MaterialDev* m;
      Surface sf = surface(s, h, origin, direction, &m);
      Bsdf b = load_bsdf(m);
      float3 wo = -direction;
      float3 hit = sf.hit_point;
      float area_pdf = __uint_as_float(sa.x), area_phat = __uint_as_float(sa.y), bsdf_pdf = __uint_as_float(sa.z);
      uint4 sb = fb.st_b[id];
      LightSample area_s{make_float2(__uint_as_float(sb.x), __uint_as_float(sb.y)), sb.z, sb.w};
      LightEval area_e{f3s(0.0f), f3s(0.0f)};
      if (NA > 0) area_e = load_eval(s, area_s, hit, lights);
      uint4 sc = fb.st_c[id];
      float3 contribution = f3(__uint_as_float(sc.x), __uint_as_float(sc.y), __uint_as_float(sc.z));
      uint4 sd4 = fb.st_d[id];
      float3 bwi = f3(__uint_as_float(sd4.x), __uint_as_float(sd4.y), __uint_as_float(sd4.z));
      LightSample bsdf_s = ls_empty();
      LightEval bsdf_e{f3s(0.0f), f3s(0.0f)};
      float bsdf_phat = 0.0f;
      if (sa.w & F_BSDF_RAY) {
        uint4 h1 = fb.hit_bsdf[id];
        if (h1.w != kNoHit) {
          const InstanceDev in = s.instances[s.tri_instance[h1.w]];
          if (in.emissive_idx != kU32Max)
            bsdf_s = LightSample{make_float2(__uint_as_float(h1.y), __uint_as_float(h1.z)), in.emissive_idx,
                                 h1.w - in.first_global_tri};
        } else {
          bsdf_s = LightSample{inverse_direction_to_sun(s.sun, bwi), kU32Max - 1, 0u};
        }
        if (!ls_is_empty(bsdf_s)) {
          bsdf_e = load_eval(s, bsdf_s, hit, lights);
          bsdf_phat = luma(contribution * bsdf_e.emission);
        }
      }
      DiRes res = di_new();
      LightEval sel{f3s(0.0f), f3s(0.0f)};
      uint32_t n_iter = NA > NB ? NA : NB;
      const DisneyCtx dctx = disney_ctx(b, sf.frame, wo);
      for (uint32_t k = 0; k < n_iter; ++k) {
        float apdf = 0.0f, aphat = 0.0f, bpdf = 0.0f;
        LightSample as{make_float2(0.0f, 0.0f), 0u, 0u};
        LightEval ae{f3s(0.0f), f3s(0.0f)};
        if (k == 0) {
          apdf = area_pdf; aphat = area_phat; as = area_s; ae = area_e; bpdf = bsdf_pdf;
        } else if (k < NA) {
          area_candidate(s, hit, wo, sf.frame, b, rng, &as, &apdf, &ae, &aphat, lights, &dctx);
        }
        if (k < NA) {
          float aw = 0.0f;
          if (apdf > 0.0f) {
            float mis = apdf / ((float)NA * apdf + (float)NB * bpdf);
            aw = mis * aphat * (1.0f / dm::fmax(apdf, 1e-8f));
          }
          if (di_update(res, aw, rng, as, aphat)) sel = ae;
        }
        if (k < NB) {
          float bw = 0.0f;
          if (bpdf > 0.0f) {
            float mis = bpdf / ((float)NB * bpdf + (float)NA * apdf);
            bw = mis * bsdf_phat * (1.0f / dm::fmax(bpdf, 1e-8f));
          }
          if (di_update(res, bw, rng, bsdf_s, bsdf_phat)) sel = bsdf_e;
        }
      }
      if (res.phat > 1e-6f) {
        sh_d = normalize(sel.point - hit);
        float dd = dist(sel.point, hit);
        sh_o = hit + sf.n * 1e-4f;
        sh_t = dd - 1e-4f * 2.0f;
        want_shadow = true;
      }
      fb.di_a[id] = di_pack_a(res);
      fb.di_b[id] = di_pack_b(res);
      fb.payload[id] = make_uint4(pl.x, rng, pl.z, pl.w);
      fb.st_a[id] = make_uint4(0u, 0u, 0u, F_SHADED | (want_shadow ? F_B_SHADOW : 0u));
    }
    push_ray(fb, Q_RIS_SHADOW, want_shadow, sh_o, sh_t, sh_d, id);
  }
}

// Stage B2: Russian roulette (trace.wgsl:220-230) and the BSDF-sampled GI
// candidate direction (InlinePathTracer::sample_ris, inline_path_tracer.wgsl:258-296),
// continuing the path's RNG stream after stage B1.
#ifndef AP_SHADE_B2_MIN_BLOCKS
#define AP_SHADE_B2_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(kBlock, AP_SHADE_B2_MIN_BLOCKS) k_shade_b2(DevScene s, FrameBuffers fb, Consts c) {
  const uint32_t count = bounce_count(fb, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    uint4 sa = fb.st_a[id];
    bool active = (sa.w & F_SHADED) != 0;
    bool want_gi = false;
    float3 gi_o = f3s(0.0f), wi = f3s(0.0f);
    if (active) {
      uint4 pl = fb.payload[id];
      float4 ray = fb.rays[id];
      float3 origin = ray_org(ray), direction = ray_dir(ray);
      float3 T = unpack_rgb9e5(pl.x);
      uint32_t rng = pl.y;
      uint4 hr = fb.hits[id];
      Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
      const MaterialDev* m;
      Surface sf = surface(s, h, origin, direction, &m);
      Bsdf b = load_bsdf(m);
      float3 wo = -direction;
      float3 hit = sf.hit_point;
      float t_out = __uint_as_float(pl.z);
      float gi_pdf = 0.0f;
      uint32_t phat_rng = 0;
      float3 tr = f3s(0.0f);
      if (c.bounce + 1 < c.cfg.max_bounces) {
        bool killed = false;
        if (c.bounce > 1) {
          float rr = dm::fmax(T.x, dm::fmax(T.y, T.z));
          if (rr < rnd(rng)) {
            t_out = -1.0f;
            killed = true;
          } else {
            T = T * (1.0f / rr);
          }
        }
        if (!killed) {
          float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng);
          float3 refl = disney_sample(b, sf.frame, wo, h.t, sf.back_face, r0, r1, r2, &wi, &gi_pdf);
          if (gi_pdf > 1e-6f) {
            float cos_in = dm::fabs_(dot(wi, sf.n));
            float3 local = cos_in * refl;
            tr = T * local;
            phat_rng = rng;
            gi_o = hit + wi * 1e-4f;
            want_gi = true;
          } else {
            GiRes z = gi_new();
            fb.gi_a[id] = gi_pack_a(z);
            fb.gi_b[id] = gi_pack_b(z);
          }
        }
      }
      uint32_t flags = ((sa.w & F_B_SHADOW) ? F_RIS_SHADOW : 0u) | (want_gi ? F_GI_RAY : 0u);
      fb.payload[id] = make_uint4(pack_rgb9e5(T), rng, __float_as_uint(t_out), 0u);
      fb.st_a[id] = make_uint4(__float_as_uint(gi_pdf), phat_rng, 0u, flags);
      fb.st_c[id] = make_uint4(__float_as_uint(tr.x), __float_as_uint(tr.y), __float_as_uint(tr.z), 0u);
      fb.st_d[id] = make_uint4(__float_as_uint(wi.x), __float_as_uint(wi.y), __float_as_uint(wi.z), 0u);
    }
    push_ray(fb, Q_GI_CAND, want_gi, gi_o, 1000.0f - 1e-4f * 2.0f, wi, id);
  }
}

APD void finish_gi(const FrameBuffers& fb, uint32_t id, float3 contribution, float pdf, float3 point, uint32_t phat_rng,
                   uint32_t& rng) {
  GiRes res = gi_new();
  float phat = luma(contribution);
  gi_update(res, phat / pdf, rng, point, phat, phat_rng);
  if (res.phat > 0.0f && res.M * res.wsum > 0.0f) res.W = (1.0f / res.phat) * (1.0f / res.M * res.wsum);
  fb.gi_a[id] = gi_pack_a(res);
  fb.gi_b[id] = gi_pack_b(res);
}

#ifndef AP_SHADE_C_MIN_BLOCKS
#define AP_SHADE_C_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(kBlock, AP_SHADE_C_MIN_BLOCKS) k_shade_c(DevScene s, FrameBuffers fb, Consts c) {
  const uint32_t count = bounce_count(fb, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    uint4 sa = fb.st_a[id];
    bool want = false;
    float3 so = f3s(0.0f), sd = f3s(0.0f);
    float st = 0.0f;
    // the RIS shadow ray is traced after this stage; k_shade_d applies it
    const uint32_t ris = sa.w & F_RIS_SHADOW;
    if (sa.w & F_GI_RAY) {
      uint4 pl = fb.payload[id];
      uint32_t rng = pl.y;
      float4 ray = fb.rays[id];
      float3 hit = ray_org(ray) + ray_dir(ray) * __uint_as_float(pl.z);
      uint4 sc = fb.st_c[id], sdd = fb.st_d[id];
      float3 tr = f3(__uint_as_float(sc.x), __uint_as_float(sc.y), __uint_as_float(sc.z));
      float3 wi = f3(__uint_as_float(sdd.x), __uint_as_float(sdd.y), __uint_as_float(sdd.z));
      float gi_pdf = __uint_as_float(sa.x);
      uint32_t phat_rng = sa.y;
      uint4 hr = fb.hit_gi[id];
      float3 acc = f3s(0.0f), point;
      if (hr.w != kNoHit) {
        Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
        const MaterialDev* m;
        Surface sf = surface(s, h, hit, wi, &m);
        Bsdf b = load_bsdf(m);
        float pdf = 0.0f;
        float r0 = rnd(rng), r1 = rnd(rng), r2 = rnd(rng), r3 = rnd(rng), r4 = rnd(rng);
        LightSample ls = sample_uniform(s, r0, r1, r2, make_float2(r3, r4), &pdf);
        float W = 1.0f / pdf;
        if (W > 0.0f) {
          LightEval ev = load_eval(s, ls, sf.hit_point);
          float3 sdir = normalize(ev.point - sf.hit_point);
          float sdist = dist(ev.point, sf.hit_point);
          float ndl = dot(sdir, sf.n);
          if (ndl > 0.0f) {
            float sp = 0.0f;
            float3 refl = disney_eval(b, sf.frame, -wi, sdir, &sp);
            acc = tr * refl * ev.emission * ndl * W;  // added when the shadow ray is unoccluded
            so = sf.hit_point + sf.n * 1e-4f;
            sd = sdir;
            st = sdist - 1e-4f * 2.0f;
            // a zero contribution (a light sample without emission) leaves +0 whether or not
            // the ray is occluded (k_shade_d adds it to +0): finish here without the ray
            want = acc.x != 0.0f || acc.y != 0.0f || acc.z != 0.0f;
            if (!want) acc = f3s(0.0f);
          }
        }
        point = sf.hit_point;
      } else {
        point = hit + wi * 1000.0f;
        acc = acc + tr * sky_radiance(s, wi, true);
      }
      if (want) {
        fb.st_a[id] = make_uint4(sa.x, sa.y, 0u, F_GI_SHADOW | ris);
        fb.st_b[id] = make_uint4(__float_as_uint(point.x), __float_as_uint(point.y), __float_as_uint(point.z), 0u);
        fb.st_c[id] = make_uint4(__float_as_uint(acc.x), __float_as_uint(acc.y), __float_as_uint(acc.z), 0u);
      } else {
        finish_gi(fb, id, acc, gi_pdf, point, phat_rng, rng);
        fb.st_a[id] = make_uint4(0u, 0u, 0u, ris);
      }
      pl.y = rng;
      fb.payload[id] = pl;
    } else if (sa.w != 0u) {
      fb.st_a[id] = make_uint4(0u, 0u, 0u, ris);
    }
    push_ray(fb, Q_GI_SHADOW, want, so, st, sd, id);
  }
}

__global__ void __launch_bounds__(kBlock) k_shade_d(FrameBuffers fb, Consts c) {
  const uint32_t count = bounce_count(fb, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    uint4 sa = fb.st_a[id];
    if (sa.w & F_RIS_SHADOW) {
      // the resampled light sample is visible: its contribution weight (nee.wgsl)
      if (fb.vis[Q_RIS_SHADOW][id]) {
        uint4 da = fb.di_a[id];
        float W = (1.0f / __uint_as_float(da.w)) * __uint_as_float(da.z);
        fb.di_a[id] = make_uint4(da.x, __float_as_uint(W), da.z, da.w);
      }
      sa.w &= ~F_RIS_SHADOW;
      fb.st_a[id] = sa;
    }
    if (!(sa.w & F_GI_SHADOW)) continue;
    uint4 pl = fb.payload[id];
    uint32_t rng = pl.y;
    uint4 sb = fb.st_b[id], sc = fb.st_c[id];
    float3 point = f3(__uint_as_float(sb.x), __uint_as_float(sb.y), __uint_as_float(sb.z));
    float3 acc = f3s(0.0f);
    if (fb.vis[Q_GI_SHADOW][id]) acc = acc + f3(__uint_as_float(sc.x), __uint_as_float(sc.y), __uint_as_float(sc.z));
    finish_gi(fb, id, acc, __uint_as_float(sa.x), point, sa.y, rng);
    pl.y = rng;
    fb.payload[id] = pl;
  }
}

// apply_di.wgsl:48-111 in two stages around its shadow ray.
constexpr uint32_t F_DI_REPACK = 1u, F_DI_SHADOW = 2u;
#ifndef AP_APPLY_MIN_BLOCKS
#define AP_APPLY_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(kBlock, AP_APPLY_MIN_BLOCKS) k_apply_di_a(DevScene s, FrameBuffers fb, Consts c) {
  const uint32_t count = bounce_count(fb, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    uint4 pl = fb.payload[id];
    float pt = __uint_as_float(pl.z);
    uint32_t flags = 0;
    bool want = false;
    float3 so = f3s(0.0f), sd = f3s(0.0f);
    float st = 0.0f;
    if (pt >= 0.0f) {
      DiRes dr = di_unpack(fb.di_a[id], fb.di_b[id]);
      if (dr.W != 0.0f) {
        flags = F_DI_REPACK;
        float4 ray = fb.rays[id];
        float3 origin = ray_org(ray), direction = ray_dir(ray);
        uint4 cx = fb.ctx[id];
        float3 T = unpack_rgb9e5(cx.y);
        Bsdf b = load_bsdf(s.materials + cx.x);
        float3 hit = origin + direction * pt;
        Frame fr = ctx_frame(cx);
        LightEval ev = load_eval(s, dr.s, hit);
        float3 sdir = normalize(ev.point - hit);
        float sdist = dist(ev.point, hit);
        float ndl = dot(sdir, fr.n);
        if (ndl > 0.0f) {
          float sp = 0.0f;
          float3 refl = disney_eval(b, fr, -direction, sdir, &sp);
          float3 contribution = T * refl * ev.emission * ndl * dr.W;
          fb.st_c[id] = make_uint4(__float_as_uint(contribution.x), __float_as_uint(contribution.y),
                                   __float_as_uint(contribution.z), 0u);
          so = hit + fr.n * 1e-4f;
          sd = sdir;
          st = sdist - 1e-4f * 2.0f;
          want = true;
          flags |= F_DI_SHADOW;
        }
      }
    }
    fb.st_a[id] = make_uint4(0u, 0u, 0u, flags);
    push_ray(fb, Q_DI_SHADOW, want, so, st, sd, id);
  }
}

__global__ void __launch_bounds__(kBlock) k_apply_di_b(FrameBuffers fb, Consts c) {
  const uint32_t count = bounce_count(fb, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t id = bounce_path(fb, c, i);
    uint32_t flags = fb.st_a[id].w;
    if (!(flags & F_DI_REPACK)) continue;
    float3 acc = unpack_rgb9e5(fb.radiance[id]);
    if ((flags & F_DI_SHADOW) && fb.vis[Q_DI_SHADOW][id]) {
      uint4 sc = fb.st_c[id];
      acc = acc + f3(__uint_as_float(sc.x), __uint_as_float(sc.y), __uint_as_float(sc.z));
    }
    fb.radiance[id] = pack_rgb9e5(acc);
  }
}

// apply_gi.wgsl:44-99, plus re-queueing of the live paths (warp ballot, one
// atomic per warp) for the next bounce.
__global__ void __launch_bounds__(kBlock, AP_APPLY_MIN_BLOCKS) k_apply_gi(DevScene s, FrameBuffers fb, Consts c) {
  const uint32_t count = c.bounce == 0 ? c.P : min(fb.counters[c.qin], c.P);
  const uint32_t* q = fb.queue[c.qin];
  uint32_t* qo = fb.queue[c.qout];
  const uint32_t lane = lane_id();
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t start = blockIdx.x * blockDim.x + threadIdx.x;
  // every lane of a warp runs the same number of iterations (ballot below)
  uint32_t iters = (count + stride - 1) / stride;
  for (uint32_t it = 0; it < iters; ++it) {
    uint32_t i = start + it * stride;
    bool alive = false;
    uint32_t id = 0;
    if (i < count) {
      id = c.bounce == 0 ? i : q[i];
      uint4 pl = fb.payload[id];
      float pt = __uint_as_float(pl.z);
      if (pt >= 0.0f) {
        float4 ray = fb.rays[id];
        float3 origin = ray_org(ray), direction = ray_dir(ray);
        float3 hit = origin + direction * pt;
        GiRes gr = gi_unpack(fb.gi_a[id], fb.gi_b[id]);
        if (gr.W > 0.0f) {
          uint4 cx = fb.ctx[id];
          float3 T = unpack_rgb9e5(pl.x);
          Bsdf b = load_bsdf(s.materials + cx.x);
          Frame fr = ctx_frame(cx);
          float3 wi = normalize(gr.point - hit);
          float sp = 0.0f;
          float3 refl = disney_eval(b, fr, -direction, wi, &sp);
          float cos_in = dm::fabs_(dot(fr.n, wi));
          T = T * (refl * cos_in * gr.W);
          pl.x = pack_rgb9e5(T);
          fb.rays[id] = make_float4(hit.x, hit.y, hit.z, __uint_as_float(pack_oct30(wi)));
          alive = true;
        } else {
          pl.z = __float_as_uint(-1.0f);
        }
        fb.payload[id] = pl;
      }
    }
    uint32_t ballot = __ballot_sync(0xffffffffu, alive);
    if (ballot) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&fb.counters[c.qout], (uint32_t)__popc(ballot));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (alive) qo[base + __popc(ballot & ((1u << lane) - 1u))] = id;
    }
  }
}

// ---- ReSTIR ---------------------------------------------------------------

struct GT {
  float3 pos;
  float depth;
  float3 n;
  float3 albedo;
};
APD GT gt_load(const uint4* a, const uint4* b, uint32_t id) {
  uint4 x = a[id], y = b[id];
  return GT{f3(__uint_as_float(x.x), __uint_as_float(x.y), __uint_as_float(x.z)), __uint_as_float(x.w),
            unpack_oct30(y.x), unpack_rgb9e5(y.y)};
}
// GBuffer::sample_prev_gbuffer (gbuffer_bindings.wgsl:20-50)
APD GT sample_prev_gbuffer(const uint4* a, const uint4* b, uint32_t W, uint32_t H, float2 pos) {
  uint32_t ix = dm::f2u(floorf(pos.x)), iy = dm::f2u(floorf(pos.y));
  float fx = dm::fract(pos.x), fy = dm::fract(pos.y);
  uint32_t x1 = min(ix + 1, W - 1), y1 = min(iy + 1, H - 1);
  GT t00 = gt_load(a, b, iy * W + ix), t10 = gt_load(a, b, iy * W + x1);
  GT t01 = gt_load(a, b, y1 * W + ix), t11 = gt_load(a, b, y1 * W + x1);
  GT r;
  r.pos = mix3(mix3(t00.pos, t10.pos, fx), mix3(t01.pos, t11.pos, fx), fy);
  r.depth = mixf(mixf(t00.depth, t10.depth, fx), mixf(t01.depth, t11.depth, fx), fy);
  r.n = normalize(mix3(mix3(t00.n, t10.n, fx), mix3(t01.n, t11.n, fx), fy));
  r.albedo = mix3(mix3(t00.albedo, t10.albedo, fx), mix3(t01.albedo, t11.albedo, fx), fy);
  return r;
}
APD bool history_valid(const GT& cur, const GT& prev) {
  bool ds = dm::fabs_(cur.depth - prev.depth) <= 0.1f * prev.depth;
  bool ns = dot(cur.n, prev.n) > 0.906f;
  return ds && ns;
}
APD bool prev_point(const FrameBuffers& fb, uint32_t cur, uint32_t x, uint32_t y, uint32_t W, uint32_t H, float2* out) {
  uint4 gb = fb.gb_b[cur][y * W + x];
  float vx = __uint_as_float(gb.z), vy = __uint_as_float(gb.w);
  float px = (float)x - ((float)W * vx), py = (float)y - ((float)H * vy);
  *out = make_float2(px, py);
  return px >= 0.0f && py >= 0.0f && px <= (float)(W - 1) && py <= (float)(H - 1);
}
APD uint32_t stochastic_prev_id(float2 p, float r0, float r1, uint32_t W, uint32_t H) {
  uint32_t px = dm::f2u(floorf(p.x + r0)), py = dm::f2u(floorf(p.y + r1));
  unsigned long long id = (unsigned long long)py * W + px;
  unsigned long long last = (unsigned long long)W * H - 1ull;
  return (uint32_t)(id < last ? id : last);
}
APD DiRes di_combine(const DiRes& r1, const DiRes& r2, uint32_t& rng) {
  DiRes c = di_new();
  di_update(c, r1.phat * r1.W * r1.M, rng, r1.s, r1.phat);
  di_update(c, r2.phat * r2.W * r2.M, rng, r2.s, r2.phat);
  c.M = r1.M + r2.M;
  if (c.phat > 1e-6f && c.M * c.wsum > 1e-6f) c.W = (1.0f / c.phat) * (1.0f / c.M * c.wsum);
  return c;
}
APD GiRes gi_combine(const GiRes& r1, const GiRes& r2, uint32_t& rng) {
  GiRes c = gi_new();
  gi_update(c, r1.phat * r1.W * r1.M, rng, r1.point, r1.phat, r1.phat_rng);
  gi_update(c, r2.phat * r2.W * r2.M, rng, r2.point, r2.phat, r2.phat_rng);
  c.M = r1.M + r2.M;
  if (c.phat > 0.0f && c.M * c.wsum > 0.0f) c.W = (1.0f / c.phat) * (1.0f / c.M * c.wsum);
  return c;
}



// LightSample::phat split at its visibility test: the unshadowed target and the
// shadow ray (helpers/trace.wgsl:7-18 offsets) that decides whether it counts.
struct PhatSplit {
  float value;
  bool ray;
  float3 o, d;
  float tmax;
};
APD PhatSplit ls_phat_split(const DevScene& s, const LightSample& l, const uint4 c, float3 hit, float3 wo) {
  LightEval ev = load_eval(s, l, hit);
  Bsdf b = load_bsdf(s.materials + c.x);
  Frame fr = ctx_frame(c);
  float3 wi = normalize(ev.point - hit);
  float wdn = dot(wi, fr.n);
  PhatSplit r;
  r.value = 0.0f;
  r.ray = false;
  r.o = f3s(0.0f);
  r.d = f3s(0.0f);
  r.tmax = 0.0f;
  if (wdn > 0.0f) {
    float sp = 0.0f;
    float3 refl = disney_eval(b, fr, wo, wi, &sp);
    r.value = luma(refl * wdn * ev.emission);
    r.ray = __float_as_uint(r.value) != 0u;  // a +0 target is +0 whether or not the ray is occluded
    r.o = hit + fr.n * 1e-4f;
    r.d = wi;
    r.tmax = dist(ev.point, hit) - 1e-4f * 2.0f;
  }
  return r;
}

// ---- temporal passes as wavefront stages -------------------------------------
//
// The temporal resampling passes (restir_di_temporal.wgsl:68-176,
// restir_gi_temporal.wgsl:67-116), split at their rays so that the rays go
// through the persistent traversal queues.  Loop state in
// the stage buffers: st_a {pixel rng, previous-frame pixel, flags, -},
// st_c {throughput or light contribution}, st_b {the target's value (DI)}.
enum : uint32_t {
  TP_HIST = 1u,    // history reprojected and valid: combine with the previous reservoir
  TP_RAY = 2u,     // the target's visibility ray was queued (DI)
  TP_SHADOW = 4u,  // GI re-trace: the NEE shadow ray was queued
  TP_DONE = 8u,    // GI re-trace: radiance known without a shadow ray (sky)
};

// DI temporal, stage 1 (restir_di_temporal.wgsl:68-158): reprojection, the
// previous reservoir and its target here, whose visibility ray is queued.
#ifndef AP_TEMPORAL_MIN_BLOCKS
#define AP_TEMPORAL_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(256, AP_TEMPORAL_MIN_BLOCKS) k_dt_a(DevScene s, FrameBuffers fb, Consts c, const uint4* prev_a,
                                              const uint4* prev_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  float pt = __uint_as_float(pl.z);
  if (pt < 0.0f) return;
  const uint32_t cur = c.frame_idx & 1u;
  uint32_t rng = pl.y;
  uint32_t flags = 0, pid = 0;
  PhatSplit ph;
  ph.ray = false;
  ph.value = 0.0f;
  float2 pp;
  if (prev_point(fb, cur, x, y, c.W, c.H, &pp)) {
    GT g = gt_load(fb.gb_a[cur], fb.gb_b[cur], id);
    GT pg = sample_prev_gbuffer(fb.gb_a[cur ^ 1u], fb.gb_b[cur ^ 1u], c.W, c.H, pp);
    if (history_valid(g, pg)) {
      float r0 = rnd(rng), r1 = rnd(rng);
      pid = stochastic_prev_id(pp, r0, r1, c.W, c.H);
      const DiRes pr = di_unpack(prev_a[pid], prev_b[pid]);
      float4 ray = fb.rays[id];
      float3 direction = ray_dir(ray);
      float3 hit = ray_org(ray) + direction * pt;
      ph = ls_phat_split(s, pr.s, fb.ctx[id], hit, -direction);
      flags = TP_HIST;
      if (c.cfg.di_unbiased) {
        if (ph.ray) flags |= TP_RAY;
      } else {
        ph.ray = false;
      }
    }
  }
  fb.st_a[id] = make_uint4(rng, pid, flags, __float_as_uint(ph.value));
  push_ray(fb, Q_DI_SHADOW, ph.ray, ph.o, ph.tmax, ph.d, id);
}

// DI temporal, stage 2 (restir_di_temporal.wgsl:159-176): M cap and combine.
__global__ void __launch_bounds__(256) k_dt_b(FrameBuffers fb, Consts c, const uint4* in_a, const uint4* in_b,
                                              uint4* out_a, uint4* out_b, const uint4* prev_a, const uint4* prev_b,
                                              uint4* pout_a, uint4* pout_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  if (__uint_as_float(pl.z) < 0.0f) return;
  const uint4 sa = fb.st_a[id];
  uint32_t rng = sa.x;
  DiRes r = di_unpack(in_a[id], in_b[id]);
  if (sa.z & TP_HIST) {
    DiRes pr = di_unpack(prev_a[sa.y], prev_b[sa.y]);
    pr.M = dm::fmin(pr.M, c.cfg.di_temporal_m_factor * r.M);
    if (!c.cfg.di_unbiased) pr.phat = __uint_as_float(sa.w);  // target without visibility
    else pr.phat = ((sa.z & TP_RAY) && fb.vis[Q_DI_SHADOW][id]) ? __uint_as_float(sa.w) : 0.0f;
    r = di_combine(r, pr, rng);
  }
  out_a[id] = di_pack_a(r);
  out_b[id] = di_pack_b(r);
  if (c.cfg.di_spatial_passes == 0) {
    pout_a[id] = di_pack_a(r);
    pout_b[id] = di_pack_b(r);
  }
  pl.y = rng;
  fb.payload[id] = pl;
}

// GI temporal, stage 1 (restir_gi_temporal.wgsl:67-96): reprojection, the
// previous reservoir, and the first ray of its target's re-trace
// (GiReservoir::phat, inline_path_tracer.wgsl:299-331).
__global__ void __launch_bounds__(256, AP_TEMPORAL_MIN_BLOCKS) k_gt_a(DevScene s, FrameBuffers fb, Consts c, const uint4* prev_a,
                                              const uint4* prev_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  float pt = __uint_as_float(pl.z);
  if (pt < 0.0f) return;
  const uint32_t cur = c.frame_idx & 1u;
  uint32_t rng = pl.y;
  uint32_t flags = 0, pid = 0;
  bool want = false;
  float3 o = f3s(0.0f), wi = f3s(0.0f), tr = f3s(0.0f);
  float2 pp;
  if (prev_point(fb, cur, x, y, c.W, c.H, &pp)) {
    float r0 = rnd(rng), r1 = rnd(rng);
    pid = stochastic_prev_id(pp, r0, r1, c.W, c.H);
    GT g = gt_load(fb.gb_a[cur], fb.gb_b[cur], id);
    GT pg = sample_prev_gbuffer(fb.gb_a[cur ^ 1u], fb.gb_b[cur ^ 1u], c.W, c.H, pp);
    if (history_valid(g, pg)) {
      const GiRes pr = gi_unpack(prev_a[pid], prev_b[pid]);
      float4 ray = fb.rays[id];
      float3 direction = ray_dir(ray);
      float3 hit = ray_org(ray) + direction * pt;
      const uint4 cx = fb.ctx[id];
      Bsdf b = load_bsdf(s.materials + cx.x);
      Frame fr = ctx_frame(cx);
      wi = normalize(pr.point - hit);
      float sp = 0.0f;
      float3 refl = disney_eval(b, fr, -direction, wi, &sp);
      float cos_in = dm::fabs_(dot(wi, fr.n));
      float3 local = cos_in * refl;
      float3 gi_origin = hit + wi * 0.0001f;
      tr = unpack_rgb9e5(pl.x) * local;
      o = gi_origin + wi * 1e-4f;
      want = true;
      flags = TP_HIST;
    }
  }
  fb.st_a[id] = make_uint4(rng, pid, flags, 0u);
  fb.st_c[id] = make_uint4(__float_as_uint(tr.x), __float_as_uint(tr.y), __float_as_uint(tr.z), 0u);
  push_ray(fb, Q_GI_CAND, want, o, 1000.0f - 1e-4f * 2.0f, wi, id);
}

// GI temporal, stage 2: the re-trace's hit (InlinePathTracer::trace with the
// approx() config, inline_path_tracer.wgsl:51-256): uniform light sample and its
// shadow ray, or the sky on a miss.
__global__ void __launch_bounds__(256, AP_TEMPORAL_MIN_BLOCKS) k_gt_b(DevScene s, FrameBuffers fb, Consts c, const uint4* prev_a,
                                              const uint4* prev_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  float pt = __uint_as_float(fb.payload[id].z);
  if (pt < 0.0f) return;
  uint4 sa = fb.st_a[id];
  if (!(sa.z & TP_HIST)) return;
  const uint4 sc = fb.st_c[id];
  const float3 throughput = f3(__uint_as_float(sc.x), __uint_as_float(sc.y), __uint_as_float(sc.z));
  const GiRes pr = gi_unpack(prev_a[sa.y], prev_b[sa.y]);
  float4 ray = fb.rays[id];
  float3 hit = ray_org(ray) + ray_dir(ray) * pt;
  const float3 wi = normalize(pr.point - hit);
  const float3 gi_origin = hit + wi * 0.0001f;
  const uint4 hr = fb.hit_gi[id];
  bool want = false;
  float3 so = f3s(0.0f), sd = f3s(0.0f), val = f3s(0.0f);
  float st = 0.0f;
  if (hr.w != kNoHit) {
    Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
    const MaterialDev* m;
    Surface sf = surface(s, h, gi_origin, wi, &m);
    Bsdf b = load_bsdf(m);
    uint32_t prng = pr.phat_rng;
    float pdf = 0.0f;
    float r0 = rnd(prng), r1 = rnd(prng), r2 = rnd(prng), r3 = rnd(prng), r4 = rnd(prng);
    LightSample ls = sample_uniform(s, r0, r1, r2, make_float2(r3, r4), &pdf);
    float W = 1.0f / pdf;
    if (W > 0.0f) {
      LightEval ev = load_eval(s, ls, sf.hit_point);
      float3 sdir = normalize(ev.point - sf.hit_point);
      float sdist = dist(ev.point, sf.hit_point);
      float ndl = dot(sdir, sf.n);
      if (ndl > 0.0f) {
        float sp = 0.0f;
        float3 refl = disney_eval(b, sf.frame, -wi, sdir, &sp);
        val = throughput * refl * ev.emission * ndl * W;
        so = sf.hit_point + sf.n * 1e-4f;
        sd = sdir;
        st = sdist - 1e-4f * 2.0f;
        want = true;
        sa.z |= TP_SHADOW;
      }
    }
  } else {
    val = f3s(0.0f) + throughput * sky_radiance(s, wi, true);
    sa.z |= TP_DONE;
  }
  fb.st_a[id] = sa;
  fb.st_c[id] = make_uint4(__float_as_uint(val.x), __float_as_uint(val.y), __float_as_uint(val.z), 0u);
  push_ray(fb, Q_GI_SHADOW, want, so, st, sd, id);
}

// GI temporal, stage 3 (restir_gi_temporal.wgsl:97-116): the target, M cap and combine.
__global__ void __launch_bounds__(256) k_gt_c(FrameBuffers fb, Consts c, const uint4* in_a, const uint4* in_b,
                                              uint4* out_a, uint4* out_b, const uint4* prev_a, const uint4* prev_b,
                                              uint4* pout_a, uint4* pout_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  if (__uint_as_float(pl.z) < 0.0f) return;
  const uint4 sa = fb.st_a[id];
  uint32_t rng = sa.x;
  GiRes r = gi_unpack(in_a[id], in_b[id]);
  if (sa.z & TP_HIST) {
    GiRes pr = gi_unpack(prev_a[sa.y], prev_b[sa.y]);
    pr.M = dm::fmin(pr.M, c.cfg.gi_temporal_m_cap);
    const uint4 sc = fb.st_c[id];
    const float3 val = f3(__uint_as_float(sc.x), __uint_as_float(sc.y), __uint_as_float(sc.z));
    float3 acc = f3s(0.0f);
    if (sa.z & TP_DONE) acc = val;
    else if ((sa.z & TP_SHADOW) && fb.vis[Q_GI_SHADOW][id]) acc = acc + val;
    pr.phat = luma(acc);
    r = gi_combine(r, pr, rng);
  }
  out_a[id] = gi_pack_a(r);
  out_b[id] = gi_pack_b(r);
  if (c.cfg.gi_spatial_passes == 0) {
    pout_a[id] = gi_pack_a(r);
    pout_b[id] = gi_pack_b(r);
  }
  pl.y = rng;
  fb.payload[id] = pl;
}

// Bitwise equality of the inputs a target evaluation depends on.
APD bool ls_same(const LightSample& a, const LightSample& b) {
  return __float_as_uint(a.uv.x) == __float_as_uint(b.uv.x) && __float_as_uint(a.uv.y) == __float_as_uint(b.uv.y) &&
         a.inst == b.inst && a.tri == b.tri;
}
APD bool gi_same_key(const GiRes& a, float3 pt, uint32_t prng) {
  return __float_as_uint(a.point.x) == __float_as_uint(pt.x) && __float_as_uint(a.point.y) == __float_as_uint(pt.y) &&
         __float_as_uint(a.point.z) == __float_as_uint(pt.z) && a.phat_rng == prng;
}
APD bool gi_same(const GiRes& a, const GiRes& b) { return gi_same_key(a, b.point, b.phat_rng); }

APD uint32_t mirror(int x, int mx) {
  int v = ((x + mx) % (2 * mx)) - mx;
  return (uint32_t)(v < 0 ? -v : v);
}
APD float ign_animated(uint32_t px, uint32_t py, uint32_t frame) {
  uint32_t fid = frame % 64u;
  float x = (float)px + 5.588238f * (float)fid;
  float y = (float)py + 5.588238f * (float)fid;
  return dm::fract(52.9829189f * dm::fract(0.06711056f * x + 0.00583715f * y));
}
APD float depth_cs(float d, float zn, float zf) {
  float zl = (d - zn) / zf;
  return (zn * zf) / (zf - zl * (zf - zn));
}

// Per-pixel setup shared by the spatial passes (restir_di_spatial.wgsl:70-100,
// restir_gi_spatial.wgsl:71-103): the primary hit, its context and the
// per-pass spiral offsets.
struct SpatialPixel {
  uint32_t x, y, id;
  float3 direction, hit, wo;
  uint4 cx;
  float cdepth;
  float3 cn;
  float roff, aoff;
};

template <bool GI>
APD void spatial_pixel(const FrameBuffers& fb, const Consts& c, uint32_t x, uint32_t y, uint32_t pass_idx,
                       uint32_t pass_count, float pt, SpatialPixel& sp) {
  sp.x = x;
  sp.y = y;
  sp.id = y * c.W + x;
  const uint32_t cur = c.frame_idx & 1u;
  float4 ray = fb.rays[sp.id];
  sp.direction = ray_dir(ray);
  sp.hit = ray_org(ray) + sp.direction * pt;
  sp.wo = -sp.direction;
  sp.cx = fb.ctx[sp.id];
  sp.cdepth = depth_cs(__uint_as_float(fb.gb_a[cur][sp.id].w), 0.001f, 10000.0f);
  sp.cn = unpack_oct30(fb.gb_b[cur][sp.id].x);
  uint32_t frame_arg = GI ? c.seed * 3u + pass_idx : c.seed * pass_count + pass_idx;
  sp.roff = ign_animated(x, y, frame_arg);
  uint32_t psx = pass_idx == 0 ? (x >> 2) : (x >> 1);
  uint32_t psy = pass_idx == 0 ? (y >> 2) : (y >> 1);
  uint32_t aseed = hash_combine(psx, hash_combine(psy, frame_arg));
  sp.aoff = __uint2float_rn(aseed) * (1.0f / 4294967296.0f) * kTwoPi;
}

APD float spatial_radius0(const Consts& c) { return (float)(c.W + c.H) / 2.0f * 0.05f; }

// Neighbour i on the golden-angle spiral (restir_di_spatial.wgsl:104-113).
APD uint32_t spatial_neighbour(const Consts& c, const SpatialPixel& sp, uint32_t i, uint32_t nsamples, float radius) {
  const float golden = 2.39996322972865332f;
  float angle = (float)i * golden + sp.aoff;
  float cr = dm::pow_((float)i / (float)nsamples, 0.5f) * radius + sp.roff;
  float sa, ca;
  dm::sincos_(angle, &sa, &ca);
  int ox = dm::f2i(cr * ca), oy = dm::f2i(cr * sa);
  // mirror_pixel (restir_*_spatial.wgsl:59-68) can return the resolution itself
  // (one past the edge, an out-of-bounds read in the reference): clamp to the edge
  uint32_t nx = min(mirror((int)sp.x + ox, (int)c.W), c.W - 1), ny = min(mirror((int)sp.y + oy, (int)c.H), c.H - 1);
  return ny * c.W + nx;
}

// Depth (10 %) and normal (25 degrees) similarity of neighbour nid.
APD bool spatial_similar(const FrameBuffers& fb, const Consts& c, const SpatialPixel& sp, uint32_t nid) {
  const uint32_t cur = c.frame_idx & 1u;
  float ndepth = __uint_as_float(fb.gb_a[cur][nid].w);
  if (ndepth == 0.0f) return false;
  float nd = depth_cs(ndepth, 0.001f, 10000.0f);
  bool vd = (dm::fabs_(sp.cdepth - nd) / sp.cdepth) < 0.1f;
  bool vn = dot(sp.cn, unpack_oct30(fb.gb_b[cur][nid].x)) > 0.906f;
  return vd && vn;
}

// restir_di_spatial.wgsl:70-163 (GI = false) and restir_gi_spatial.wgsl:71-166 (GI = true)
template <bool GI>
__global__ void k_spatial(DevScene s, FrameBuffers fb, Consts c, uint32_t pass_idx, uint32_t pass_count,
                          uint32_t nsamples, uint32_t unbiased, const uint4* in_a, const uint4* in_b, uint4* out_a,
                          uint4* out_b, uint4* prev_a, uint4* prev_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  float pt = __uint_as_float(pl.z);
  if (pt < 0.0f) return;
  SpatialPixel sp;
  spatial_pixel<GI>(fb, c, x, y, pass_idx, pass_count, pt, sp);
  const uint32_t cur = c.frame_idx & 1u;
  const uint4* ga = fb.gb_a[cur];
  uint32_t rng = pl.y;
  float3 T = unpack_rgb9e5(pl.x);
  const float3 hit = sp.hit, wo = sp.wo;
  const uint4 cx = sp.cx;
  float radius = spatial_radius0(c);
  DiRes rdi;
  GiRes rgi;
  if (GI) rgi = gi_unpack(in_a[id], in_b[id]);
  else rdi = di_unpack(in_a[id], in_b[id]);
  // Memo of the last target value evaluated at this pixel: the unbiased combine
  // re-evaluates the combined sample here, and that sample is always either the
  // neighbour's (evaluated just before) or this pixel's previous one.
  bool memo = false;
  LightSample memo_ls = ls_empty();
  float3 memo_pt = f3s(0.0f);
  uint32_t memo_rng = 0u;
  float memo_val = 0.0f;
  for (uint32_t i = 0; i < nsamples; ++i) {
    uint32_t nid = spatial_neighbour(c, sp, i, nsamples, radius);
    if (nid == id) continue;
    bool valid = spatial_similar(fb, c, sp, nid);
    uint4 nga = ga[nid];
    if (valid) {
      float3 npos = f3(__uint_as_float(nga.x), __uint_as_float(nga.y), __uint_as_float(nga.z));
      if (!GI) {
        DiRes nr = di_unpack(in_a[nid], in_b[nid]);
        nr.phat = ls_phat(s, nr.s, cx, hit, wo, unbiased > 0);
        valid = nr.phat > 0.0f;
        if (!unbiased) {
          rdi = di_combine(rdi, nr, rng);
        } else {
          float3 nwo = -ray_dir(fb.rays[nid]);
          uint4 ncx = fb.ctx[nid];
          DiRes cmb = di_new();
          di_update(cmb, rdi.phat * rdi.W * rdi.M, rng, rdi.s, rdi.phat);
          di_update(cmb, nr.phat * nr.W * nr.M, rng, nr.s, nr.phat);
          cmb.M = rdi.M + nr.M;
          float z = 0.0f;
          float zc;
          if (ls_same(cmb.s, nr.s)) zc = nr.phat;
          else if (memo && ls_same(cmb.s, memo_ls)) zc = memo_val;
          else zc = ls_phat(s, cmb.s, cx, hit, wo, true);
          memo = true;
          memo_ls = cmb.s;
          memo_val = zc;
          if (zc > 0.0f) z = z + rdi.M;
          if (ls_phat(s, cmb.s, ncx, npos, nwo, true) > 0.0f) z = z + nr.M;
          if (cmb.phat > 1e-6f && z * cmb.wsum > 1e-6f) cmb.W = (1.0f / cmb.phat) * (1.0f / z * cmb.wsum);
          rdi = cmb;
        }
      } else {
        GiRes nr = gi_unpack(in_a[nid], in_b[nid]);
        nr.phat = gi_phat(s, nr, cx, T, hit, wo);
        valid = nr.phat > 0.0f;
        if (!unbiased) {
          rgi = gi_combine(rgi, nr, rng);
        } else {
          float3 nwo = -ray_dir(fb.rays[nid]);
          float3 nT = unpack_rgb9e5(fb.payload[nid].x);
          uint4 ncx = fb.ctx[nid];
          GiRes cmb = gi_new();
          gi_update(cmb, rgi.phat * rgi.W * rgi.M, rng, rgi.point, rgi.phat, rgi.phat_rng);
          gi_update(cmb, nr.phat * nr.W * nr.M, rng, nr.point, nr.phat, nr.phat_rng);
          cmb.M = rgi.M + nr.M;
          float z = 0.0f;
          float zc;
          if (gi_same(cmb, nr)) zc = nr.phat;
          else if (memo && gi_same_key(cmb, memo_pt, memo_rng)) zc = memo_val;
          else zc = gi_phat(s, cmb, cx, T, hit, wo);
          memo = true;
          memo_pt = cmb.point;
          memo_rng = cmb.phat_rng;
          memo_val = zc;
          if (zc > 0.0f) z = z + rgi.M;
          if (gi_phat(s, cmb, ncx, nT, npos, nwo) > 0.0f) z = z + nr.M;
          if (cmb.phat > 0.0f && z * cmb.wsum > 0.0f) cmb.W = (1.0f / cmb.phat) * (1.0f / z * cmb.wsum);
          rgi = cmb;
        }
      }
    }
    if (!valid) radius = dm::fmax(radius * 0.5f, 3.0f);
  }
  if (GI) {
    out_a[id] = gi_pack_a(rgi);
    out_b[id] = gi_pack_b(rgi);
    if (pass_idx == pass_count - 1) {
      prev_a[id] = gi_pack_a(rgi);
      prev_b[id] = gi_pack_b(rgi);
    }
  } else {
    out_a[id] = di_pack_a(rdi);
    out_b[id] = di_pack_b(rdi);
    if (pass_idx == pass_count - 1) {
      prev_a[id] = di_pack_a(rdi);
      prev_b[id] = di_pack_b(rdi);
    }
  }
  pl.y = rng;
  fb.payload[id] = pl;
}

// ---- unbiased ReSTIR DI spatial pass as wavefront stages ---------------------
//
// The same pass as k_spatial<false> with unbiased = 1, split at its visibility
// tests so that every shadow ray goes through the persistent any-hit queue
// kernel instead of being traversed inline.  Per neighbour i:
//   k_dsp_ca(i)  finishes neighbour i-1 (its Z, hence W), picks neighbour i,
//                queues the visibility ray of the neighbour's sample here;
//   any-hit queue Q_DI_SHADOW;
//   k_dsp_b(i)   combines; queues the visibility ray of the combined sample
//                here (unless its target is already known) on Q_RIS_SHADOW
//                and at the neighbour on Q_GI_SHADOW;
//   any-hit queues.
// k_dsp_ca(nsamples) finishes the last neighbour and writes the history and
// the payload's RNG.  The reservoir being built lives in out_a/out_b; the loop
// state in the stage buffers:
//   st_a {radius, rng, neighbour id, flags}   st_b memoised light sample
//   st_c {memo target, target of the neighbour's sample here, of the combined
//         sample here, of the combined sample at the neighbour}
//   st_d {M of the pixel's reservoir, M of the neighbour's, known target here}
// Targets are the unshadowed values of LightSample::phat
// (di_reservoir.wgsl:58-97); a target counts only when its ray is unoccluded.
enum : uint32_t {
  SP_ACTIVE = 1u,    // neighbour passed the depth/normal test this iteration
  SP_RAY_N = 2u,     // visibility ray of the neighbour's sample here queued
  SP_RAY_C = 4u,     // visibility ray of the combined sample here queued
  SP_RAY_CN = 8u,    // visibility ray of the combined sample at the neighbour queued
  SP_ZC_KNOWN = 16u, // target of the combined sample here known without a ray
  SP_MEMO = 32u,     // st_b/st_c.x hold a memoised target
};

#ifndef AP_DSP_MIN_BLOCKS
#define AP_DSP_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(256, AP_DSP_MIN_BLOCKS) k_dsp_ca(DevScene s, FrameBuffers fb, Consts c, uint32_t pass_idx,
                                                uint32_t pass_count, uint32_t nsamples, uint32_t i,
                                                const uint4* in_a, const uint4* in_b, uint4* out_a, uint4* out_b,
                                                uint4* prev_a, uint4* prev_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  const uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  const float pt = __uint_as_float(pl.z);
  if (pt < 0.0f) return;
  uint4 sa, sb, sc;
  if (i == 0) {
    sa = make_uint4(__float_as_uint(spatial_radius0(c)), pl.y, 0u, 0u);
    sb = make_uint4(0u, 0u, 0u, 0u);
    sc = make_uint4(0u, 0u, 0u, 0u);
    out_a[id] = in_a[id];
    out_b[id] = in_b[id];
  } else {
    sa = fb.st_a[id];
    sb = fb.st_b[id];
    sc = fb.st_c[id];
    if (sa.w & SP_ACTIVE) {
      // finish neighbour i-1: Z of the combined sample, then W
      const uint4 sd = fb.st_d[id];
      float zc;
      if (sa.w & SP_ZC_KNOWN) zc = __uint_as_float(sd.z);
      else zc = ((sa.w & SP_RAY_C) && fb.vis[Q_RIS_SHADOW][id]) ? __uint_as_float(sc.z) : 0.0f;
      DiRes cmb = di_unpack(out_a[id], out_b[id]);
      sb = di_pack_b(cmb);  // memo: the combined sample and its target here
      sc.x = __float_as_uint(zc);
      sa.w |= SP_MEMO;
      float z = 0.0f;
      if (zc > 0.0f) z = z + __uint_as_float(sd.x);
      const bool nbr = (sa.w & SP_RAY_CN) && fb.vis[Q_GI_SHADOW][id] && __uint_as_float(sc.w) > 0.0f;
      if (nbr) z = z + __uint_as_float(sd.y);
      if (cmb.phat > 1e-6f && z * cmb.wsum > 1e-6f) {
        cmb.W = (1.0f / cmb.phat) * (1.0f / z * cmb.wsum);
        out_a[id] = di_pack_a(cmb);
      }
    }
  }
  sa.w &= SP_MEMO;
  if (i == nsamples) {
    if (pass_idx == pass_count - 1) {
      prev_a[id] = out_a[id];
      prev_b[id] = out_b[id];
    }
    pl.y = sa.y;
    fb.payload[id] = pl;
    return;
  }
  SpatialPixel sp;
  spatial_pixel<false>(fb, c, x, y, pass_idx, pass_count, pt, sp);
  float radius = __uint_as_float(sa.x);
  const uint32_t nid = spatial_neighbour(c, sp, i, nsamples, radius);
  PhatSplit ph;
  ph.ray = false;
  ph.value = 0.0f;
  if (nid != id) {
    if (spatial_similar(fb, c, sp, nid)) {
      const DiRes nr = di_unpack(in_a[nid], in_b[nid]);
      ph = ls_phat_split(s, nr.s, sp.cx, sp.hit, sp.wo);
      sa.w |= SP_ACTIVE | (ph.ray ? SP_RAY_N : 0u);
      sc.y = __float_as_uint(ph.value);
    } else {
      radius = dm::fmax(radius * 0.5f, 3.0f);
    }
  }
  sa.x = __float_as_uint(radius);
  sa.z = nid;
  fb.st_a[id] = sa;
  fb.st_b[id] = sb;
  fb.st_c[id] = sc;
  push_ray(fb, Q_DI_SHADOW, ph.ray, ph.o, ph.tmax, ph.d, id);
}

__global__ void __launch_bounds__(256, AP_DSP_MIN_BLOCKS) k_dsp_b(DevScene s, FrameBuffers fb, Consts c, uint32_t pass_idx,
                                               uint32_t pass_count, const uint4* in_a, const uint4* in_b,
                                               uint4* out_a, uint4* out_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  const uint32_t id = y * c.W + x;
  const float pt = __uint_as_float(fb.payload[id].z);
  if (pt < 0.0f) return;
  uint4 sa = fb.st_a[id];
  if (!(sa.w & SP_ACTIVE)) return;
  uint4 sc = fb.st_c[id];
  const uint4 sb = fb.st_b[id];
  const uint32_t nid = sa.z;
  uint32_t rng = sa.y;
  DiRes rdi = di_unpack(out_a[id], out_b[id]);
  DiRes nr = di_unpack(in_a[nid], in_b[nid]);
  nr.phat = ((sa.w & SP_RAY_N) && fb.vis[Q_DI_SHADOW][id]) ? __uint_as_float(sc.y) : 0.0f;
  const bool valid = nr.phat > 0.0f;
  DiRes cmb = di_new();
  di_update(cmb, rdi.phat * rdi.W * rdi.M, rng, rdi.s, rdi.phat);
  di_update(cmb, nr.phat * nr.W * nr.M, rng, nr.s, nr.phat);
  cmb.M = rdi.M + nr.M;
  SpatialPixel sp;
  spatial_pixel<false>(fb, c, x, y, pass_idx, pass_count, pt, sp);
  const LightSample memo_ls{make_float2(__uint_as_float(sb.x), __uint_as_float(sb.y)), sb.z, sb.w};
  float zc = 0.0f;
  PhatSplit here;
  here.ray = false;
  here.value = 0.0f;
  if (ls_same(cmb.s, nr.s)) {
    zc = nr.phat;
    sa.w |= SP_ZC_KNOWN;
  } else if ((sa.w & SP_MEMO) && ls_same(cmb.s, memo_ls)) {
    zc = __uint_as_float(sc.x);
    sa.w |= SP_ZC_KNOWN;
  } else {
    here = ls_phat_split(s, cmb.s, sp.cx, sp.hit, sp.wo);
    if (here.ray) sa.w |= SP_RAY_C;
    else sa.w |= SP_ZC_KNOWN;  // target 0 without a ray
    sc.z = __float_as_uint(here.value);
  }
  const uint4 nga = fb.gb_a[c.frame_idx & 1u][nid];
  const float3 npos = f3(__uint_as_float(nga.x), __uint_as_float(nga.y), __uint_as_float(nga.z));
  const float3 nwo = -ray_dir(fb.rays[nid]);
  const PhatSplit there = ls_phat_split(s, cmb.s, fb.ctx[nid], npos, nwo);
  if (there.ray) sa.w |= SP_RAY_CN;
  sc.w = __float_as_uint(there.value);
  float radius = __uint_as_float(sa.x);
  if (!valid) radius = dm::fmax(radius * 0.5f, 3.0f);
  sa.x = __float_as_uint(radius);
  sa.y = rng;
  out_a[id] = di_pack_a(cmb);
  out_b[id] = di_pack_b(cmb);
  fb.st_a[id] = sa;
  fb.st_c[id] = sc;
  fb.st_d[id] = make_uint4(__float_as_uint(rdi.M), __float_as_uint(nr.M), __float_as_uint(zc), 0u);
  push_ray(fb, Q_RIS_SHADOW, here.ray, here.o, here.tmax, here.d, id);
  push_ray(fb, Q_GI_SHADOW, there.ray, there.o, there.tmax, there.d, id);
}

// ---- unbiased ReSTIR GI spatial pass as wavefront stages ---------------------
//
// The same pass as k_spatial<true> with unbiased = 1 (restir_gi_spatial.wgsl:
// 71-166), split at the rays of its target evaluations.  A target
// (GiReservoir::phat, inline_path_tracer.wgsl:299-331) re-traces a closest-hit
// ray toward the sample point and, at its hit, a shadow ray of a uniform light
// sample (InlinePathTracer::trace with the approx() config, :51-256).  Per
// neighbour i:
//   k_gsp_a(i)  finishes neighbour i-1 (its Z, hence W), picks neighbour i
//               and queues the re-trace of its sample's target here (Q_GI_CAND);
//   closest-hit queue;
//   k_gsp_b(i)  shades that hit and queues its shadow ray (Q_GI_SHADOW);
//   any-hit queue;
//   k_gsp_c(i)  combines; queues the re-traces of the combined sample's target
//               here (Q_BSDF_CAND; none when it is known: the neighbour's own
//               sample, or the memoised one) and at the neighbour (Q_GI_CAND);
//   both closest-hit queues in one launch;
//   k_gsp_d(i)  shades those hits and queues their shadow rays (Q_RIS_SHADOW,
//               Q_GI_SHADOW);
//   both any-hit queues in one launch.
// k_gsp_a(nsamples) finishes the last neighbour and writes the history and the
// payload's RNG.  The reservoir being built lives in out_a/out_b; the loop
// state in the stage buffers:
//   st_a {radius, rng, neighbour id, flags}   st_b memo {point.xyz, phat_rng}
//   st_c {memoised target, throughput of the pending re-trace here (.yzw),
//         later the neighbour's sample's target here if unoccluded (.y)}
//   st_d {M of the pixel's reservoir, M of the neighbour's, target of the
//         combined sample here (known, or if unoccluded), -}
//   st_e {throughput of the re-trace at the neighbour}
// The target of the combined sample at the neighbour only counts by its sign.
// With a zero re-trace throughput it is not positive whatever the rays find
// (the radiance is 0, or NaN from an infinite factor), so that re-trace is not
// traced.
enum : uint32_t {
  GS_ACTIVE = 1u,      // neighbour passed the depth/normal test: its sample is combined
  GS_N_SHADOW = 2u,    // neighbour's sample here: shadow ray queued
  GS_C_RAY = 4u,       // combined sample here: re-trace queued (target not known)
  GS_C_SHADOW = 8u,    // combined sample here: shadow ray queued
  GS_CN_RAY = 16u,     // combined sample at the neighbour: re-trace queued
  GS_CN_SHADOW = 32u,  // combined sample at the neighbour: shadow ray queued
  GS_CN_POS = 64u,     // combined sample at the neighbour: target positive if unoccluded
  GS_MEMO = 128u,      // st_b / st_c.x hold a memoised target
};

// First half of GiReservoir::phat at a surface (hit point, wo, light-sample
// context cx, path throughput T): direction to the sample point, the
// re-trace's origin and throughput.
struct GiRetrace {
  float3 wi, gi_origin, tr;
};
APD GiRetrace gi_retrace_begin(const DevScene& s, float3 point, const uint4 cx, float3 T, float3 hit, float3 wo) {
  Bsdf b = load_bsdf(s.materials + cx.x);
  Frame fr = ctx_frame(cx);
  GiRetrace g;
  g.wi = normalize(point - hit);
  float sp = 0.0f;
  float3 refl = disney_eval(b, fr, wo, g.wi, &sp);
  float cos_in = dm::fabs_(dot(g.wi, fr.n));
  float3 local = cos_in * refl;
  g.gi_origin = hit + g.wi * 0.0001f;
  g.tr = T * local;
  return g;
}
APD GiRetrace gi_retrace_at(float3 point, float3 hit, float3 tr) {
  GiRetrace g;
  g.wi = normalize(point - hit);
  g.gi_origin = hit + g.wi * 0.0001f;
  g.tr = tr;
  return g;
}

// Second half: the re-trace's closest hit `hr` shaded with a uniform light
// sample drawn from the sample's own stream (prng), or the sky on a miss.
// acc is the radiance when the shadow ray (if any) is unoccluded.
struct GiShade {
  float3 acc, o, d;
  float tmax;
  bool ray;
};
APD GiShade gi_retrace_hit(const DevScene& s, const uint4 hr, const GiRetrace& g, uint32_t prng) {
  GiShade r;
  r.acc = f3s(0.0f);
  r.o = f3s(0.0f);
  r.d = f3s(0.0f);
  r.tmax = 0.0f;
  r.ray = false;
  if (hr.w != kNoHit) {
    Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
    const MaterialDev* m;
    Surface sf = surface(s, h, g.gi_origin, g.wi, &m);
    Bsdf b = load_bsdf(m);
    float pdf = 0.0f;
    float r0 = rnd(prng), r1 = rnd(prng), r2 = rnd(prng), r3 = rnd(prng), r4 = rnd(prng);
    LightSample ls = sample_uniform(s, r0, r1, r2, make_float2(r3, r4), &pdf);
    float W = 1.0f / pdf;
    if (W > 0.0f) {
      LightEval ev = load_eval(s, ls, sf.hit_point);
      float3 sdir = normalize(ev.point - sf.hit_point);
      float sdist = dist(ev.point, sf.hit_point);
      float ndl = dot(sdir, sf.n);
      if (ndl > 0.0f) {
        float sp = 0.0f;
        float3 refl = disney_eval(b, sf.frame, -g.wi, sdir, &sp);
        r.acc = f3s(0.0f) + g.tr * refl * ev.emission * ndl * W;
        r.o = sf.hit_point + sf.n * 1e-4f;
        r.d = sdir;
        r.tmax = sdist - 1e-4f * 2.0f;
        r.ray = true;
      }
    }
  } else {
    r.acc = f3s(0.0f) + g.tr * sky_radiance(s, g.wi, true);
  }
  return r;
}

APD float3 f3_bits(uint32_t x, uint32_t y, uint32_t z) { return f3(__uint_as_float(x), __uint_as_float(y), __uint_as_float(z)); }
APD float3 primary_hit(const FrameBuffers& fb, uint32_t id, float pt) {
  const float4 ray = fb.rays[id];
  return ray_org(ray) + ray_dir(ray) * pt;
}

#ifndef AP_GSP_MIN_BLOCKS
// resident blocks of 256 per SM the GI spatial stages are register-capped for
// (1080p benchmark frame, CUDA events: 2, 3, 4, 5, 6 blocks gave 5.5, 4.4,
// 4.0, 4.0, 4.0 ms for the 21 stage launches)
#define AP_GSP_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(256, AP_GSP_MIN_BLOCKS) k_gsp_a(DevScene s, FrameBuffers fb, Consts c, uint32_t pass_idx,
                                                uint32_t pass_count, uint32_t nsamples, uint32_t i,
                                                const uint4* in_a, const uint4* in_b, uint4* out_a, uint4* out_b,
                                                uint4* prev_a, uint4* prev_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  const uint32_t id = y * c.W + x;
  uint4 pl = fb.payload[id];
  const float pt = __uint_as_float(pl.z);
  if (pt < 0.0f) return;
  uint4 sa, sb, sc;
  if (i == 0) {
    sa = make_uint4(__float_as_uint(spatial_radius0(c)), pl.y, 0u, 0u);
    sb = make_uint4(0u, 0u, 0u, 0u);
    sc = make_uint4(0u, 0u, 0u, 0u);
    out_a[id] = in_a[id];
    out_b[id] = in_b[id];
  } else {
    sa = fb.st_a[id];
    sb = fb.st_b[id];
    sc = fb.st_c[id];
    if (sa.w & GS_ACTIVE) {
      // finish neighbour i-1: Z of the combined sample, then W
      const uint4 sd = fb.st_d[id];
      float zc = __uint_as_float(sd.z);
      if ((sa.w & GS_C_SHADOW) && !fb.vis[Q_RIS_SHADOW][id]) zc = luma(f3s(0.0f));
      GiRes cmb = gi_unpack(out_a[id], out_b[id]);
      sb = gi_pack_b(cmb);  // memo: the combined sample and its target here
      sc.x = __float_as_uint(zc);
      sa.w |= GS_MEMO;
      float z = 0.0f;
      if (zc > 0.0f) z = z + __uint_as_float(sd.x);
      const bool there = (sa.w & GS_CN_POS) && (!(sa.w & GS_CN_SHADOW) || fb.vis[Q_GI_SHADOW][id]);
      if (there) z = z + __uint_as_float(sd.y);
      if (cmb.phat > 0.0f && z * cmb.wsum > 0.0f) {
        cmb.W = (1.0f / cmb.phat) * (1.0f / z * cmb.wsum);
        out_a[id] = gi_pack_a(cmb);
      }
    }
  }
  sa.w &= GS_MEMO;
  if (i == nsamples) {
    if (pass_idx == pass_count - 1) {
      prev_a[id] = out_a[id];
      prev_b[id] = out_b[id];
    }
    pl.y = sa.y;
    fb.payload[id] = pl;
    return;
  }
  SpatialPixel sp;
  spatial_pixel<true>(fb, c, x, y, pass_idx, pass_count, pt, sp);
  float radius = __uint_as_float(sa.x);
  const uint32_t nid = spatial_neighbour(c, sp, i, nsamples, radius);
  bool want = false;
  GiRetrace g;
  g.wi = f3s(0.0f);
  g.gi_origin = f3s(0.0f);
  if (nid != id) {
    if (spatial_similar(fb, c, sp, nid)) {
      const GiRes nr = gi_unpack(in_a[nid], in_b[nid]);
      g = gi_retrace_begin(s, nr.point, sp.cx, unpack_rgb9e5(pl.x), sp.hit, sp.wo);
      want = true;
      sa.w |= GS_ACTIVE;
      sc.y = __float_as_uint(g.tr.x);
      sc.z = __float_as_uint(g.tr.y);
      sc.w = __float_as_uint(g.tr.z);
    } else {
      radius = dm::fmax(radius * 0.5f, 3.0f);
    }
  }
  sa.x = __float_as_uint(radius);
  sa.z = nid;
  fb.st_a[id] = sa;
  fb.st_b[id] = sb;
  fb.st_c[id] = sc;
  push_ray(fb, Q_GI_CAND, want, g.gi_origin + g.wi * 1e-4f, 1000.0f - 1e-4f * 2.0f, g.wi, id);
}

__global__ void __launch_bounds__(256, AP_GSP_MIN_BLOCKS) k_gsp_b(DevScene s, FrameBuffers fb, Consts c, const uint4* in_a,
                                                const uint4* in_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  const uint32_t id = y * c.W + x;
  const float pt = __uint_as_float(fb.payload[id].z);
  if (pt < 0.0f) return;
  uint4 sa = fb.st_a[id];
  if (!(sa.w & GS_ACTIVE)) return;
  uint4 sc = fb.st_c[id];
  const GiRes nr = gi_unpack(in_a[sa.z], in_b[sa.z]);
  const GiRetrace g = gi_retrace_at(nr.point, primary_hit(fb, id, pt), f3_bits(sc.y, sc.z, sc.w));
  const GiShade sh = gi_retrace_hit(s, fb.hit_gi[id], g, nr.phat_rng);
  if (sh.ray) sa.w |= GS_N_SHADOW;
  sc.y = __float_as_uint(luma(sh.acc));
  fb.st_a[id] = sa;
  fb.st_c[id] = sc;
  push_ray(fb, Q_GI_SHADOW, sh.ray, sh.o, sh.tmax, sh.d, id);
}

__global__ void __launch_bounds__(256, AP_GSP_MIN_BLOCKS) k_gsp_c(DevScene s, FrameBuffers fb, Consts c, uint32_t pass_idx,
                                                uint32_t pass_count, const uint4* in_a, const uint4* in_b,
                                                uint4* out_a, uint4* out_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  const uint32_t id = y * c.W + x;
  const uint4 pl = fb.payload[id];
  const float pt = __uint_as_float(pl.z);
  if (pt < 0.0f) return;
  uint4 sa = fb.st_a[id];
  if (!(sa.w & GS_ACTIVE)) return;
  uint4 sc = fb.st_c[id];
  const uint4 sb = fb.st_b[id];
  const uint32_t nid = sa.z;
  uint32_t rng = sa.y;
  const GiRes rgi = gi_unpack(out_a[id], out_b[id]);
  GiRes nr = gi_unpack(in_a[nid], in_b[nid]);
  nr.phat = ((sa.w & GS_N_SHADOW) && !fb.vis[Q_GI_SHADOW][id]) ? luma(f3s(0.0f)) : __uint_as_float(sc.y);
  const bool valid = nr.phat > 0.0f;
  GiRes cmb = gi_new();
  gi_update(cmb, rgi.phat * rgi.W * rgi.M, rng, rgi.point, rgi.phat, rgi.phat_rng);
  gi_update(cmb, nr.phat * nr.W * nr.M, rng, nr.point, nr.phat, nr.phat_rng);
  cmb.M = rgi.M + nr.M;
  SpatialPixel sp;
  spatial_pixel<true>(fb, c, x, y, pass_idx, pass_count, pt, sp);
  float zc = 0.0f;
  bool here = false;
  GiRetrace gc;
  gc.wi = f3s(0.0f);
  gc.gi_origin = f3s(0.0f);
  if (gi_same(cmb, nr)) {
    zc = nr.phat;
  } else if ((sa.w & GS_MEMO) && gi_same_key(cmb, f3_bits(sb.x, sb.y, sb.z), sb.w)) {
    zc = __uint_as_float(sc.x);
  } else {
    gc = gi_retrace_begin(s, cmb.point, sp.cx, unpack_rgb9e5(pl.x), sp.hit, sp.wo);
    here = true;
    sa.w |= GS_C_RAY;
    sc.y = __float_as_uint(gc.tr.x);
    sc.z = __float_as_uint(gc.tr.y);
    sc.w = __float_as_uint(gc.tr.z);
  }
  const uint4 nga = fb.gb_a[c.frame_idx & 1u][nid];
  const float3 npos = f3_bits(nga.x, nga.y, nga.z);
  const float3 nwo = -ray_dir(fb.rays[nid]);
  const float3 nT = unpack_rgb9e5(fb.payload[nid].x);
  const GiRetrace gn = gi_retrace_begin(s, cmb.point, fb.ctx[nid], nT, npos, nwo);
  const bool there = !(gn.tr.x == 0.0f && gn.tr.y == 0.0f && gn.tr.z == 0.0f);
  if (there) sa.w |= GS_CN_RAY;
  float radius = __uint_as_float(sa.x);
  if (!valid) radius = dm::fmax(radius * 0.5f, 3.0f);
  sa.x = __float_as_uint(radius);
  sa.y = rng;
  out_a[id] = gi_pack_a(cmb);
  out_b[id] = gi_pack_b(cmb);
  fb.st_a[id] = sa;
  fb.st_c[id] = sc;
  fb.st_d[id] = make_uint4(__float_as_uint(rgi.M), __float_as_uint(nr.M), __float_as_uint(zc), 0u);
  fb.st_e[id] = make_uint4(__float_as_uint(gn.tr.x), __float_as_uint(gn.tr.y), __float_as_uint(gn.tr.z), 0u);
  push_ray(fb, Q_BSDF_CAND, here, gc.gi_origin + gc.wi * 1e-4f, 1000.0f - 1e-4f * 2.0f, gc.wi, id);
  push_ray(fb, Q_GI_CAND, there, gn.gi_origin + gn.wi * 1e-4f, 1000.0f - 1e-4f * 2.0f, gn.wi, id);
}

__global__ void __launch_bounds__(256, AP_GSP_MIN_BLOCKS) k_gsp_d(DevScene s, FrameBuffers fb, Consts c, const uint4* out_a,
                                                const uint4* out_b) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  const uint32_t id = y * c.W + x;
  const float pt = __uint_as_float(fb.payload[id].z);
  if (pt < 0.0f) return;
  uint4 sa = fb.st_a[id];
  if (!(sa.w & GS_ACTIVE)) return;
  const GiRes cmb = gi_unpack(out_a[id], out_b[id]);
  GiShade hc = {}, hn = {};
  if (sa.w & GS_C_RAY) {
    const uint4 sc = fb.st_c[id];
    uint4 sd = fb.st_d[id];
    const GiRetrace g = gi_retrace_at(cmb.point, primary_hit(fb, id, pt), f3_bits(sc.y, sc.z, sc.w));
    hc = gi_retrace_hit(s, fb.hit_bsdf[id], g, cmb.phat_rng);
    if (hc.ray) sa.w |= GS_C_SHADOW;
    sd.z = __float_as_uint(luma(hc.acc));
    fb.st_d[id] = sd;
  }
  if (sa.w & GS_CN_RAY) {
    const uint4 se = fb.st_e[id];
    const uint4 nga = fb.gb_a[c.frame_idx & 1u][sa.z];
    const GiRetrace g = gi_retrace_at(cmb.point, f3_bits(nga.x, nga.y, nga.z), f3_bits(se.x, se.y, se.z));
    hn = gi_retrace_hit(s, fb.hit_gi[id], g, cmb.phat_rng);
    if (hn.ray) sa.w |= GS_CN_SHADOW;
    if (luma(hn.acc) > 0.0f) sa.w |= GS_CN_POS;
  }
  fb.st_a[id] = sa;
  push_ray(fb, Q_RIS_SHADOW, hc.ray, hc.o, hc.tmax, hc.d, id);
  push_ray(fb, Q_GI_SHADOW, hn.ray, hn.o, hn.tmax, hn.d, id);
}

// ---- radiance cache mode ------------------------------------------------------

// Query of the cache at a path vertex: position, roughness, outgoing direction,
// diffuse albedo color (1 - metallic)(1 - transmission), specular albedo
// mix(0.08 specular, color, metallic).
APD void rc_query(const Surface& sf, const MaterialDev* m, float3 wo, float4* q) {
  const float3 col = ld3(m->color);
  const float kd = (1.0f - m->metallic) * (1.0f - m->transmission);
  const float3 spec = f3s(0.08f * m->specular) * (1.0f - m->metallic) + col * m->metallic;
  q[0] = make_float4(sf.hit_point.x, sf.hit_point.y, sf.hit_point.z, m->roughness);
  q[1] = make_float4(wo.x, wo.y, wo.z, 0.0f);
  q[2] = make_float4(col.x * kd, col.y * kd, col.z * kd, spec.x);
  q[3] = make_float4(spec.y, spec.z, 0.0f, 0.0f);
}

APD bool rc_training_pixel(uint32_t id, uint32_t frame_idx, uint32_t stride) {
  return id % stride == (frame_idx * 7u + 3u) % stride;
}

// After the extension rays of a bounce: training pixels record each suffix
// vertex (query, throughput, radiance so far); other pixels retire their path
// at the prefix-th hit into the cache.
__global__ void __launch_bounds__(kBlock) k_rc_vertex(DevScene s, FrameBuffers fb, Consts c, RcFrame rc) {
  const uint32_t count = bounce_count(fb, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t id = bounce_path(fb, c, i);
    const uint4 hr = fb.hits[id];
    if (hr.w == kNoHit) continue;
    const bool tp = rc_training_pixel(id, c.frame_idx, rc.stride);
    if (!tp && c.bounce != rc.prefix) continue;
    if (tp && (c.bounce == 0 || c.bounce >= kRcMaxBounces)) continue;
    const float4 ray = fb.rays[id];
    const float3 origin = ray_org(ray), direction = ray_dir(ray);
    Hit h{__uint_as_float(hr.x), __uint_as_float(hr.y), __uint_as_float(hr.z), hr.w};
    const MaterialDev* m;
    const Surface sf = surface(s, h, origin, direction, &m);
    float4 q[4];
    rc_query(sf, m, -direction, q);
    const float3 T = unpack_rgb9e5(fb.payload[id].x);
    if (tp) {
      float4* r = rc.rec + ((size_t)(id / rc.stride) * kRcMaxBounces + c.bounce) * 6;
      const float3 acc = unpack_rgb9e5(fb.radiance[id]);
      r[0] = q[0]; r[1] = q[1]; r[2] = q[2]; r[3] = q[3];
      r[4] = make_float4(T.x, T.y, T.z, 0.0f);
      r[5] = make_float4(acc.x, acc.y, acc.z, (float)(c.sample + 1));  // tag: the sample that wrote it
    } else {  // retired: its query goes to the next compact slot (one atomic per warp)
      const unsigned am = __activemask();
      const int lane = (int)lane_id(), leader = __ffs(am) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(&rc.counts[2], (uint32_t)__popc(am));
      const uint32_t j = __shfl_sync(am, base, leader) + __popc(am & ((1u << lane) - 1u));
      float4* dst = rc.q + 4 * (size_t)j;
      dst[0] = q[0]; dst[1] = q[1]; dst[2] = q[2]; dst[3] = q[3];
      rc.T[j] = make_float4(T.x, T.y, T.z, 1.0f);
      rc.own[j] = id;
      fb.hits[id].w = kRcRetired;
    }
  }
}

APD float3 rc_target(const float4* r, float3 acc_end) {
  const float3 T = f3(r[4].x, r[4].y, r[4].z), a = f3(r[5].x, r[5].y, r[5].z);
  const float3 d = acc_end - a;
  return f3(T.x > 0.0f ? dm::fmax(d.x, 0.0f) / T.x : 0.0f, T.y > 0.0f ? dm::fmax(d.y, 0.0f) / T.y : 0.0f,
            T.z > 0.0f ? dm::fmax(d.z, 0.0f) / T.z : 0.0f);
}

// Pass 1: count the valid records.  Pass 2: keep each with probability
// batch / count (a hash of the record slot and frame), up to `batch`.
// Only records of the frame's last sample pair with its final radiance.
__global__ void k_rc_count(RcFrame rc, uint32_t slots, float last_tag) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  bool v = k < slots && rc.rec[6 * (size_t)k + 5].w == last_tag;
  unsigned b = __ballot_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(&rc.counts[0], (uint32_t)__popc(b));
}

// A record of the last sample goes into the training batch with probability
// batch / candidates, drawn from its slot index and the frame index.
APD bool rc_kept(const RcFrame& rc, uint32_t k, uint32_t slots, uint32_t frame_idx, float last_tag) {
  if (k >= slots || rc.rec[6 * (size_t)k + 5].w != last_tag) return false;
  const uint32_t cand = rc.counts[0];
  const float keep = cand <= rc.batch ? 1.0f : (float)rc.batch / (float)cand;
  const float u = (float)(pcg_hash(k ^ xor_shift(frame_idx * 0x9E3779B9u)) >> 8) * (1.0f / 16777216.0f);
  return u < keep;
}

// Records kept per block of 256 slots (count_scan turns them into the
// blocks' first batch slots, so the batch is in record order).
__global__ void k_rc_keep(RcFrame rc, uint32_t slots, uint32_t frame_idx, float last_tag) {
  uint32_t tot;
  block_prefix(rc_kept(rc, blockIdx.x * blockDim.x + threadIdx.x, slots, frame_idx, last_tag), &tot);
  if (threadIdx.x == 0) rc.bcount[blockIdx.x] = tot;
}

__global__ void k_rc_batch(FrameBuffers fb, RcFrame rc, uint32_t slots, uint32_t frame_idx, float last_tag) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool kept = rc_kept(rc, k, slots, frame_idx, last_tag);
  uint32_t tot;
  const uint32_t slot = rc.bcount[blockIdx.x] + block_prefix(kept, &tot);
  if (!kept || slot >= rc.batch) return;
  const float4* r = rc.rec + 6 * (size_t)k;
  const uint32_t pixel = (k / kRcMaxBounces) * rc.stride + (frame_idx * 7u + 3u) % rc.stride;
  const float3 t = rc_target(r, unpack_rgb9e5(fb.radiance[pixel]));
  float4* q = rc.bq + 4 * (size_t)slot;
  q[0] = r[0]; q[1] = r[1]; q[2] = r[2]; q[3] = r[3];
  rc.bt[3 * slot + 0] = t.x;
  rc.bt[3 * slot + 1] = t.y;
  rc.bt[3 * slot + 2] = t.z;
}

// Adds throughput x predicted radiance to every retired path's pixel.
__global__ void k_rc_apply(FrameBuffers fb, RcFrame rc, uint32_t P) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= min(rc.counts[2], P)) return;
  const uint32_t id = rc.own[j];
  const float4 T = rc.T[j];
  const float3 L = f3(rc.out[3 * (size_t)j], rc.out[3 * (size_t)j + 1], rc.out[3 * (size_t)j + 2]);
  fb.radiance[id] = pack_rgb9e5(unpack_rgb9e5(fb.radiance[id]) + f3(T.x, T.y, T.z) * L);
}

// ---- denoising -------------------------------------------------------------

// demodulate_radiance.wgsl:24-42
__global__ void k_demodulate(FrameBuffers fb, uint32_t P, uint32_t cur, const uint32_t* in, uint32_t* out,
                             int remodulate) {
  uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= P) return;
  float3 alb = unpack_rgb9e5(fb.gb_b[cur][id].y);
  float3 r = unpack_rgb9e5(in[id]);
  if (remodulate) r = r * alb;
  else r = f3(alb.x > 0.0f ? r.x / alb.x : 0.0f, alb.y > 0.0f ? r.y / alb.y : 0.0f, alb.z > 0.0f ? r.z / alb.z : 0.0f);
  out[id] = pack_rgb9e5(r);
}

// firefly_filter.wgsl:20-85; neighbours come from the unfiltered copy `src`.
__global__ void k_firefly(FrameBuffers fb, uint32_t W, uint32_t H, uint32_t cur, const uint32_t* src, uint32_t* dst) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  uint32_t id = y * W + x;
  const uint4* ga = fb.gb_a[cur];
  if (__uint_as_float(ga[id].w) == 0.0f) return;
  float3 curc = unpack_rgb9e5(src[id]);
  float min_l = dm::F32_MAX, max_l = 0.0f;
  float3 min_c = curc, max_c = f3s(0.0f);
  float cl = luma(curc);
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy) {
      if (dx == 0 && dy == 0) continue;
      int sx = (int)x + dx, sy = (int)y + dy;
      if (sx < 0 || sy < 0 || sx >= (int)W || sy >= (int)H) continue;
      uint32_t sid = (uint32_t)sy * W + (uint32_t)sx;
      if (__uint_as_float(ga[sid].w) == 0.0f) continue;
      float3 nc = unpack_rgb9e5(src[sid]);
      float nl = luma(nc);
      if (nl < min_l) {
        min_l = nl;
        min_c = nc;
      } else if (nl > max_l) {
        max_l = nl;
        max_c = nc;
      }
    }
  float3 rec = cl < min_l ? min_c : (cl > max_l ? max_c : curc);
  if (min_l > max_l) rec = curc;
  dst[id] = pack_rgb9e5(rec);
}

// svgf_temporal.wgsl:87-139.  Besides the packed temporal radiance (kept for
// the reference's buffer ping-pong, which the sky pixels of later frames read)
// it writes the a-trous passes' records: oct30 normal + depth, and packed
// radiance + variance.
// Register-capped for 6 blocks of 256 per SM: its reprojection gathers are
// latency-bound, and the extra resident warps hide more of them than the few
// spilled registers cost.
#ifndef AP_SVGF_MIN_BLOCKS
#define AP_SVGF_MIN_BLOCKS 6
#endif
__global__ void __launch_bounds__(256, AP_SVGF_MIN_BLOCKS) k_svgf_temporal(FrameBuffers fb, Consts c, const uint32_t* demod, uint32_t* out_rad,
                                const float2* in_mom, float2* out_mom, int write_records) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= c.W || y >= c.H) return;
  uint32_t id = y * c.W + x;
  const uint32_t cur = c.frame_idx & 1u;
  const uint4 ga = fb.gb_a[cur][id], gbv = fb.gb_b[cur][id];
  GT g = GT{f3(__uint_as_float(ga.x), __uint_as_float(ga.y), __uint_as_float(ga.z)), __uint_as_float(ga.w),
            unpack_oct30(gbv.x), unpack_rgb9e5(gbv.y)};
  float3 rad = unpack_rgb9e5(demod[id]);
  if (write_records) fb.atr_nd[id] = make_uint2(gbv.x, ga.w);
  if (g.depth == 0.0f) {
    out_rad[id] = pack_rgb9e5(rad);
    return;
  }
  float mx = luma(rad);
  float my = sqr(mx);
  float3 trad = f3s(0.0f);
  float tmx = 0.0f, tmy = 0.0f;
  uint32_t count = 0;
  // the previous point from this pixel's velocity (prev_point's arithmetic on
  // the G-buffer texel already read)
  const float ppx = (float)x - ((float)c.W * __uint_as_float(gbv.z));
  const float ppy = (float)y - ((float)c.H * __uint_as_float(gbv.w));
  if (ppx >= 0.0f && ppy >= 0.0f && ppx <= (float)(c.W - 1) && ppy <= (float)(c.H - 1)) {
    const float2 pp = make_float2(ppx, ppy);
    uint32_t ix = dm::f2u(floorf(pp.x)), iy = dm::f2u(floorf(pp.y));
    float fx = dm::fract(pp.x), fy = dm::fract(pp.y);
    uint32_t x1 = min(ix + 1, c.W - 1), y1 = min(iy + 1, c.H - 1);
    uint32_t i00 = iy * c.W + ix, i10 = iy * c.W + x1, i01 = y1 * c.W + ix, i11 = y1 * c.W + x1;
    // the history taps share the previous G-buffer taps' positions: all of
    // them are read before the validity test, in one round trip
    const uint32_t h00 = fb.svgf_hist[i00], h10 = fb.svgf_hist[i10], h01 = fb.svgf_hist[i01], h11 = fb.svgf_hist[i11];
    const float2 m00 = in_mom[i00], m10 = in_mom[i10], m01 = in_mom[i01], m11 = in_mom[i11];
    const uint32_t prev_count = fb.svgf_count[id];
    GT pg = sample_prev_gbuffer(fb.gb_a[cur ^ 1u], fb.gb_b[cur ^ 1u], c.W, c.H, pp);
    if (history_valid(g, pg)) {
      float3 c0 = mix3(unpack_rgb9e5(h00), unpack_rgb9e5(h10), fx);
      float3 c1 = mix3(unpack_rgb9e5(h01), unpack_rgb9e5(h11), fx);
      trad = mix3(c0, c1, fy);
      float m0x = mixf(m00.x, m10.x, fx), m0y = mixf(m00.y, m10.y, fx);
      float m1x = mixf(m01.x, m11.x, fx), m1y = mixf(m01.y, m11.y, fx);
      tmx = mixf(m0x, m1x, fy);
      tmy = mixf(m0y, m1y, fy);
      count = min(prev_count + 1u, c.cfg.svgf_max_history);
    }
  }
  float alpha = 1.0f / (1.0f + (float)count);
  tmx = mixf(tmx, mx, alpha);
  tmy = mixf(tmy, my, alpha);
  trad = mix3(trad, rad, alpha);
  const float var = dm::fmax(tmy - sqr(tmx), 0.0f);
  const uint32_t packed = pack_rgb9e5(trad);
  out_rad[id] = packed;
  if (write_records) fb.atr_rv[0][id] = make_uint2(packed, __float_as_uint(var));
  out_mom[id] = make_float2(tmx, tmy);
  fb.svgf_count[id] = count;
}

// svgf_atrous.wgsl:48-117, one pass of step STEP.
//
// A block filters a 16x16 lattice of pixels STEP apart (one residue class of a
// (16 STEP)^2 pixel tile), so that every tap of every pixel, at offsets of
// +-STEP and +-2 STEP, falls on the same lattice: the block stages a 20x20
// lattice tile in shared memory, decoding each record once (normal, depth,
// radiance, luma, variance), and the 24 taps read shared memory only, for
// every step.  Pixels outside the image are staged as sky (depth 0), which
// the taps skip as the reference skips both.
//
// Arithmetic: the tap weight, pow(n.n', 128) times the two exponential
// weights times the kernel weight, is one hardware base-2 exponential of
// 128 log2(n.n') (hardware log2) plus the summed exponents in base 2; sums use
// fused multiply-adds.  The result therefore differs from the reference's
// literal expressions in the last bits of the weights; after RGB9E5 packing
// (9-bit mantissas) most pixels are bit-identical and the rest differ by a
// rounding step.
//
// Stores: the next pass's record (packed radiance, variance); pass 0 the
// history radiance of the next frame's temporal pass (svgf_hist); the last
// pass whose output lands in svgf_rad[(frame + 1) % 2] in the reference's
// ping-pong stores it there (sky pixels of the next frame read it); the final
// pass writes the filtered frame, and for sky pixels, which no pass writes in
// the reference, the value the reference's final buffer still holds.
// Hardware base-2 exponential (ex2.approx.ftz.f32).
APD float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr int kAtrousTile = 16;
constexpr int kAtrousSpan = kAtrousTile + 4;
enum : uint32_t { ATR_HIST = 1u, ATR_STATE = 2u, ATR_FINAL = 4u, ATR_NEXT = 8u };
template <int STEP>
__global__ void __launch_bounds__(256) k_atrous(FrameBuffers fb, uint32_t W, uint32_t H, uint32_t flags,
                                                const uint2* in_rv, uint2* out_rv, uint32_t* state_rad,
                                                const uint32_t* final_src, uint32_t* final_dst) {
  __shared__ float4 s_rad[kAtrousSpan * kAtrousSpan];  // radiance, luma
  __shared__ float4 s_nd[kAtrousSpan * kAtrousSpan];   // normal, depth (0: sky or outside)
  __shared__ float s_var[kAtrousSpan * kAtrousSpan];
  const int tiles_x = (int)((W + kAtrousTile * STEP - 1) / (kAtrousTile * STEP));
  (void)tiles_x;
  const int bx = (int)blockIdx.x / STEP, rx = (int)blockIdx.x % STEP;
  const int by = (int)blockIdx.y / STEP, ry = (int)blockIdx.y % STEP;
  const int base_x = bx * kAtrousTile * STEP + rx, base_y = by * kAtrousTile * STEP + ry;
  if (base_x >= (int)W || base_y >= (int)H) return;  // the whole lattice lies outside
  const int tid = threadIdx.y * kAtrousTile + threadIdx.x;
  for (int k = tid; k < kAtrousSpan * kAtrousSpan; k += kAtrousTile * kAtrousTile) {
    const int px = base_x + STEP * (k % kAtrousSpan - 2), py = base_y + STEP * (k / kAtrousSpan - 2);
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f), n = r;
    float v = 0.0f;
    if (px >= 0 && py >= 0 && px < (int)W && py < (int)H) {
      const uint32_t sid = (uint32_t)py * W + (uint32_t)px;
      const uint2 nd = fb.atr_nd[sid];
      n.w = __uint_as_float(nd.y);
      if (n.w != 0.0f) {
        const float3 nn = unpack_oct30(nd.x);
        n.x = nn.x;
        n.y = nn.y;
        n.z = nn.z;
        const uint2 rv = in_rv[sid];
        const float3 rr = unpack_rgb9e5(rv.x);
        r = make_float4(rr.x, rr.y, rr.z, luma(rr));
        v = __uint_as_float(rv.y);
      }
    }
    s_rad[k] = r;
    s_nd[k] = n;
    s_var[k] = v;
  }
  __syncthreads();
  const int x = base_x + STEP * (int)threadIdx.x, y = base_y + STEP * (int)threadIdx.y;
  if (x >= (int)W || y >= (int)H) return;
  const uint32_t id = (uint32_t)y * W + (uint32_t)x;
  const int c = ((int)threadIdx.y + 2) * kAtrousSpan + (int)threadIdx.x + 2;
  const float4 cnd = s_nd[c];
  if (cnd.w == 0.0f) {  // sky: the reference writes nothing for this pixel
    if (flags & ATR_FINAL) final_dst[id] = final_src[id];
    return;
  }
  const float4 crad = s_rad[c];
  float vsum = s_var[c];
  float3 rsum = f3(crad.x, crad.y, crad.z);
  float wsum = 1.0f;
  // exp(-dd^2 / (2 PHI_DEPTH^2)) * exp(-ld / max(PHI_LUMA sqrt(var), 1e-8)),
  // PHI_DEPTH 0.1, PHI_LUMA 4, PHI_NORMAL 128 (svgf_atrous.wgsl:7-9)
  // in base 2: w = 2^(128 log2(d) - |dl| log2(e) / lum - dd^2 log2(e) / (2 PHI_DEPTH^2) + log2(K))
  const float kLog2e = 1.44269504f;
  const float inv_lum2 = kLog2e / fmaxf(4.0f * sqrtf(vsum), 1e-8f);
  const float depth_k2 = kLog2e / (2.0f * 0.1f * 0.1f);
  const float LOG2_KW[3] = {-1.41503751f, -2.0f, -4.0f};  // log2 of 3/8, 1/4, 1/16
#pragma unroll
  for (int dy = -2; dy <= 2; ++dy)
#pragma unroll
    for (int dx = -2; dx <= 2; ++dx) {
      if (dy == 0 && dx == 0) continue;
      const int k = c + dy * kAtrousSpan + dx;
      const float4 snd = s_nd[k];
      const float4 srad = s_rad[k];
      const float svar = s_var[k];
      float d = __fmaf_rn(cnd.x, snd.x, __fmaf_rn(cnd.y, snd.y, __fmul_rn(cnd.z, snd.z)));
      d = fmaxf(d, 0.0f);
      const float dd = cnd.w - snd.w;
      const float lk = LOG2_KW[dx < 0 ? -dx : dx] + LOG2_KW[dy < 0 ? -dy : dy];
      float e = __fmaf_rn(-(dd * dd), depth_k2, lk);
      e = __fmaf_rn(-fabsf(crad.w - srad.w), inv_lum2, e);
      // a sky neighbour or one outside the image is staged with a zero
      // normal and zero radiance and variance: d = 0 gives w = 0 exactly
      const float w = ex2_approx(__fmaf_rn(128.0f, __log2f(d), e));
      rsum.x = __fmaf_rn(srad.x, w, rsum.x);
      rsum.y = __fmaf_rn(srad.y, w, rsum.y);
      rsum.z = __fmaf_rn(srad.z, w, rsum.z);
      vsum = __fmaf_rn(svar, w * w, vsum);
      wsum += w;
    }
  const float inv_w = 1.0f / wsum;
  rsum = rsum * inv_w;
  vsum = vsum * (inv_w * inv_w);
  const uint32_t packed = pack_rgb9e5(rsum);
  if (flags & ATR_NEXT) out_rv[id] = make_uint2(packed, __float_as_uint(vsum));
  if (flags & ATR_HIST) fb.svgf_hist[id] = packed;
  if (flags & ATR_STATE) state_rad[id] = packed;
  if (flags & ATR_FINAL) final_dst[id] = packed;
}

// taa.wgsl:67-171.  A 16x16 block stages the 18x18 neighbourhood of the
// pre-TAA frame `src` in shared memory (unpacked once, clamped at zero, with
// the filter's 1 / (1 + luma)); the 3x3 filter and the colour-box statistics
// read it from there.
// Weights and the history clip use hardware division and square root.  Sky
// pixels keep `src`'s value (the reference leaves them untouched).
APD float mitchell(float x_, float B, float C) {
  float x = dm::fabs_(2.0f * x_);
  float ods = 1.0f / 6.0f;
  if (x > 1.0f)
    return ((-B - 6.0f * C) * x * x * x + (6.0f * B + 30.0f * C) * x * x + (-12.0f * B - 48.0f * C) * x +
            (8.0f * B + 24.0f * C)) * ods;
  return ((12.0f - 9.0f * B - 6.0f * C) * x * x * x + (-18.0f + 12.0f * B + 6.0f * C) * x * x + (6.0f - 2.0f * B)) *
         ods;
}
constexpr int kTaaTile = 16;
constexpr int kTaaSpan = kTaaTile + 2;
__global__ void __launch_bounds__(256) k_taa(FrameBuffers fb, Consts c, const uint32_t* src, uint32_t* dst,
                                             const uint32_t* prevb) {
  __shared__ float4 s_c[kTaaSpan * kTaaSpan];  // max(colour, 0), 1 / (1 + luma); w < 0 outside the image
  const int x0 = blockIdx.x * kTaaTile, y0 = blockIdx.y * kTaaTile;
  const int tid = threadIdx.y * kTaaTile + threadIdx.x;
  const uint32_t x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  const bool in_image = x < c.W && y < c.H;
  const uint32_t id = in_image ? y * c.W + x : 0u;
  const uint32_t cur = c.frame_idx & 1u;
  // This pixel's depth, colour and velocity, then its history taps and the
  // previous depth, are read before the neighbourhood is staged, so that their
  // round trips overlap the staging loads.
  float cdepth = 0.0f;
  uint32_t csrc = 0u, hp[4] = {0u, 0u, 0u, 0u}, pid = id;
  float tx = 0.0f, ty = 0.0f, pdepth = 0.0f;
  bool bilinear = false;
  if (in_image) {
    cdepth = __uint_as_float(fb.gb_a[cur][id].w);
    csrc = src[id];
    float2 pp;
    bilinear = prev_point(fb, cur, x, y, c.W, c.H, &pp);
    if (cdepth != 0.0f) {
      if (bilinear) {
        uint32_t fx = dm::f2u(floorf(pp.x)), fy = dm::f2u(floorf(pp.y));
        uint32_t cxp = dm::f2u(ceilf(pp.x)), cyp = dm::f2u(ceilf(pp.y));
        pid = fy * c.W + fx;
        hp[0] = prevb[min(fy, c.H - 1) * c.W + min(fx, c.W - 1)];
        hp[1] = prevb[min(cyp, c.H - 1) * c.W + min(fx, c.W - 1)];
        hp[2] = prevb[min(fy, c.H - 1) * c.W + min(cxp, c.W - 1)];
        hp[3] = prevb[min(cyp, c.H - 1) * c.W + min(cxp, c.W - 1)];
        tx = dm::fract(pp.x);
        ty = dm::fract(pp.y);
      } else {
        hp[0] = prevb[id];
      }
      pdepth = __uint_as_float(fb.gb_a[cur ^ 1u][pid].w);
    }
  }
  for (int k = tid; k < kTaaSpan * kTaaSpan; k += kTaaTile * kTaaTile) {
    const int px = x0 + k % kTaaSpan - 1, py = y0 + k / kTaaSpan - 1;
    float4 v = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    if (px >= 0 && py >= 0 && px < (int)c.W && py < (int)c.H) {
      const float3 sc = vmax(unpack_rgb9e5(src[(uint32_t)py * c.W + (uint32_t)px]), f3s(0.0f));
      v = make_float4(sc.x, sc.y, sc.z, __frcp_rn(1.0f + luma(sc)));
    }
    s_c[k] = v;
  }
  __syncthreads();
  if (!in_image) return;
  if (cdepth == 0.0f) {
    dst[id] = csrc;
    return;
  }
  const float3 curc = unpack_rgb9e5(csrc);
  float wsum = sqr(mitchell(0.0f, 0.33f, 0.33f));
  float3 rec = curc * wsum;
  float3 m1 = curc, m2 = curc * curc;
  float cnt = 1.0f;
  const int cs = ((int)threadIdx.y + 1) * kTaaSpan + (int)threadIdx.x + 1;
#pragma unroll
  for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
      if (dx == 0 && dy == 0) continue;
      const float4 v = s_c[cs + dy * kTaaSpan + dx];
      if (v.w < 0.0f) continue;
      const float3 sc = f3(v.x, v.y, v.z);
      const float w = (mitchell((float)dx, 0.33f, 0.33f) * mitchell((float)dy, 0.33f, 0.33f)) * v.w;
      rec = rec + sc * w;
      wsum = wsum + w;
      m1 = m1 + sc;
      m2 = m2 + sc * sc;
      cnt = cnt + 1.0f;
    }
  rec = rec * __frcp_rn(fmaxf(wsum, 1e-5f));
  float3 hist;
  if (bilinear) {
    float3 h00 = unpack_rgb9e5(hp[0]), h10 = unpack_rgb9e5(hp[1]);
    float3 h01 = unpack_rgb9e5(hp[2]), h11 = unpack_rgb9e5(hp[3]);
    float3 a = h00 * (1.0f - tx) + h10 * tx;
    float3 b = h01 * (1.0f - tx) + h11 * tx;
    hist = a * (1.0f - ty) + b * ty;
  } else {
    hist = unpack_rgb9e5(hp[0]);
  }
  float cdcs = depth_cs(cdepth, 0.001f, 10000.0f), pdcs = depth_cs(pdepth, 0.001f, 10000.0f);
  bool vdd = (dm::fabs_(cdcs - pdcs) / cdcs) < 0.1f;
  const float inv_cnt = __frcp_rn(cnt);
  float3 mean = m1 * inv_cnt;
  float3 sd = vabs(m2 - (m1 * m1) * inv_cnt);
  sd = sd * __frcp_rn(cnt - 1.0f);
  sd = f3(sqrtf(sd.x), sqrtf(sd.y), sqrtf(sd.z));
  float3 lo = mean - sd, hi = mean + sd;
  float3 center = 0.5f * (hi + lo);
  float3 ext = 0.5f * (hi - lo);
  float3 rtc = hist - center;
  float3 rtcu = vabs(f3(__fdividef(rtc.x, ext.x), __fdividef(rtc.y, ext.y), __fdividef(rtc.z, ext.z)));
  float mxv = dm::fmax(rtcu.x, dm::fmax(rtcu.y, rtcu.z));
  float3 clipped = mxv > 1.0f ? center + rtc * __frcp_rn(mxv) : hist;
  float blend = 1.0f - (c.cfg.taa_history_influence * (vdd ? 1.0f : 0.0f));
  float cw = dm::saturate(blend * __frcp_rn(1.0f + luma(rec)));
  float hw = dm::saturate((1.0f - blend) * __frcp_rn(1.0f + luma(clipped)));
  rec = (cw * rec + hw * clipped) * __frcp_rn(cw + hw);
  dst[id] = pack_rgb9e5(rec);
}

// resolve.wgsl:48-49 (before the tonemap): linear HDR = radiance / sample_count.
__global__ void k_resolve(FrameBuffers fb, uint32_t P, float inv_count_den) {
  uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= P) return;
  float3 r = unpack_rgb9e5(fb.radiance[id]);
  r = r / inv_count_den;
  fb.out_rgb[3 * id + 0] = r.x;
  fb.out_rgb[3 * id + 1] = r.y;
  fb.out_rgb[3 * id + 2] = r.z;
}

// resolve.wgsl:29-38 (hdr_to_sdr, the ACES fit)
APD float3 hdr_to_sdr(float3 hdr) {
  const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  float3 sdr = (hdr * (a * hdr + f3s(b))) / (hdr * (c * hdr + f3s(d)) + f3s(e));
  return f3(dm::fmin(dm::fmax(sdr.x, 0.0f), 1.0f), dm::fmin(dm::fmax(sdr.y, 0.0f), 1.0f),
            dm::fmin(dm::fmax(sdr.z, 0.0f), 1.0f));
}

// block.wgsl:3-16: texture position of pixel (x, y) in 64x64 blocks.
APD uint2 linear_to_block_pixel(uint32_t x, uint32_t y, uint32_t width) {
  const uint32_t B = 64;
  uint32_t blocks_per_row = (width + B - 1) / B;
  uint32_t block_index = (y / B) * blocks_per_row + x / B;
  uint32_t pixel_index = block_index * (B * B) + (y % B) * B + x % B;
  return make_uint2(pixel_index % width, pixel_index / width);
}

APD uint32_t unorm8(float v) { return __float2uint_rn(v * 255.0f); }  // v in [0, 1]

// resolve.wgsl:40-59
__global__ void k_resolve_rgba8(FrameBuffers fb, uint32_t W, uint32_t H, uint32_t spp, uint32_t accum_count) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  uint32_t i = y * W + x;
  float3 r = unpack_rgb9e5(fb.radiance[i]);
  r = r / (float)spp;
  r = hdr_to_sdr(r);
  float4 acc = fb.accum[i];
  float3 a = f3(acc.x, acc.y, acc.z) + r;
  fb.accum[i] = make_float4(a.x, a.y, a.z, 0.0f);
  uint2 p = linear_to_block_pixel(x, y, W);
  if (p.x >= W || p.y >= H) return;  // outside the texture: the store is dropped
  float3 o = a / (float)(accum_count + 1);
  fb.rgba[p.y * W + p.x] = unorm8(o.x) | (unorm8(o.y) << 8) | (unorm8(o.z) << 16) | (255u << 24);
}

// Batch traversal for the ray-query entry points (persistent, per-lane refill).
template <bool kAny>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_batch(DevScene s, const float4* origins, const float4* dirs,
                                                        uint32_t n, uint4* out, uint32_t* cursor) {
  persistent_trace<kAny, false>(
      s, n, cursor,
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const float4 a = origins[i], b = dirs[i];
        o = f3(a.x, a.y, a.z);
        d = f3(b.x, b.y, b.z);
        tmax = a.w;
      },
      [&](uint32_t i, const Trav& t, const Visits&) {
        if (kAny) out[i] = make_uint4(t.hit.tri != kNoHit ? 1u : 0u, 0u, 0u, 0u);
        else out[i] = make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
      });
}

// The same batch over a two-level scene (traverse2.cuh).
template <bool kAny>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_trace_batch2(DevScene s, TwoLevel tl,
                                                                         const float4* origins, const float4* dirs,
                                                                         uint32_t n, uint4* out, uint32_t* cursor) {
  persistent_trace2<kAny, false>(
      s, tl, n, cursor,
      [&](uint32_t i, float3& o, float3& d, float& tmax) {
        const float4 a = origins[i], b = dirs[i];
        o = f3(a.x, a.y, a.z);
        d = f3(b.x, b.y, b.z);
        tmax = a.w;
      },
      [&](uint32_t i, const Trav& t, const Visits&) {
        if (kAny) out[i] = make_uint4(t.hit.tri != kNoHit ? 1u : 0u, 0u, 0u, 0u);
        else out[i] = make_uint4(__float_as_uint(t.hit.t), __float_as_uint(t.hit.u), __float_as_uint(t.hit.v), t.hit.tri);
      });
}

template <typename T>
T* carve(char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += ((count * sizeof(T) + 255) / 256) * 256;
  return r;
}

}  // namespace

size_t frame_buffer_bytes(uint32_t W, uint32_t H) {
  FrameBuffers fb;
  char* p = nullptr;
  size_t P = (size_t)W * H;
  (void)fb;
  size_t n = 0;
  auto add = [&](size_t bytes) { n += ((bytes + 255) / 256) * 256; };
  add(P * 16);  // rays
  add(P * 16);  // payload
  add(P * 4);   // radiance
  add(P * 16);  // hits
  for (int i = 0; i < 6; ++i) add(P * 16);  // di a,b inter a,b prev a,b[0]
  add(P * 16); add(P * 16);                 // di prev [1] a,b
  add(P * 16);                              // ctx
  for (int i = 0; i < 6; ++i) add(P * 16);  // gi
  add(P * 16); add(P * 16);
  for (int i = 0; i < 4; ++i) add(P * 16);  // gbuffer
  add(P * 4); add(P * 4);                   // demod
  add(P * 4); add(P * 4);                   // svgf rad
  add(P * 8); add(P * 8);                   // moments
  add(P * 4); add(P * 4);                   // count, hist
  add(P * 4);                               // snapshot
  add(P * 4); add(P * 4);                   // queues
  for (int i = 0; i < 10; ++i) add(P * 16);  // ray queues (origin, direction) x 5
  add(P * 16); add(P * 16);                 // hit_bsdf, hit_gi
  for (int i = 0; i < 5; ++i) add(P);       // visibility
  for (int i = 0; i < 5; ++i) add(P * 16);  // stage state
  add(64 * 4);                              // counters
  add(3 * K_NUM_KINDS * 8);                 // visit counters
  add(P * 12);                              // out rgb
  add(P * 16);                              // display accumulation
  add(P * 4);                               // RGBA8 texture
  (void)p;
  return n;
}

void frame_buffers_carve(void* base, uint32_t W, uint32_t H, FrameBuffers* fb) {
  char* p = static_cast<char*>(base);
  size_t P = (size_t)W * H;
  fb->rays = carve<float4>(p, P);
  fb->payload = carve<uint4>(p, P);
  fb->radiance = carve<uint32_t>(p, P);
  fb->hits = carve<uint4>(p, P);
  fb->di_a = carve<uint4>(p, P);
  fb->di_b = carve<uint4>(p, P);
  fb->di_inter_a = carve<uint4>(p, P);
  fb->di_inter_b = carve<uint4>(p, P);
  fb->di_prev_a[0] = carve<uint4>(p, P);
  fb->di_prev_b[0] = carve<uint4>(p, P);
  fb->di_prev_a[1] = carve<uint4>(p, P);
  fb->di_prev_b[1] = carve<uint4>(p, P);
  fb->ctx = carve<uint4>(p, P);
  fb->gi_a = carve<uint4>(p, P);
  fb->gi_b = carve<uint4>(p, P);
  fb->gi_inter_a = carve<uint4>(p, P);
  fb->gi_inter_b = carve<uint4>(p, P);
  fb->gi_prev_a[0] = carve<uint4>(p, P);
  fb->gi_prev_b[0] = carve<uint4>(p, P);
  fb->gi_prev_a[1] = carve<uint4>(p, P);
  fb->gi_prev_b[1] = carve<uint4>(p, P);
  fb->gb_a[0] = carve<uint4>(p, P);
  fb->gb_b[0] = carve<uint4>(p, P);
  fb->gb_a[1] = carve<uint4>(p, P);
  fb->gb_b[1] = carve<uint4>(p, P);
  fb->demod[0] = carve<uint32_t>(p, P);
  fb->demod[1] = carve<uint32_t>(p, P);
  fb->svgf_rad[0] = carve<uint32_t>(p, P);
  fb->svgf_rad[1] = carve<uint32_t>(p, P);
  fb->svgf_mom[0] = carve<float2>(p, P);
  fb->svgf_mom[1] = carve<float2>(p, P);
  fb->svgf_count = carve<uint32_t>(p, P);
  fb->svgf_hist = carve<uint32_t>(p, P);
  fb->snapshot = carve<uint32_t>(p, P);
  fb->queue[0] = carve<uint32_t>(p, P);
  fb->queue[1] = carve<uint32_t>(p, P);
  for (int q = 0; q < 5; ++q) {
    fb->rq_o[q] = carve<float4>(p, P);
    fb->rq_d[q] = carve<float4>(p, P);
  }
  fb->hit_bsdf = carve<uint4>(p, P);
  fb->hit_gi = carve<uint4>(p, P);
  for (int q = 0; q < 5; ++q) fb->vis[q] = carve<uint8_t>(p, P);
  fb->st_a = carve<uint4>(p, P);
  fb->st_b = carve<uint4>(p, P);
  fb->st_c = carve<uint4>(p, P);
  fb->st_d = carve<uint4>(p, P);
  fb->st_e = carve<uint4>(p, P);
  fb->counters = carve<uint32_t>(p, 64);
  fb->visits = carve<unsigned long long>(p, 3 * K_NUM_KINDS);
  fb->atr_nd = reinterpret_cast<uint2*>(fb->rq_o[0]);
  fb->atr_rv[0] = reinterpret_cast<uint2*>(fb->rq_d[0]);
  fb->atr_rv[1] = reinterpret_cast<uint2*>(fb->rq_o[1]);
  fb->out_rgb = carve<float>(p, 3 * P);
  fb->accum = carve<float4>(p, P);
  fb->rgba = carve<uint32_t>(p, P);
}

size_t rc_frame_bytes(uint32_t W, uint32_t H, uint32_t stride, uint32_t batch) {
  const size_t P = (size_t)W * H, slots = ((P + stride - 1) / stride) * kRcMaxBounces;
  auto a = [](size_t b) { return ((b + 255) / 256) * 256; };
  return a(P * 64) + a(P * 16) + a(P * 4) + a(P * 12) + a(slots * 96) + a((size_t)batch * 64) + a((size_t)batch * 12) +
         a(12) + a(4 * ((slots + 255) / 256));
}

void rc_frame_carve(void* base, uint32_t W, uint32_t H, uint32_t stride, uint32_t batch, RcFrame* rc) {
  char* p = static_cast<char*>(base);
  const size_t P = (size_t)W * H, slots = ((P + stride - 1) / stride) * kRcMaxBounces;
  rc->q = carve<float4>(p, 4 * P);
  rc->T = carve<float4>(p, P);
  rc->own = carve<uint32_t>(p, P);
  rc->out = carve<float>(p, 3 * P);
  rc->rec = carve<float4>(p, 6 * slots);
  rc->bq = carve<float4>(p, 4 * (size_t)batch);
  rc->bt = carve<float>(p, 3 * (size_t)batch);
  rc->counts = carve<uint32_t>(p, 3);
  rc->bcount = carve<uint32_t>(p, (slots + 255) / 256);
}

__global__ void __launch_bounds__(1024) k_count_scan(uint32_t* c, uint32_t n, uint32_t* total, uint32_t cap) {
  __shared__ uint32_t s[1024];
  const uint32_t t = threadIdx.x, per = (n + 1023u) / 1024u;
  const uint32_t b0 = min(t * per, n), b1 = min(b0 + per, n);
  uint32_t sum = 0;
  for (uint32_t i = b0; i < b1; ++i) sum += c[i];
  s[t] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < 1024u; off <<= 1) {  // inclusive scan of the per-thread sums
    const uint32_t v = t >= off ? s[t - off] : 0u;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  uint32_t run = t ? s[t - 1] : 0u;
  for (uint32_t i = b0; i < b1; ++i) {
    const uint32_t v = c[i];
    c[i] = run;
    run += v;
  }
  if (t == 1023u) *total = min(s[1023], cap);
}

void count_scan(uint32_t* counts, uint32_t n, uint32_t* total, uint32_t cap, cudaStream_t st) {
  k_count_scan<<<1, 1024, 0, st>>>(counts, n, total, cap);
}

const char* kernel_kind_name(int k) {
  static const char* names[K_NUM_KINDS] = {"memset", "raygen", "extend", "shade", "di_temporal", "di_spatial",
                                           "gi_temporal", "gi_spatial", "apply_di", "apply_gi", "demodulate",
                                           "firefly", "svgf_temporal", "atrous", "taa", "resolve", "copy",
                                           "trace_closest", "trace_any", "shade_b", "shade_c", "shade_d", "shade_b2", "rc",
                                           "rc_infer", "rc_train", "atrous_prep"};
  return (k >= 0 && k < K_NUM_KINDS) ? names[k] : "?";
}

template <bool kAny>
void trace_queue(bool counting, int blocks, cudaStream_t st, const DevScene& scene, const FrameBuffers& fb, int q,
                 uint32_t cap, uint4* hits, uint8_t* vis) {
  if (counting) k_trace_queue<kAny, true><<<blocks, kBlock, 0, st>>>(scene, fb, q, cap, hits, vis);
  else k_trace_queue<kAny, false><<<blocks, kBlock, 0, st>>>(scene, fb, q, cap, hits, vis);
}

// The RIS shadow queue and the GI shadow queue, traced by one any-hit launch.
void trace_shadow_pair(bool counting, int blocks, cudaStream_t st, const DevScene& scene, const FrameBuffers& fb,
                       uint32_t cap) {
  if (counting) k_trace_pair<Q_RIS_SHADOW, Q_GI_SHADOW, true><<<blocks, kBlock, 0, st>>>(scene, fb, cap);
  else k_trace_pair<Q_RIS_SHADOW, Q_GI_SHADOW, false><<<blocks, kBlock, 0, st>>>(scene, fb, cap);
}

// The two closest-hit candidate queues (BSDF, GI) in one launch.
void trace_candidate_pair(bool counting, int blocks, cudaStream_t st, const DevScene& scene, const FrameBuffers& fb,
                          uint32_t cap) {
  if (counting)
    k_trace_pair_closest<Q_BSDF_CAND, Q_GI_CAND, true><<<blocks, kBlock, 0, st>>>(scene, fb, cap, fb.hit_bsdf, fb.hit_gi);
  else
    k_trace_pair_closest<Q_BSDF_CAND, Q_GI_CAND, false><<<blocks, kBlock, 0, st>>>(scene, fb, cap, fb.hit_bsdf, fb.hit_gi);
}

int frame_streams_create(FrameStreams* fs) {
  cudaError_t e = cudaStreamCreateWithFlags(&fs->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&fs->side2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&fs->side3, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fs->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fs->join, cudaEventDisableTiming);
  if (e != cudaSuccess) frame_streams_destroy(fs);
  return (int)e;
}

void frame_streams_destroy(FrameStreams* fs) {
  if (fs->side) cudaStreamSynchronize(fs->side);
  if (fs->side2) cudaStreamSynchronize(fs->side2);
  if (fs->side3) cudaStreamSynchronize(fs->side3);
  if (fs->fork) cudaEventDestroy(fs->fork);
  if (fs->join) cudaEventDestroy(fs->join);
  if (fs->side) cudaStreamDestroy(fs->side);
  if (fs->side2) cudaStreamDestroy(fs->side2);
  if (fs->side3) cudaStreamDestroy(fs->side3);
  *fs = FrameStreams();
}

int encode_frame(const DevScene& scene, const FrameBuffers& fb, const FrameConfig& cfg, const Mats& mats,
                 uint32_t W, uint32_t H, uint32_t frame_idx, int num_sms, cudaStream_t st, FrameProfiler* prof,
                 const RcFrame* rc, const FrameStreams* fs) {
  int launches = 0;
  const bool overlap = fs && fs->side && fs->fork && fs->join && !prof;
  bool di_pending = false;  // a DI shadow pass in flight on fs->side; k_apply_di_b waits for it
  Consts di_c{};
  const bool counting = prof && prof->count_visits;
  if (counting) cudaMemsetAsync(fb.visits, 0, 3 * K_NUM_KINDS * sizeof(unsigned long long), st);
  if (prof) {
    prof->n = 0;
    cudaEventRecord(prof->ev[0], st);
  }
  auto mark = [&](int kind) {
    if (kind != K_MEMSET && kind != K_COPY) ++launches;
    if (prof && prof->n < FrameProfiler::kMax) {
      prof->kind[prof->n] = kind;
      cudaEventRecord(prof->ev[prof->n + 1], st);
      prof->n += 1;
    }
  };
  const uint32_t P = W * H;
  const uint32_t cur = frame_idx & 1u;
  dim3 b2(16, 16), g2((W + 15) / 16, (H + 15) / 16);
  const int persistent_blocks = num_sms * kTraceMinBlocks;
  const int linear_blocks = (int)std::min<uint32_t>((P + kBlock - 1) / kBlock, (uint32_t)num_sms * 16u);
  Consts c;
  c.W = W;
  c.H = H;
  c.P = P;
  c.frame_idx = frame_idx;
  c.sample = 0;
  c.cfg = cfg;
  cudaMemsetAsync(fb.radiance, 0, (size_t)P * 4, st);
  cudaMemsetAsync(fb.counters + 3, 0, 4, st);
  mark(K_MEMSET);
  const bool cache = rc && rc->cache && cfg.max_bounces > rc->prefix;
  const uint32_t rc_slots = cache ? ((P + rc->stride - 1) / rc->stride) * kRcMaxBounces : 0;
  if (cache) {
    cudaMemsetAsync(rc->rec, 0, (size_t)rc_slots * 6 * sizeof(float4), st);
    cudaMemsetAsync(rc->counts, 0, 3 * sizeof(uint32_t), st);
    mark(K_MEMSET);
  }
  for (uint32_t sample = 0; sample < cfg.sample_count; ++sample) {
    c.seed = frame_idx * cfg.sample_count + sample;
    c.sample = sample;
    if (cache) {
      cudaMemsetAsync(rc->counts + 2, 0, sizeof(uint32_t), st);  // retired paths of this sample
      mark(K_MEMSET);
    }
    k_raygen<<<g2, b2, 0, st>>>(fb, W, H, mats);
    mark(K_RAYGEN);
    for (uint32_t i = 0; i < cfg.max_bounces; ++i) {
      c.bounce = i;
      c.qin = i & 1u;
      c.qout = (i + 1) & 1u;
      cudaMemsetAsync(fb.counters + 2, 0, 4, st);
      mark(K_MEMSET);
      if (counting) k_extend<true><<<persistent_blocks, kBlock, 0, st>>>(scene, fb, c);
      else k_extend<false><<<persistent_blocks, kBlock, 0, st>>>(scene, fb, c);
      mark(K_EXTEND);
      if (di_pending) {  // the previous bounce's DI shadow rays, traced beside this extension
        cudaEventRecord(fs->join, fs->side);
        cudaStreamWaitEvent(st, fs->join, 0);
        k_apply_di_b<<<linear_blocks, kBlock, 0, st>>>(fb, di_c);
        mark(K_APPLY_DI);
        di_pending = false;
      }
      if (cache) {
        k_rc_vertex<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c, *rc);
        mark(K_RC);
      }
      cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
      mark(K_MEMSET);
      k_shade_a<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c, mats);
      mark(K_SHADE);
      trace_queue<false>(counting, persistent_blocks, st, scene, fb, Q_BSDF_CAND, P, fb.hit_bsdf, nullptr);
      mark(K_TRACE_CLOSEST);
      k_shade_b<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c);
      mark(K_SHADE_B);
      k_shade_b2<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c);
      mark(K_SHADE_B2);
      trace_queue<false>(counting, persistent_blocks, st, scene, fb, Q_GI_CAND, P, fb.hit_gi, nullptr);
      mark(K_TRACE_CLOSEST);
      k_shade_c<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c);
      mark(K_SHADE_C);
      // the RIS shadow rays (queued by k_shade_b, read by k_shade_d) with the GI shadow rays
      trace_shadow_pair(counting, persistent_blocks, st, scene, fb, P);
      mark(K_TRACE_ANY);
      k_shade_d<<<linear_blocks, kBlock, 0, st>>>(fb, c);
      mark(K_SHADE_D);
      if (i == 0) {
        if (cfg.restir_di) {
          uint4* pin_a = fb.di_prev_a[cur];
          uint4* pin_b = fb.di_prev_b[cur];
          uint4* pout_a = fb.di_prev_a[cur ^ 1u];
          uint4* pout_b = fb.di_prev_b[cur ^ 1u];
          cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
          mark(K_MEMSET);
          k_dt_a<<<g2, b2, 0, st>>>(scene, fb, c, pin_a, pin_b);
          mark(K_DI_TEMPORAL);
          trace_queue<true>(counting, persistent_blocks, st, scene, fb, Q_DI_SHADOW, P, nullptr, fb.vis[Q_DI_SHADOW]);
          mark(K_TRACE_ANY);
          k_dt_b<<<g2, b2, 0, st>>>(fb, c, fb.di_a, fb.di_b, fb.di_inter_a, fb.di_inter_b, pin_a, pin_b, pout_a,
                                    pout_b);
          mark(K_DI_TEMPORAL);
          uint32_t n = cfg.di_spatial_passes;
          for (uint32_t k = 0; k < n; ++k) {
            bool odd = (k % 2) != 0;
            const uint4* in_a = odd ? fb.di_a : fb.di_inter_a;
            const uint4* in_b = odd ? fb.di_b : fb.di_inter_b;
            uint4* out_a = odd ? fb.di_inter_a : fb.di_a;
            uint4* out_b = odd ? fb.di_inter_b : fb.di_b;
            if (!cfg.di_unbiased) {
              k_spatial<false><<<g2, b2, 0, st>>>(scene, fb, c, k, n, cfg.di_spatial_samples, 0u, in_a, in_b, out_a,
                                                  out_b, pout_a, pout_b);
              mark(K_DI_SPATIAL);
              continue;
            }
            // unbiased: wavefront stages, shadow rays through the any-hit queues
            const uint32_t ns = cfg.di_spatial_samples;
            for (uint32_t j = 0; j <= ns; ++j) {
              cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
              mark(K_MEMSET);
              k_dsp_ca<<<g2, b2, 0, st>>>(scene, fb, c, k, n, ns, j, in_a, in_b, out_a, out_b, pout_a, pout_b);
              mark(K_DI_SPATIAL);
              if (j == ns) break;
              trace_queue<true>(counting, persistent_blocks, st, scene, fb, Q_DI_SHADOW, P, nullptr, fb.vis[Q_DI_SHADOW]);
              mark(K_TRACE_ANY);
              k_dsp_b<<<g2, b2, 0, st>>>(scene, fb, c, k, n, in_a, in_b, out_a, out_b);
              mark(K_DI_SPATIAL);
              trace_shadow_pair(counting, persistent_blocks, st, scene, fb, P);
              mark(K_TRACE_ANY);
            }
          }
          if (n % 2 == 0) {
            cudaMemcpyAsync(fb.di_a, fb.di_inter_a, (size_t)P * 16, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(fb.di_b, fb.di_inter_b, (size_t)P * 16, cudaMemcpyDeviceToDevice, st);
            mark(K_COPY);
          }
        }
        if (cfg.restir_gi) {
          uint4* pin_a = fb.gi_prev_a[cur];
          uint4* pin_b = fb.gi_prev_b[cur];
          uint4* pout_a = fb.gi_prev_a[cur ^ 1u];
          uint4* pout_b = fb.gi_prev_b[cur ^ 1u];
          cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
          mark(K_MEMSET);
          k_gt_a<<<g2, b2, 0, st>>>(scene, fb, c, pin_a, pin_b);
          mark(K_GI_TEMPORAL);
          trace_queue<false>(counting, persistent_blocks, st, scene, fb, Q_GI_CAND, P, fb.hit_gi, nullptr);
          mark(K_TRACE_CLOSEST);
          k_gt_b<<<g2, b2, 0, st>>>(scene, fb, c, pin_a, pin_b);
          mark(K_GI_TEMPORAL);
          trace_queue<true>(counting, persistent_blocks, st, scene, fb, Q_GI_SHADOW, P, nullptr, fb.vis[Q_GI_SHADOW]);
          mark(K_TRACE_ANY);
          k_gt_c<<<g2, b2, 0, st>>>(fb, c, fb.gi_a, fb.gi_b, fb.gi_inter_a, fb.gi_inter_b, pin_a, pin_b, pout_a,
                                    pout_b);
          mark(K_GI_TEMPORAL);
          uint32_t n = cfg.gi_spatial_passes;
          if (n == 0) {
            cudaMemcpyAsync(fb.gi_a, fb.gi_inter_a, (size_t)P * 16, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(fb.gi_b, fb.gi_inter_b, (size_t)P * 16, cudaMemcpyDeviceToDevice, st);
            mark(K_COPY);
          }
          for (uint32_t k = 0; k < n; ++k) {
            bool odd = (k % 2) != 0;
            const uint4* in_a = odd ? fb.gi_a : fb.gi_inter_a;
            const uint4* in_b = odd ? fb.gi_b : fb.gi_inter_b;
            uint4* out_a = odd ? fb.gi_inter_a : fb.gi_a;
            uint4* out_b = odd ? fb.gi_inter_b : fb.gi_b;
            if (!cfg.gi_unbiased) {
              k_spatial<true><<<g2, b2, 0, st>>>(scene, fb, c, k, n, cfg.gi_spatial_samples, 0u, in_a, in_b, out_a,
                                                 out_b, pout_a, pout_b);
              mark(K_GI_SPATIAL);
              continue;
            }
            // unbiased: wavefront stages, the targets' re-traces through the queues
            const uint32_t ns = cfg.gi_spatial_samples;
            for (uint32_t j = 0; j <= ns; ++j) {
              cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
              mark(K_MEMSET);
              k_gsp_a<<<g2, b2, 0, st>>>(scene, fb, c, k, n, ns, j, in_a, in_b, out_a, out_b, pout_a, pout_b);
              mark(K_GI_SPATIAL);
              if (j == ns) break;
              trace_queue<false>(counting, persistent_blocks, st, scene, fb, Q_GI_CAND, P, fb.hit_gi, nullptr);
              mark(K_TRACE_CLOSEST);
              k_gsp_b<<<g2, b2, 0, st>>>(scene, fb, c, in_a, in_b);
              mark(K_GI_SPATIAL);
              trace_queue<true>(counting, persistent_blocks, st, scene, fb, Q_GI_SHADOW, P, nullptr, fb.vis[Q_GI_SHADOW]);
              mark(K_TRACE_ANY);
              cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
              mark(K_MEMSET);
              k_gsp_c<<<g2, b2, 0, st>>>(scene, fb, c, k, n, in_a, in_b, out_a, out_b);
              mark(K_GI_SPATIAL);
              trace_candidate_pair(counting, persistent_blocks, st, scene, fb, P);
              mark(K_TRACE_CLOSEST);
              cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
              mark(K_MEMSET);
              k_gsp_d<<<g2, b2, 0, st>>>(scene, fb, c, out_a, out_b);
              mark(K_GI_SPATIAL);
              trace_shadow_pair(counting, persistent_blocks, st, scene, fb, P);
              mark(K_TRACE_ANY);
            }
          }
          if (n > 0 && n % 2 == 0) {
            cudaMemcpyAsync(fb.gi_a, fb.gi_inter_a, (size_t)P * 16, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(fb.gi_b, fb.gi_inter_b, (size_t)P * 16, cudaMemcpyDeviceToDevice, st);
            mark(K_COPY);
          }
        }
      }
      if (i == 0 && (cfg.restir_di || cfg.restir_gi)) {
        // the resampling passes used the ray queues: start the DI shadow queue empty
        cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
        mark(K_MEMSET);
      }
      k_apply_di_a<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c);
      mark(K_APPLY_DI);
      if (overlap && i + 1 < cfg.max_bounces) {
        // nothing before the next extension reads these rays' results (k_apply_di_b
        // follows it, still before the next bounce adds to the radiance)
        cudaEventRecord(fs->fork, st);
        cudaStreamWaitEvent(fs->side, fs->fork, 0);
        trace_queue<true>(false, persistent_blocks, fs->side, scene, fb, Q_DI_SHADOW, P, nullptr,
                          fb.vis[Q_DI_SHADOW]);
        mark(K_TRACE_ANY);
        di_pending = true;
        di_c = c;
      } else {
        trace_queue<true>(counting, persistent_blocks, st, scene, fb, Q_DI_SHADOW, P, nullptr, fb.vis[Q_DI_SHADOW]);
        mark(K_TRACE_ANY);
        k_apply_di_b<<<linear_blocks, kBlock, 0, st>>>(fb, c);
        mark(K_APPLY_DI);
      }
      if (i + 1 < cfg.max_bounces) {
        cudaMemsetAsync(fb.counters + c.qout, 0, 4, st);
        mark(K_MEMSET);
        k_apply_gi<<<linear_blocks, kBlock, 0, st>>>(scene, fb, c);
        mark(K_APPLY_GI);
      }
    }
    if (cache) {  // this sample's retired paths: predicted radiance on the tensor cores
      rc_infer_device(rc->cache, rc->q, P, rc->out, st, rc->counts + 2);  // the retired queries only
      mark(K_RC_INFER);
      k_rc_apply<<<(P + 255) / 256, 256, 0, st>>>(fb, *rc, P);
      mark(K_RC);
    }
  }
  if (cache && rc->train) {
    // training targets of the last sample's suffix vertices (the radiance of
    // the training pixels is final here), one Adam step
    const float last_tag = (float)cfg.sample_count;
    const uint32_t nb = (rc_slots + 255) / 256;
    k_rc_count<<<nb, 256, 0, st>>>(*rc, rc_slots, last_tag);
    k_rc_keep<<<nb, 256, 0, st>>>(*rc, rc_slots, frame_idx, last_tag);
    count_scan(rc->bcount, nb, rc->counts + 1, rc->batch, st);
    k_rc_batch<<<nb, 256, 0, st>>>(fb, *rc, rc_slots, frame_idx, last_tag);
    mark(K_RC);
    {
      rc_train_device(rc->cache, rc->bq, rc->bt, rc->counts + 1, rc->batch, rc->lr, 1, st);
      mark(K_RC_TRAIN);
    }
  }
  // demodulate -> firefly -> SVGF -> TAA -> remodulate -> resolve (lib.rs:492-576)
  const int lb = (int)((P + 255) / 256);
  uint32_t* dcur = fb.demod[cur];
  uint32_t* dprev = fb.demod[cur ^ 1u];
  k_demodulate<<<lb, 256, 0, st>>>(fb, P, cur, fb.radiance, dcur, 0);
  mark(K_DEMODULATE);
  if (cfg.firefly_filter) {
    cudaMemcpyAsync(fb.snapshot, dcur, (size_t)P * 4, cudaMemcpyDeviceToDevice, st);
    mark(K_COPY);
    k_firefly<<<g2, b2, 0, st>>>(fb, W, H, cur, fb.snapshot, dcur);
    mark(K_FIREFLY);
  }
  // With a-trous passes the last pass writes the pre-TAA frame straight into
  // the TAA's neighbourhood copy; otherwise the copy is made here.
  const bool atrous = cfg.svgf && cfg.svgf_atrous_passes > 0;
  const bool taa = cfg.taa && frame_idx > 0;
  if (cfg.svgf) {
    const uint32_t f = frame_idx, passes = cfg.svgf_atrous_passes;
    k_svgf_temporal<<<g2, b2, 0, st>>>(fb, c, dcur, fb.svgf_rad[(f + 1) % 2], fb.svgf_mom[f % 2],
                                       fb.svgf_mom[(f + 1) % 2], atrous ? 1 : 0);
    mark(K_SVGF_TEMPORAL);
    // the reference ping-pongs pass i's output into svgf_rad[(f + i) % 2]; of
    // those stores only the last odd pass's survive into the next frame
    const int last_odd = passes >= 2 ? (int)(((passes - 1) & 1u) ? passes - 1 : passes - 2) : -1;
    uint32_t* final_dst = taa ? fb.snapshot : dcur;
    for (uint32_t i = 0; i < passes; ++i) {
      const bool last = i == passes - 1;
      const uint32_t flags = (i == 0 ? ATR_HIST : 0u) | ((int)i == last_odd ? ATR_STATE : 0u) |
                             (last ? ATR_FINAL : ATR_NEXT);
      const uint2* in_rv = fb.atr_rv[i & 1u];
      uint2* out_rv = fb.atr_rv[(i + 1) & 1u];
      uint32_t* state_rad = fb.svgf_rad[(f + 1) % 2];
      const uint32_t* final_src = fb.svgf_rad[(f + passes - 1) % 2];
      const uint32_t step = i < 8 ? (1u << i) : 128u;
      const uint32_t span = kAtrousTile * step;
      dim3 bt(kAtrousTile, kAtrousTile), gt(((W + span - 1) / span) * step, ((H + span - 1) / span) * step);
      switch (step) {
        case 1: k_atrous<1><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        case 2: k_atrous<2><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        case 4: k_atrous<4><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        case 8: k_atrous<8><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        case 16: k_atrous<16><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        case 32: k_atrous<32><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        case 64: k_atrous<64><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
        default: k_atrous<128><<<gt, bt, 0, st>>>(fb, W, H, flags, in_rv, out_rv, state_rad, final_src, final_dst); break;
      }
      mark(K_ATROUS);
    }
  }
  if (taa) {
    if (!atrous) {
      cudaMemcpyAsync(fb.snapshot, dcur, (size_t)P * 4, cudaMemcpyDeviceToDevice, st);
      mark(K_COPY);
    }
    k_taa<<<g2, b2, 0, st>>>(fb, c, fb.snapshot, dcur, dprev);
    mark(K_TAA);
  }
  k_demodulate<<<lb, 256, 0, st>>>(fb, P, cur, dcur, fb.radiance, 1);
  mark(K_DEMODULATE);
  k_resolve<<<lb, 256, 0, st>>>(fb, P, (float)cfg.sample_count);
  mark(K_RESOLVE);
  return launches;
}

JobTrace job_trace(const DevScene& scene, const FrameBuffers& fb, uint32_t P) {
  JobTrace j{};
  j.nodes = scene.nodes;
  j.tris = scene.tris;
  j.rays = fb.rays;
  j.hits = fb.hits;
  j.queue[0] = fb.queue[0];
  j.queue[1] = fb.queue[1];
  j.counters = fb.counters;
  for (int q = 0; q < 5; ++q) {
    j.rq_o[q] = fb.rq_o[q];
    j.rq_d[q] = fb.rq_d[q];
    j.vis[q] = fb.vis[q];
  }
  j.hit_bsdf = fb.hit_bsdf;
  j.hit_gi = fb.hit_gi;
  j.P = P;
  return j;
}

bool batchable(const FrameConfig& cfg) {
  return !cfg.restir_di && !cfg.restir_gi && !cfg.svgf && !cfg.taa && !cfg.firefly_filter;
}

// The plain-estimator launch sequence of encode_frame (same kernels, same
// order per frame), with the traversal stages shared by the batch.
int encode_batch_plain(const BatchFrame* fr, int nj, const FrameConfig& cfg, const JobTrace* d_jobs, int num_sms,
                       cudaStream_t st) {
  if (nj < 1 || nj > kMaxBatch || !batchable(cfg)) return -1;
  int launches = 0;
  const int persistent_blocks = num_sms * kTraceMinBlocks;
  Consts cs[kMaxBatch];
  int linear[kMaxBatch];
  for (int j = 0; j < nj; ++j) {
    const uint32_t P = fr[j].W * fr[j].H;
    Consts& c = cs[j];
    c = Consts{};
    c.W = fr[j].W;
    c.H = fr[j].H;
    c.P = P;
    c.frame_idx = fr[j].frame_idx;
    c.sample = 0;
    c.cfg = cfg;
    linear[j] = (int)std::min<uint32_t>((P + kBlock - 1) / kBlock, (uint32_t)num_sms * 16u);
    cudaMemsetAsync(fr[j].fb.radiance, 0, (size_t)P * 4, st);
    cudaMemsetAsync(fr[j].fb.counters + 3, 0, 4, st);
  }
  auto each = [&](auto&& f) {
    for (int j = 0; j < nj; ++j) f(j, fr[j].scene, fr[j].fb, cs[j]);
  };
  for (uint32_t sample = 0; sample < cfg.sample_count; ++sample) {
    each([&](int j, const DevScene&, const FrameBuffers& fb, Consts& c) {
      c.seed = c.frame_idx * cfg.sample_count + sample;
      c.sample = sample;
      dim3 b2(16, 16), g2((c.W + 15) / 16, (c.H + 15) / 16);
      k_raygen<<<g2, b2, 0, st>>>(fb, c.W, c.H, fr[j].mats);
      ++launches;
    });
    for (uint32_t i = 0; i < cfg.max_bounces; ++i) {
      each([&](int, const DevScene&, const FrameBuffers& fb, Consts& c) {
        c.bounce = i;
        c.qin = i & 1u;
        c.qout = (i + 1) & 1u;
        cudaMemsetAsync(fb.counters + 2, 0, 4, st);
      });
      k_extend_batch<<<persistent_blocks, kBlock, 0, st>>>(d_jobs, nj, i, i & 1u);
      ++launches;
      each([&](int j, const DevScene& s, const FrameBuffers& fb, Consts& c) {
        cudaMemsetAsync(fb.counters + kCounterQueueSize, 0, 10 * sizeof(uint32_t), st);
        k_shade_a<<<linear[j], kBlock, 0, st>>>(s, fb, c, fr[j].mats);
        ++launches;
      });
      k_trace_queue_batch<false><<<persistent_blocks, kBlock, 0, st>>>(d_jobs, nj, Q_BSDF_CAND);
      ++launches;
      each([&](int j, const DevScene& s, const FrameBuffers& fb, Consts& c) {
        k_shade_b<<<linear[j], kBlock, 0, st>>>(s, fb, c);
        k_shade_b2<<<linear[j], kBlock, 0, st>>>(s, fb, c);
        launches += 2;
      });
      k_trace_queue_batch<false><<<persistent_blocks, kBlock, 0, st>>>(d_jobs, nj, Q_GI_CAND);
      ++launches;
      each([&](int j, const DevScene& s, const FrameBuffers& fb, Consts& c) {
        k_shade_c<<<linear[j], kBlock, 0, st>>>(s, fb, c);
        ++launches;
      });
      k_trace_pair_batch<Q_RIS_SHADOW, Q_GI_SHADOW><<<persistent_blocks, kBlock, 0, st>>>(d_jobs, nj);
      ++launches;
      each([&](int j, const DevScene& s, const FrameBuffers& fb, Consts& c) {
        k_shade_d<<<linear[j], kBlock, 0, st>>>(fb, c);
        k_apply_di_a<<<linear[j], kBlock, 0, st>>>(s, fb, c);
        launches += 2;
      });
      k_trace_queue_batch<true><<<persistent_blocks, kBlock, 0, st>>>(d_jobs, nj, Q_DI_SHADOW);
      ++launches;
      each([&](int j, const DevScene& s, const FrameBuffers& fb, Consts& c) {
        k_apply_di_b<<<linear[j], kBlock, 0, st>>>(fb, c);
        ++launches;
        if (i + 1 < cfg.max_bounces) {
          cudaMemsetAsync(fb.counters + c.qout, 0, 4, st);
          k_apply_gi<<<linear[j], kBlock, 0, st>>>(s, fb, c);
          ++launches;
        }
      });
    }
  }
  // demodulate -> remodulate -> resolve (no filter passes in the plain estimator)
  each([&](int, const DevScene&, const FrameBuffers& fb, Consts& c) {
    const uint32_t cur = c.frame_idx & 1u;
    const int lb = (int)((c.P + 255) / 256);
    uint32_t* dcur = fb.demod[cur];
    k_demodulate<<<lb, 256, 0, st>>>(fb, c.P, cur, fb.radiance, dcur, 0);
    k_demodulate<<<lb, 256, 0, st>>>(fb, c.P, cur, dcur, fb.radiance, 1);
    k_resolve<<<lb, 256, 0, st>>>(fb, c.P, (float)cfg.sample_count);
    launches += 3;
  });
  return launches;
}

void encode_resolve_rgba8(const FrameBuffers& fb, uint32_t W, uint32_t H, uint32_t spp, uint32_t accum_count,
                          cudaStream_t st) {
  dim3 b2(16, 16), g2((W + 15) / 16, (H + 15) / 16);
  k_resolve_rgba8<<<g2, b2, 0, st>>>(fb, W, H, spp, accum_count);
}

void launch_trace_batch(const DevScene& scene, const float4* origins, const float4* dirs, uint32_t n, int any_hit,
                        uint4* out, uint32_t* cursor, int num_sms, cudaStream_t st, const TwoLevel* tl) {
  cudaMemsetAsync(cursor, 0, 4, st);
  if (tl) {
    if (any_hit) k_trace_batch2<true><<<num_sms * kTraceMinBlocks, kBlock, 0, st>>>(scene, *tl, origins, dirs, n, out, cursor);
    else k_trace_batch2<false><<<num_sms * kTraceMinBlocks, kBlock, 0, st>>>(scene, *tl, origins, dirs, n, out, cursor);
    return;
  }
  if (any_hit) k_trace_batch<true><<<num_sms * kTraceMinBlocks, kBlock, 0, st>>>(scene, origins, dirs, n, out, cursor);
  else k_trace_batch<false><<<num_sms * kTraceMinBlocks, kBlock, 0, st>>>(scene, origins, dirs, n, out, cursor);
}

}  // namespace ap
