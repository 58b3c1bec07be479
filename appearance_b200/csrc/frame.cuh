// Per-frame device buffers, constants and kernel launchers of the wavefront
// path tracer (one frame = PathTracerGpu::render, crates/appearance-path-
// tracer-gpu/src/lib.rs:314-615).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "scene_layout.h"

namespace ap {

// Same field order as ap_frame_config (include/appearance_cuda.h).
struct FrameConfig {
  uint32_t max_bounces, sample_count;
  uint32_t restir_di, restir_gi, svgf, firefly_filter, taa;
  uint32_t di_area_samples, di_bsdf_samples;
  float di_temporal_m_factor;
  uint32_t di_spatial_passes, di_spatial_samples, di_unbiased;
  float gi_temporal_m_cap;
  uint32_t gi_spatial_passes, gi_spatial_samples, gi_unbiased;
  uint32_t svgf_max_history, svgf_atrous_passes;
  float taa_history_influence;
};

// Per-pixel state, structure-of-arrays, every record 4 or 16 bytes so that a
// warp reads whole 128-byte lines.
struct FrameBuffers {
  float4* rays;        // origin.xyz, oct30 direction bits
  uint4* payload;      // throughput rgb9e5, rng, t bits, unused
  uint32_t* radiance;  // rgb9e5
  uint4* hits;         // t, u, v bits, global triangle id (extension stage)
  uint4 *di_a, *di_b;  // DiReservoir: (M, W, wsum, phat), (uv, emissive instance, triangle)
  uint4 *di_inter_a, *di_inter_b, *di_prev_a[2], *di_prev_b[2];
  uint4* ctx;          // LightSampleCtx: material, throughput, n, clearcoat n
  uint4 *gi_a, *gi_b;  // GiReservoir: (M, W, wsum, phat), (point.xyz, phat_rng)
  uint4 *gi_inter_a, *gi_inter_b, *gi_prev_a[2], *gi_prev_b[2];
  uint4 *gb_a[2], *gb_b[2];  // G-buffer: (pos.xyz, depth), (n oct30, albedo rgb9e5, velocity.xy)
  uint32_t* demod[2];
  uint32_t* svgf_rad[2];
  float2* svgf_mom[2];
  uint32_t* svgf_count;
  uint32_t* svgf_hist;
  uint32_t* snapshot;  // pre-filter copy for the firefly filter and TAA
  uint32_t* queue[2];  // active path ids (ping-pong)
  // Secondary-ray queues of one bounce (origin.xyz + tmax, direction.xyz + owner
  // path id): Q_BSDF_CAND closest, Q_RIS_SHADOW any, Q_GI_CAND closest,
  // Q_GI_SHADOW any, Q_DI_SHADOW any.
  float4* rq_o[5];
  float4* rq_d[5];
  uint4* hit_bsdf;     // closest hit of the NEE BSDF candidate ray, per path
  uint4* hit_gi;       // closest hit of the GI candidate ray, per path
  uint8_t* vis[5];     // any-hit queues: 1 = unoccluded, per path
  uint4 *st_a, *st_b, *st_c, *st_d, *st_e;  // per-path state between shading stages
  uint32_t* counters;  // [0..1] path queue sizes, [2] extend cursor, [3] rays traced,
                       // [4..8] ray queue sizes, [9..13] ray queue cursors
  unsigned long long* visits;  // instrumented traversal: per kernel kind {rays, nodes, tris}
  // a-trous records: oct30 normal + depth per pixel, and (ping-pong) packed
  // RGB9E5 radiance + variance; aliases of ray-queue storage, idle after the
  // bounce loop
  uint2* atr_nd;
  uint2* atr_rv[2];
  float* out_rgb;      // linear HDR output, 3 floats per pixel (device)
  float4* accum;       // display accumulation (resolve.wgsl accum_radiance)
  uint32_t* rgba;      // RGBA8 display texture, 64x64-block swizzled
};

enum RayQueue { Q_BSDF_CAND = 0, Q_RIS_SHADOW = 1, Q_GI_CAND = 2, Q_GI_SHADOW = 3, Q_DI_SHADOW = 4 };
constexpr int kCounterQueueSize = 4;
constexpr int kCounterQueueCursor = 9;

struct Mats {
  float inv_view[16], inv_proj[16], view_proj[16], prev_view_proj[16];
};

struct FrameStats {
  unsigned long long rays_extend, rays_secondary;
};

size_t frame_buffer_bytes(uint32_t W, uint32_t H);
// Carves `base` (frame_buffer_bytes(W,H) bytes, zeroed by the caller) into buffers.
void frame_buffers_carve(void* base, uint32_t W, uint32_t H, FrameBuffers* fb);

// Kernel kinds for per-kernel timing (FrameProfiler) and launch counting.
enum KernelKind : int {
  K_MEMSET = 0, K_RAYGEN, K_EXTEND, K_SHADE, K_DI_TEMPORAL, K_DI_SPATIAL, K_GI_TEMPORAL, K_GI_SPATIAL,
  K_APPLY_DI, K_APPLY_GI, K_DEMODULATE, K_FIREFLY, K_SVGF_TEMPORAL, K_ATROUS, K_TAA, K_RESOLVE, K_COPY,
  K_TRACE_CLOSEST, K_TRACE_ANY, K_SHADE_B, K_SHADE_C, K_SHADE_D, K_SHADE_B2, K_RC, K_RC_INFER, K_RC_TRAIN, K_ATROUS_PREP, K_NUM_KINDS
};
const char* kernel_kind_name(int k);

// Optional instrumentation: when passed to encode_frame, an event is recorded
// after every launch so that the device time of each kernel kind is the gap
// between consecutive events on the (in-order) stream.
struct FrameProfiler {
  static constexpr int kMax = 512;
  cudaEvent_t ev[kMax + 1];
  int kind[kMax];
  int n = 0;
  bool created = false;
  bool count_visits = false;  // use the visit-counting traversal kernels (fb.visits)
};

// Encodes one frame on `stream`.  `frame_idx` selects the ping-pong parity.
// Returns the number of kernels launched (memsets and copies excluded).
// Radiance-cache mode of a frame (a cache attached with ap_rc_attach): paths of
// most pixels end at their `prefix`-th hit with the cache's prediction; the
// paths of one pixel in `stride` (a different subset each frame) go to full
// depth and give the training targets of their suffix vertices.
struct RcFrame {
  void* cache = nullptr;  // radiance cache (mlp.cu)
  uint32_t prefix = 2, stride = 16, batch = 65536;
  float lr = 1e-3f;
  int train = 1;
  float4* q = nullptr;       // per retired path (compacted): query of its last vertex (4 float4)
  float4* T = nullptr;       //   throughput at that vertex
  uint32_t* own = nullptr;   //   its pixel
  float* out = nullptr;      //   predicted RGB
  float4* rec = nullptr;     // per training pixel and bounce: query (4), throughput (1), radiance so far (1; w = valid)
  float4* bq = nullptr;      // training batch queries (batch x 4)
  float* bt = nullptr;       // training batch targets (batch x 3)
  uint32_t* counts = nullptr;  // [0] candidate records, [1] batch entries, [2] retired paths of the sample
  uint32_t* bcount = nullptr;  // per 256 record slots: records kept for the batch, then their first batch slot
};
constexpr uint32_t kRcMaxBounces = 8;        // record slots per training pixel
constexpr uint32_t kRcRetired = 0xFFFFFFFEu;  // hit id of a path retired into the cache
size_t rc_frame_bytes(uint32_t W, uint32_t H, uint32_t stride, uint32_t batch);
// In place: counts[0..n) -> their exclusive prefix sums; *total = min(sum, cap).
// Assembles training batches in record order (one block, any n).
void count_scan(uint32_t* counts, uint32_t n, uint32_t* total, uint32_t cap, cudaStream_t st);
void rc_frame_carve(void* base, uint32_t W, uint32_t H, uint32_t stride, uint32_t batch, RcFrame* rc);

// mlp.cu: inference over n queries, and one training step on a device-assembled batch
// (n_dev, when given: the number of queries, read on the device, at most n)
int rc_infer_device(void* cache, const float4* queries, uint32_t n, float* out, cudaStream_t st,
                    const uint32_t* n_dev = nullptr);
int rc_train_device(void* cache, const float4* queries, const float* targets, const uint32_t* n_dev, uint32_t cap,
                    float lr, int update, cudaStream_t st);
// After the stream drained: the first error of those calls since the last
// check, or AP_E_TIMEOUT for an inference wait that ran out; clears it.
int rc_take_status(void* cache, std::string* msg);

// Optional second stream for encode_frame (side2 and side3 serve the spectral mode): the DI shadow rays of every bounce
// but the last are traced on `side` beside the next bounce's path extension
// (apply_gi -> extend), which reads none of their results, so one persistent
// launch's drain tail overlaps the other's work; `fork` and `join` order the
// two streams.  Ignored while profiling (per-kernel times need one stream).
struct FrameStreams {
  cudaStream_t side = nullptr;
  cudaStream_t side2 = nullptr, side3 = nullptr;  // the spectral mode's third and fourth sample passes
  cudaEvent_t fork = nullptr, join = nullptr;
};
int frame_streams_create(FrameStreams* fs);  // cudaError_t of the first failing call
void frame_streams_destroy(FrameStreams* fs);

int encode_frame(const DevScene& scene, const FrameBuffers& fb, const FrameConfig& cfg, const Mats& mats,
                 uint32_t W, uint32_t H, uint32_t frame_idx, int num_sms, cudaStream_t stream,
                 FrameProfiler* prof = nullptr, const RcFrame* rc = nullptr, const FrameStreams* fs = nullptr);

// ---- batches of frames sharing their traversal launches (serving) ----------
//
// Frames of the plain estimator (no reuse passes, denoising or radiance cache)
// with the same sample and bounce counts have the same launch sequence; a
// batch of up to kMaxBatch of them, each with its own scene, size, camera,
// seed and frame state, runs as one sequence: the shading stages launch per
// frame, and every traversal stage is one persistent launch over all the
// frames' ray queues, each ray traced through its own frame's BVH.  A frame's
// result is the one it has alone (its rays, random streams and queues are its
// own; only which lane traces a ray changes).
constexpr int kMaxBatch = 8;

// What the batch traversal kernels read and write of one frame (a device
// array of these is the kernels' argument).
struct JobTrace {
  const uint4* nodes;
  const float4* tris;
  const float4* rays;
  uint4* hits;
  const uint32_t* queue[2];
  uint32_t* counters;
  const float4* rq_o[5];
  const float4* rq_d[5];
  uint4* hit_bsdf;
  uint4* hit_gi;
  uint8_t* vis[5];
  uint32_t P;
};

struct BatchFrame {
  DevScene scene;
  FrameBuffers fb;
  Mats mats;
  uint32_t W, H, frame_idx;
};

JobTrace job_trace(const DevScene& scene, const FrameBuffers& fb, uint32_t P);
// Whether frames of `cfg` can share launches (the plain estimator).
bool batchable(const FrameConfig& cfg);
// Encodes the batch frames[0..nj) on `stream`; d_jobs holds job_trace() of
// each frame, in the same order, in device memory.  Returns the kernels launched.
int encode_batch_plain(const BatchFrame* frames, int nj, const FrameConfig& cfg, const JobTrace* d_jobs, int num_sms,
                       cudaStream_t stream);

// Closest / any hit for a batch of rays (parity tests and traversal bench).
// rays: origin.xyz + tmax (float4), dirs: float4; out: t, u, v, tri bits.
// The display resolve (resolve.wgsl:40-59): ACES-fit tonemap of radiance /
// spp, accumulated over `accum_count` earlier frames, stored as RGBA8 at the
// 64x64-block-swizzled position (block.wgsl:3-16).
void encode_resolve_rgba8(const FrameBuffers& fb, uint32_t W, uint32_t H, uint32_t spp, uint32_t accum_count,
                          cudaStream_t st);

struct TwoLevel;
// Closest or any hit of n rays (origin + tmax, direction): over `scene`, or
// over the two-level scene `tl` (with `scene` holding its BLAS pool) when
// given.
void launch_trace_batch(const DevScene& scene, const float4* origins, const float4* dirs, uint32_t n,
                        int any_hit, uint4* out, uint32_t* cursor, int num_sms, cudaStream_t stream,
                        const TwoLevel* tl = nullptr);

}  // namespace ap
