/* C ABI of the B200 path-tracing frame: the boundary a host (Rust over FFI,
 * C++, or Python ctypes) binds in place of the reference's GPU renderer.
 *
 * Reference interfaces replaced:
 *   NodeRenderer::visible_world_action / NodeRenderer::render
 *       crates/appearance-render-loop/src/node.rs:14-25
 *   DistributedRenderer (its NodeRenderer impl)
 *       crates/appearance-distributed-renderer/src/lib.rs:60-82
 *   PathTracerGpu::new / handle_visible_world_action / render
 *       crates/appearance-path-tracer-gpu/src/lib.rs:260-302, 314-615
 *   PathTracerGpuConfig (+ the pass literals of render)
 *       crates/appearance-path-tracer-gpu/src/lib.rs:220-245, 413-545
 *   VisibleWorldActionType wire format
 *       crates/appearance-world/src/visible_world_action.rs:9-125
 *
 * Ownership: the library owns all device memory and the per-handle temporal
 * state (reservoirs, G-buffers, SVGF/TAA history); the caller owns every host
 * buffer it passes, and no pointer escapes a call.  A handle is used by one
 * host thread at a time.  Every entry point returns an AP_* status; none
 * aborts.  ap_last_error() describes the last failure of a handle.
 */
#ifndef APPEARANCE_CUDA_H
#define APPEARANCE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  AP_OK = 0,
  AP_E_INVALID = 1,     /* bad argument, size or state */
  AP_E_OOM = 2,         /* device allocation failed */
  AP_E_CUDA = 3,        /* CUDA runtime error (message in ap_last_error) */
  AP_E_TIMEOUT = 4,     /* a bounded device wait ran out */
  AP_E_UNSUPPORTED = 5, /* valid request this library does not implement */
  AP_E_NO_SCENE = 6,    /* render before any geometry was uploaded */
  AP_E_CANCELLED = 7    /* a serving job was cancelled (ap_server_cancel) */
};

/* PathTracerGpuConfig plus the literals the reference hard-codes in render()
 * and in its shaders.  ap_frame_config_default() gives the reference values. */
typedef struct ap_frame_config {
  uint32_t max_bounces;         /* 2   lib.rs:235 */
  uint32_t sample_count;        /* 1   lib.rs:236 */
  uint32_t restir_di;           /* 1   lib.rs:238 */
  uint32_t restir_gi;           /* 1   lib.rs:239 */
  uint32_t svgf;                /* 0   lib.rs:240 */
  uint32_t firefly_filter;      /* 1   lib.rs:241 */
  uint32_t taa;                 /* 0   lib.rs:242 */
  uint32_t di_area_samples;     /* 4   helpers/nee.wgsl:125 */
  uint32_t di_bsdf_samples;     /* 1   helpers/nee.wgsl:126 */
  float di_temporal_m_factor;   /* 20  restir_di_temporal.wgsl:159 */
  uint32_t di_spatial_passes;   /* 1   lib.rs:417 */
  uint32_t di_spatial_samples;  /* 3   restir_di_spatial.wgsl:15 */
  uint32_t di_unbiased;         /* 1   lib.rs:419 */
  float gi_temporal_m_cap;      /* 30  restir_gi_temporal.wgsl:100 */
  uint32_t gi_spatial_passes;   /* 0   lib.rs:441 */
  uint32_t gi_spatial_samples;  /* 5   restir_gi_spatial.wgsl:16 */
  uint32_t gi_unbiased;         /* 1   lib.rs:443 */
  uint32_t svgf_max_history;    /* 24  lib.rs:522 */
  uint32_t svgf_atrous_passes;  /* 5   lib.rs:523 */
  float taa_history_influence;  /* 0.8 lib.rs:538 */
} ap_frame_config;

/* MaterialDescriptor (shared/material/material_pool.wgsl:6-41) without the
 * texture slots; 26 floats. */
typedef struct ap_material {
  float color[3];
  float metallic, roughness;
  float emission[3];
  float transmission, eta, subsurface;
  float absorption[3];
  float specular;
  float specular_tint[3];
  float anisotropic, sheen;
  float sheen_tint[3];
  float clearcoat, clearcoat_roughness, alpha_cutoff;
} ap_material;

/* One mesh of the scene (a VertexPoolSlice, shared/vertex_pool.wgsl:3-12). */
typedef struct ap_mesh {
  uint32_t first_vertex, num_vertices; /* into positions/normals */
  uint32_t first_index, num_indices;   /* into indices (3 per triangle) */
  uint32_t material_idx;               /* first material of the mesh */
  uint32_t emissive;                   /* 1: mesh takes part in light sampling */
} ap_mesh;

/* A whole scene: world-space vertex pool, per-triangle material indices
 * relative to the mesh's material_idx, materials, an optional equirect
 * environment (RGB f32, env_w x env_h) and the analytic sun (SunInfo,
 * scene_resources/sky.rs:11-22: direction xyz, size, color xyz, intensity). */
typedef struct ap_scene_desc {
  const float* positions;        /* 3 floats per vertex */
  const float* normals;          /* 3 floats per vertex, unit length */
  uint32_t num_vertices;
  const uint32_t* indices;       /* 3 per triangle, relative to the mesh's first_vertex */
  const uint32_t* tri_material;  /* 1 per triangle */
  uint32_t num_tris;
  const ap_mesh* meshes;
  uint32_t num_meshes;
  const ap_material* materials;
  uint32_t num_materials;
  const float* env;              /* may be NULL (black sky) */
  uint32_t env_w, env_h;
  float sun[8];
} ap_scene_desc;

typedef struct ap_frame_stats {
  double gpu_ms;            /* device time of the frame (CUDA events) */
  uint64_t extension_rays;  /* closest-hit rays of the path-extension stage */
  uint32_t width, height;
  uint32_t frame_idx;
  uint32_t kernel_launches; /* kernels launched for the frame (copies/memsets excluded) */
} ap_frame_stats;

/* Fills the reference defaults (PathTracerGpuConfig::default + pass literals). */
void ap_frame_config_default(ap_frame_config* cfg);

/* PathTracerGpu::new (lib.rs:260-281).  Returns NULL and sets *err on failure.
 * The handle owns four non-blocking CUDA streams on `device`: the frame's,
 * one for traversal that overlaps the next bounce, and (with those two) the
 * spectral mode's concurrent sample passes; all are idle when a render call
 * returns. */
void* ap_create(const ap_frame_config* cfg, int device, int* err);
void ap_destroy(void* handle);
const char* ap_last_error(const void* handle);
/* Replaces the frame configuration and restarts the frame sequence (the
 * temporal state is dropped, the next frame is frame 0). */
int ap_set_config(void* handle, const ap_frame_config* cfg);

/* NodeRenderer::visible_world_action (node.rs:16): `ty` and `bytes` exactly as
 * VisibleWorldActionType::from_ty_and_bytes (visible_world_action.rs:87-96),
 * handled as PathTracerGpu's SceneResources does
 * (crates/appearance-path-tracer-gpu/src/scene_resources/mod.rs:107-156):
 *   0 CameraUpdate {Mat4 transform, fov deg, near, far, pad}, 80 bytes;
 *   1 SpawnModel {Mat4 transform, Uuid entity, [u8; 256] asset path}, 336
 *     bytes: an instance of the model registered under that path
 *     (ap_model_register; AP_E_INVALID when none is), keyed by the uuid;
 *   2 TransformModel {Mat4 transform, Uuid entity}, 80 bytes: moves the
 *     instance (AP_E_INVALID for an unknown uuid, which the reference only
 *     logs);
 *   3 DestroyModel {Uuid entity}, 16 bytes: removes it;
 *   4 Clear (u32), 4 bytes: drops the base scene and all instances.
 * Matrices are glam Mat4, column-major.  The scene the renders see is the
 * uploaded base scene plus every instance, flattened to world space; a world
 * action that changes it takes effect at the next render (which rebuilds
 * the BVH, as the reference rebuilds its TLAS before every frame) and drops
 * the spectral tables (call ap_spectral_setup again). */
int ap_world_action(void* handle, uint32_t ty, const void* bytes, size_t len);

/* Uploads (replaces) the base scene, removes every spawned instance, and
 * builds the wide BVH. */
int ap_scene_upload(void* handle, const ap_scene_desc* desc);

/* Registers (or replaces) the model SpawnModel names by `asset_path` (1..255
 * bytes): its meshes, materials and vertex pool in model space, as an
 * ap_scene_desc whose environment and sun are ignored.  The reference loads a
 * model from its asset database by that path (a glTF file,
 * AssetDatabase<Model>::get, scene_resources/mod.rs:121); a host loads the
 * file itself (appearance_b200/gltf.py reads glTF 2.0) and registers its
 * geometry here. */
int ap_model_register(void* handle, const char* asset_path, const ap_scene_desc* model);

/* Explicit camera: inv_view, inv_proj, view_proj, prev_view_proj as 4
 * column-major float[16], used for the next render (overrides CameraUpdate). */
int ap_set_camera_matrices(void* handle, const float* mats16x4);

/* NodeRenderer::render (node.rs:18-24) / PathTracerGpu::render: renders one
 * frame of w x h pixels and writes linear HDR RGB f32 (radiance / sample
 * count, before the reference's tonemap, resolve.wgsl:48-50) for rows
 * [row_start, row_end) to `out_rgb` (3 floats per pixel, row-major).
 * Synchronous: returns when `out_rgb` holds the result. */
int ap_render_hdr(void* handle, uint32_t w, uint32_t h, uint32_t row_start, uint32_t row_end, float* out_rgb,
                  size_t out_bytes, ap_frame_stats* stats);

/* The byte output of NodeRenderer::render / PathTracerGpu::render
 * (lib.rs:556-609): the same frame, then the display resolve (resolve.wgsl:
 * 29-59): radiance / sample count through the ACES fit, averaged over the
 * frames rendered by this call since the camera last moved when `accumulate`
 * != 0 (PathTracerGpuConfig::accum_frames, lib.rs:223,349-352), stored as RGBA8
 * at the 64x64-block-swizzled position of block.wgsl:3-16 (the texture the
 * reference reads back).  Rows [row_start, row_end) of the w x h texture
 * (4 bytes per pixel, row-major) go to `out_rgba`. */
int ap_render_rgba8(void* handle, uint32_t w, uint32_t h, uint32_t row_start, uint32_t row_end, int accumulate,
                    uint8_t* out_rgba, size_t out_bytes, ap_frame_stats* stats);

/* Renders one frame into the device-resident framebuffer only (no copy to
 * the host); ap_device_framebuffer() returns its device address. */
int ap_render_device(void* handle, uint32_t w, uint32_t h, ap_frame_stats* stats);
const float* ap_device_framebuffer(const void* handle);

/* Closest-hit (any_hit = 0) or any-hit (1) queries against the uploaded BVH.
 * origins_tmax: n x {ox, oy, oz, tmax}; dirs: n x {dx, dy, dz, unused};
 * out: n x {t, u, v, triangle id} (as raw 32-bit words; any-hit: {hit, 0,0,0}).
 * Host buffers; tmin is 0. */
int ap_trace_rays(void* handle, const float* origins_tmax, const float* dirs, uint32_t n, int any_hit,
                  uint32_t* out4);

/* The query of ap_trace_rays for callers that cannot allocate device memory
 * (a host that owns the whole device-memory budget, or a thread that cannot
 * take cudaMalloc's device-wide synchronisation).  It has no counterpart in the
 * reference.  It allocates nothing: its device staging is a fixed static array
 * of the library, so n is at most 65536 rays per call (AP_E_INVALID above
 * that).  All calls on a device share that array: calls that overlap on the
 * GPU race, so serialise them.  The first call on a device looks up the
 * array's device address; make that first call before any stream capture.
 * Same buffers and results as ap_trace_rays. */
int ap_trace_rays_static(void* handle, const float* origins_tmax, const float* dirs, uint32_t n, int any_hit,
                         uint32_t* out4);

/* Copies a per-pixel state buffer of the last frame to the host, for
 * stage-by-stage comparisons: 0 radiance (1 word), 1 payload (4), 2 current
 * G-buffer (8), 3 DI reservoirs (8), 4 GI reservoirs (8), 5 light-sample
 * context (4), 7 rays (4); working buffers of the last bounce that used them:
 * 8 BSDF-candidate hits (4), 9 GI-candidate hits (4), 10 GI-candidate ray
 * queue (8: origin+tmax, direction+owner), 11 and 12 shading-stage state (8). */
int ap_read_buffer(void* handle, uint32_t which, uint32_t* out, size_t out_bytes);

/* Renders one frame (advancing the frame sequence like ap_render_device) with
 * an event after every launch, and returns the device milliseconds and the
 * launch count of each kernel kind: kind_ms and kind_count hold `max_kinds`
 * entries; names[i] receives a static string naming kind i; *num_kinds the
 * number of kinds written.  With count_visits != 0 the traversal kernels run
 * in their instrumented form (slower; times are then not representative) and
 * visits[3*i .. 3*i+2] receives {rays, BVH nodes visited, triangles tested}
 * of kind i. */
int ap_profile_frame(void* handle, uint32_t w, uint32_t h, double* kind_ms, uint32_t* kind_count,
                     const char** names, uint32_t max_kinds, uint32_t* num_kinds, int count_visits,
                     uint64_t* visits, ap_frame_stats* stats);

/* BVH statistics of the uploaded scene: nodes, triangles, max depth, max
 * traversal stack, build ms (as double bits in out[4..5]). */
int ap_bvh_stats(void* handle, uint32_t* out8);

/* ---- spectral mode: the CPU tracer's estimator (appearance-path-tracer) ----
 *
 * Replaces the render of crates/appearance-path-tracer/src/lib.rs:79-195
 * (PathTracer::render -> path_tracer::render_pixels, path_tracer.rs:28-67 ->
 * PathIntegrator::li, path_integrator.rs:103-307): four hero wavelengths per
 * path, RGB albedos and emitters upsampled to spectra, diffuse / gold
 * conductor / dielectric BxDFs, interpolated vertex normals, the distant light
 * by next-event estimation and the environment on escape, weighted by the
 * power heuristic against its compensated sampling density.
 *
 * ap_spectral_setup builds the spectral tables of the uploaded scene (call
 * again after every ap_scene_upload): the distant light travels along
 * sun_dir3 with radiance sun_scale x the illuminant spectrum of sun_rgb3, its
 * shadow rays end 2 x scene_radius away (DistantLight::new(dir, spectrum,
 * scale, scene_radius), geometry_resources.rs:52-64: (0,-1,0.2), (1,1,0.95),
 * 100, 1000); the environment's texels are scaled by env_scale. */
int ap_spectral_setup(void* handle, const float* sun_dir3, const float* sun_rgb3, float sun_scale, float scene_radius,
                      float env_scale);
/* Renders rows [row_start, row_end) of a w x h image with `spp` paths per
 * pixel through the pixel centre, paths of at most max_depth surface
 * interactions (the reference uses 4).  Sample k of every pixel is the
 * reference's 1-sample frame with frame index seed + k: the same ZSobol
 * sampler (zsobol_sampler.rs, seeded with the frame index) at the pixel the
 * reference derives from the flipped uv (path_tracer.rs:52-56).  out_rgb
 * receives linear sRGB, 3 floats per pixel, the mean over the samples; with
 * out_rgb NULL the image stays on the device (timing).  Synchronous;
 * stats->gpu_ms is the kernel's device time and stats->extension_rays the rays
 * it traced (closest and shadow). */
int ap_render_spectral(void* handle, uint32_t w, uint32_t h, uint32_t row_start, uint32_t row_end, uint32_t spp,
                       uint32_t max_depth, uint32_t seed, float* out_rgb, size_t out_bytes, ap_frame_stats* stats);
/* ap_render_spectral (image kept on the device) with the traversal kernels in
 * their instrumented form: visits6 receives closest-hit rays, nodes visited,
 * triangles tested, then the same for the any-hit (shadow) rays.  Times are
 * not representative.  It has no counterpart in the reference. */
int ap_profile_spectral(void* handle, uint32_t w, uint32_t h, uint32_t row_start, uint32_t row_end, uint32_t spp,
                        uint32_t max_depth, uint32_t seed, uint64_t* visits6, ap_frame_stats* stats);

/* ---- render-serving loop ------------------------------------------------
 * No reference counterpart as an API: it takes the role of the reference's
 * frame farm (Host/Node, crates/appearance-render-loop/src/host.rs:250-505,
 * node.rs:27-147), where each node renders one request at a time.  Here one
 * server owns the GPU: scenes stay resident, submitted jobs are admitted in
 * arrival order while their frame state fits `hbm_budget` (scene bytes
 * included) and one of `max_inflight` slots is free, and jobs in flight run
 * concurrently, one stream each.  A job renders `spp` samples per pixel with
 * `max_depth` bounces using the server's frame configuration otherwise, from
 * a fresh frame sequence with PCG frame index `seed`; its result is the same
 * alone and in any mix of jobs.  With a plain-estimator configuration
 * (restir_di, restir_gi, svgf, taa and firefly_filter all 0), queued jobs of
 * the same spp and max_depth are admitted together, up to 8
 * (ap_server_set_batching), and run as one launch sequence whose traversal
 * stages are shared persistent launches over all their ray queues; each
 * job's result is still its alone result.  use_graphs != 0 launches each
 * slot's work as a CUDA graph (captured per launch, updated in place when the
 * slot ran a launch sequence of the same shape before: same spp, depth and
 * batch size).  The server's dispatcher thread and CUDA callbacks do the
 * work; all entry points are thread-safe. */
typedef struct ap_job {
  uint32_t scene;           /* id from ap_server_add_scene */
  uint32_t width, height;
  uint32_t spp;             /* 1..4096 */
  uint32_t max_depth;       /* bounces, 1..64 */
  uint32_t seed;            /* frame index of the per-pixel PCG streams */
  uint32_t deadline_ms;     /* 0: none; else a job still queued this long after submission is not
                               started and completes with AP_E_TIMEOUT */
  float mats[64];           /* inv_view, inv_proj, view_proj, prev_view_proj (column-major) */
} ap_job;

typedef struct ap_job_result {
  double queued_ms;         /* submit -> admitted */
  double total_ms;          /* submit -> result in the caller's buffer */
  double gpu_ms;            /* the job's span on its stream (CUDA events) */
  uint64_t device_bytes;    /* frame state held while it ran */
  uint32_t graph_mode;      /* 0 direct launches, 1 graph instantiated, 2 graph updated in place */
  uint32_t slot;
  uint32_t batch;           /* jobs of the launch sequence it ran in (1: alone) */
  uint32_t pad;
} ap_job_result;

void* ap_server_create(const ap_frame_config* cfg, int device, uint64_t hbm_budget, uint32_t max_inflight,
                       int use_graphs, int* err);
/* Finishes queued and in-flight jobs, then frees everything. */
void ap_server_destroy(void* server);
const char* ap_server_last_error(const void* server);
int ap_server_add_scene(void* server, const ap_scene_desc* desc, uint32_t* scene_id);
/* Device bytes of one job's frame state at width x height. */
uint64_t ap_server_job_bytes(uint32_t width, uint32_t height);
/* Queues a job; returns at once.  The linear HDR RGB f32 result (w*h*3 floats,
 * row-major) is written to out_rgb, which must stay valid until the job is
 * waited for; page-locked memory (cudaHostAlloc) receives it directly. */
int ap_server_submit(void* server, const ap_job* job, float* out_rgb, size_t out_bytes, uint64_t* ticket);
int ap_server_query(void* server, uint64_t ticket, int* done);
/* Blocks until the job is done; returns its status and releases the ticket. */
int ap_server_wait(void* server, uint64_t ticket, ap_job_result* result);
/* Cancels a job: a queued job is dropped without running; a job already on
 * the GPU runs to the end of its launches (device work is not interrupted),
 * and its output buffer may have been written.  Either way its wait returns
 * AP_E_CANCELLED.  A finished job is left as it is (AP_OK); an unknown ticket
 * is AP_E_INVALID. */
int ap_server_cancel(void* server, uint64_t ticket);
/* Largest batch of jobs admitted together (1..8, default 8; 1 runs every job
 * on its own).  Takes effect at the next admission. */
int ap_server_set_batching(void* server, uint32_t max_batch);
/* completed, in flight, queued, device bytes in use, peak device bytes, scene
 * bytes, graphs instantiated, graphs updated in place */
int ap_server_stats(void* server, uint64_t* out8);

/* ---- radiance cache -------------------------------------------------------
 * No reference counterpart (the reference traces every path to full depth).
 * A small MLP (144 encoded inputs, 4 hidden layers of 64 with ReLU, 3 outputs
 * with exp; FP16 weights and activations, FP32 accumulation and master
 * weights) predicting the outgoing radiance of a path vertex, trained online
 * with Adam on a relative L2 loss.  A query is 16 floats: position (3),
 * roughness, outgoing direction (3, unit), 0, diffuse albedo (3), specular
 * albedo (3), 0, 0.  Positions are normalised to the box [scene_lo, scene_hi].
 * Parameters: AP_RC_NUM_PARAMS floats, W0 (64 x 144), W1, W2, W3 (64 x 64),
 * W4 (3 x 64), each row-major [out][in]. */
#define AP_RC_NUM_PARAMS 21696
void* ap_rc_create(int device, const float* scene_lo, const float* scene_hi, uint32_t seed, int* err);
void ap_rc_destroy(void* cache);
const char* ap_rc_last_error(const void* cache);
/* Replaces the master weights and restarts Adam. */
int ap_rc_set_params(void* cache, const float* params, uint32_t count);
int ap_rc_get_params(void* cache, float* params, uint32_t count);
/* Predicted RGB radiance of n queries (tensor-core inference); host buffers. */
int ap_rc_infer(void* cache, const float* queries, uint32_t n, float* out_rgb);
/* One training step on n (query, target RGB) pairs: loss and gradients, then
 * an Adam update (lr; beta1 0.9, beta2 0.999, eps 1e-8) when update != 0.
 * Writes the batch loss to *loss and, when grad_out is not NULL, the
 * gradient of the loss (AP_RC_NUM_PARAMS floats). */
int ap_rc_train(void* cache, const float* queries, const float* targets, uint32_t n, float lr, int update,
                float* loss, float* grad_out);
/* Self-test of the bounded tensor-core completion wait used by ap_rc_infer
 * (no counterpart in the reference): on `device`, a barrier that nothing
 * arrives on must give up after `limit` tries (1..2^22) and report it,
 * out2[0] = 0; one that has completed must report success, out2[1] = 1.
 * The error path it exercises is the one that turns a stalled tensor-core
 * wait into AP_E_TIMEOUT instead of a hung kernel. */
int ap_rc_wait_selftest(int device, int limit, uint32_t* out2);
/* Radiance-cache mode of a renderer (cache NULL detaches): in every frame the
 * paths of most pixels end at their `prefix_bounces`-th hit with T x the
 * cache's prediction (the frame's max_bounces must exceed prefix_bounces);
 * one pixel in `train_stride`, a different subset each frame, traces to
 * max_bounces and its suffix vertices (bounces 1..7) give training targets
 * (the radiance measured after the vertex divided by the throughput at it),
 * of which `train_batch` are drawn at random for one Adam step (learning rate
 * `lr`) per frame when `train` != 0.  The cache must outlive the attachment.
 * ap_render_spectral uses the attachment too: each sample pass is a frame,
 * the prediction (RGB) is upsampled to each path's wavelengths, and training
 * targets are the RGB of the spectral suffix estimates. */
int ap_rc_attach(void* handle, void* cache, uint32_t prefix_bounces, uint32_t train_stride, uint32_t train_batch,
                 float lr, int train);

#ifdef __cplusplus
}
#endif

#endif /* APPEARANCE_CUDA_H */
