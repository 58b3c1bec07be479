//! `extern "C"` declarations of include/appearance_cuda.h, one to one: the
//! structs are `#[repr(C)]` with the header's field order, pointers are raw,
//! statuses are `c_int` (AP_OK = 0).  See the header for each call's contract.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const AP_OK: c_int = 0;
pub const AP_E_INVALID: c_int = 1;
pub const AP_E_OOM: c_int = 2;
pub const AP_E_CUDA: c_int = 3;
pub const AP_E_TIMEOUT: c_int = 4;
pub const AP_E_UNSUPPORTED: c_int = 5;
pub const AP_E_NO_SCENE: c_int = 6;
pub const AP_E_CANCELLED: c_int = 7;
pub const AP_RC_NUM_PARAMS: u32 = 21696;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ApFrameConfig {
    pub max_bounces: u32,
    pub sample_count: u32,
    pub restir_di: u32,
    pub restir_gi: u32,
    pub svgf: u32,
    pub firefly_filter: u32,
    pub taa: u32,
    pub di_area_samples: u32,
    pub di_bsdf_samples: u32,
    pub di_temporal_m_factor: f32,
    pub di_spatial_passes: u32,
    pub di_spatial_samples: u32,
    pub di_unbiased: u32,
    pub gi_temporal_m_cap: f32,
    pub gi_spatial_passes: u32,
    pub gi_spatial_samples: u32,
    pub gi_unbiased: u32,
    pub svgf_max_history: u32,
    pub svgf_atrous_passes: u32,
    pub taa_history_influence: f32,
}

/// MaterialDescriptor without texture slots (26 floats).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ApMaterial {
    pub color: [f32; 3],
    pub metallic: f32,
    pub roughness: f32,
    pub emission: [f32; 3],
    pub transmission: f32,
    pub eta: f32,
    pub subsurface: f32,
    pub absorption: [f32; 3],
    pub specular: f32,
    pub specular_tint: [f32; 3],
    pub anisotropic: f32,
    pub sheen: f32,
    pub sheen_tint: [f32; 3],
    pub clearcoat: f32,
    pub clearcoat_roughness: f32,
    pub alpha_cutoff: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ApMesh {
    pub first_vertex: u32,
    pub num_vertices: u32,
    pub first_index: u32,
    pub num_indices: u32,
    pub material_idx: u32,
    pub emissive: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ApSceneDesc {
    pub positions: *const f32,
    pub normals: *const f32,
    pub num_vertices: u32,
    pub indices: *const u32,
    pub tri_material: *const u32,
    pub num_tris: u32,
    pub meshes: *const ApMesh,
    pub num_meshes: u32,
    pub materials: *const ApMaterial,
    pub num_materials: u32,
    pub env: *const f32,
    pub env_w: u32,
    pub env_h: u32,
    pub sun: [f32; 8],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ApFrameStats {
    pub gpu_ms: f64,
    pub extension_rays: u64,
    pub width: u32,
    pub height: u32,
    pub frame_idx: u32,
    pub kernel_launches: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ApJob {
    pub scene: u32,
    pub width: u32,
    pub height: u32,
    pub spp: u32,
    pub max_depth: u32,
    pub seed: u32,
    pub deadline_ms: u32,
    pub mats: [f32; 64],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ApJobResult {
    pub queued_ms: f64,
    pub total_ms: f64,
    pub gpu_ms: f64,
    pub device_bytes: u64,
    pub graph_mode: u32,
    pub slot: u32,
    pub batch: u32,
    pub pad: u32,
}

extern "C" {
    // renderer handle
    pub fn ap_frame_config_default(cfg: *mut ApFrameConfig);
    pub fn ap_create(cfg: *const ApFrameConfig, device: c_int, err: *mut c_int) -> *mut c_void;
    pub fn ap_destroy(handle: *mut c_void);
    pub fn ap_last_error(handle: *const c_void) -> *const c_char;
    pub fn ap_set_config(handle: *mut c_void, cfg: *const ApFrameConfig) -> c_int;

    // world
    pub fn ap_world_action(handle: *mut c_void, ty: u32, bytes: *const c_void, len: usize) -> c_int;
    pub fn ap_scene_upload(handle: *mut c_void, desc: *const ApSceneDesc) -> c_int;
    pub fn ap_model_register(handle: *mut c_void, asset_path: *const c_char, model: *const ApSceneDesc) -> c_int;
    pub fn ap_set_camera_matrices(handle: *mut c_void, mats16x4: *const f32) -> c_int;

    // frames
    pub fn ap_render_hdr(handle: *mut c_void, w: u32, h: u32, row_start: u32, row_end: u32, out_rgb: *mut f32,
                         out_bytes: usize, stats: *mut ApFrameStats) -> c_int;
    pub fn ap_render_rgba8(handle: *mut c_void, w: u32, h: u32, row_start: u32, row_end: u32, accumulate: c_int,
                           out_rgba: *mut u8, out_bytes: usize, stats: *mut ApFrameStats) -> c_int;
    pub fn ap_render_device(handle: *mut c_void, w: u32, h: u32, stats: *mut ApFrameStats) -> c_int;
    pub fn ap_device_framebuffer(handle: *const c_void) -> *const f32;

    // ray queries and diagnostics
    pub fn ap_trace_rays(handle: *mut c_void, origins_tmax: *const f32, dirs: *const f32, n: u32, any_hit: c_int,
                         out4: *mut u32) -> c_int;
    pub fn ap_trace_rays_static(handle: *mut c_void, origins_tmax: *const f32, dirs: *const f32, n: u32,
                                any_hit: c_int, out4: *mut u32) -> c_int;
    pub fn ap_read_buffer(handle: *mut c_void, which: u32, out: *mut u32, out_bytes: usize) -> c_int;
    pub fn ap_profile_frame(handle: *mut c_void, w: u32, h: u32, kind_ms: *mut f64, kind_count: *mut u32,
                            names: *mut *const c_char, max_kinds: u32, num_kinds: *mut u32, count_visits: c_int,
                            visits: *mut u64, stats: *mut ApFrameStats) -> c_int;
    pub fn ap_bvh_stats(handle: *mut c_void, out8: *mut u32) -> c_int;

    // spectral mode (the CPU tracer's estimator)
    pub fn ap_spectral_setup(handle: *mut c_void, sun_dir3: *const f32, sun_rgb3: *const f32, sun_scale: f32,
                             scene_radius: f32, env_scale: f32) -> c_int;
    pub fn ap_render_spectral(handle: *mut c_void, w: u32, h: u32, row_start: u32, row_end: u32, spp: u32,
                              max_depth: u32, seed: u32, out_rgb: *mut f32, out_bytes: usize,
                              stats: *mut ApFrameStats) -> c_int;
    pub fn ap_profile_spectral(handle: *mut c_void, w: u32, h: u32, row_start: u32, row_end: u32, spp: u32,
                               max_depth: u32, seed: u32, visits6: *mut u64, stats: *mut ApFrameStats) -> c_int;

    // render-serving loop
    pub fn ap_server_create(cfg: *const ApFrameConfig, device: c_int, hbm_budget: u64, max_inflight: u32,
                            use_graphs: c_int, err: *mut c_int) -> *mut c_void;
    pub fn ap_server_destroy(server: *mut c_void);
    pub fn ap_server_last_error(server: *const c_void) -> *const c_char;
    pub fn ap_server_add_scene(server: *mut c_void, desc: *const ApSceneDesc, scene_id: *mut u32) -> c_int;
    pub fn ap_server_job_bytes(width: u32, height: u32) -> u64;
    pub fn ap_server_submit(server: *mut c_void, job: *const ApJob, out_rgb: *mut f32, out_bytes: usize,
                            ticket: *mut u64) -> c_int;
    pub fn ap_server_query(server: *mut c_void, ticket: u64, done: *mut c_int) -> c_int;
    pub fn ap_server_wait(server: *mut c_void, ticket: u64, result: *mut ApJobResult) -> c_int;
    pub fn ap_server_cancel(server: *mut c_void, ticket: u64) -> c_int;
    pub fn ap_server_set_batching(server: *mut c_void, max_batch: u32) -> c_int;
    pub fn ap_server_stats(server: *mut c_void, out8: *mut u64) -> c_int;

    // radiance cache
    pub fn ap_rc_create(device: c_int, scene_lo: *const f32, scene_hi: *const f32, seed: u32, err: *mut c_int)
                        -> *mut c_void;
    pub fn ap_rc_destroy(cache: *mut c_void);
    pub fn ap_rc_last_error(cache: *const c_void) -> *const c_char;
    pub fn ap_rc_set_params(cache: *mut c_void, params: *const f32, count: u32) -> c_int;
    pub fn ap_rc_get_params(cache: *mut c_void, params: *mut f32, count: u32) -> c_int;
    pub fn ap_rc_infer(cache: *mut c_void, queries: *const f32, n: u32, out_rgb: *mut f32) -> c_int;
    pub fn ap_rc_train(cache: *mut c_void, queries: *const f32, targets: *const f32, n: u32, lr: f32, update: c_int,
                       loss: *mut f32, grad_out: *mut f32) -> c_int;
    pub fn ap_rc_wait_selftest(device: c_int, limit: c_int, out2: *mut u32) -> c_int;
    pub fn ap_rc_attach(handle: *mut c_void, cache: *mut c_void, prefix_bounces: u32, train_stride: u32,
                        train_batch: u32, lr: f32, train: c_int) -> c_int;
}
