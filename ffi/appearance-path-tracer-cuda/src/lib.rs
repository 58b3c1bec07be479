//! `PathTracerCuda`: the reference's `NodeRenderer` (crates/appearance-render-
//! loop/src/node.rs:14-25) over libappearance_cuda, a drop-in for
//! `DistributedRenderer` (crates/appearance-distributed-renderer/src/lib.rs:
//! 60-82) at its call sites (`Node::start_render`, node.rs:44-105, and the
//! render host's local branch, apps/render-host/src/lib.rs:331-366).
//!
//! World actions go to the library byte for byte (`ap_world_action`, the
//! wire format of `VisibleWorldActionType::from_ty_and_bytes`); `render`
//! returns the reference's byte output (ACES-fit RGBA8 at 64x64-block-swizzled
//! positions, resolve.wgsl:29-59, block.wgsl:3-16) through the same borrowed-
//! slice callback.  Models that SpawnModel names are registered first with
//! `register_model` (the host loads them, as the reference's asset database
//! does, and passes their geometry).  Errors never abort: they are logged, as
//! the reference logs failed world actions.

pub mod ffi;

use std::ffi::{CStr, CString};
use std::os::raw::c_void;

use appearance_render_loop::node::NodeRenderer;
use appearance_world::visible_world_action::VisibleWorldActionType;
use glam::UVec2;

/// One model or scene in the library's flat layout (ap_scene_desc): a vertex
/// pool, meshes as contiguous index ranges, per-triangle material indices
/// relative to the mesh's first material, and materials.
pub struct Geometry<'a> {
    pub positions: &'a [[f32; 3]],
    pub normals: &'a [[f32; 3]],
    pub indices: &'a [[u32; 3]],
    pub tri_material: &'a [u32],
    pub meshes: &'a [ffi::ApMesh],
    pub materials: &'a [ffi::ApMaterial],
    /// equirect RGB f32 environment (width, height, texels), scenes only
    pub env: Option<(u32, u32, &'a [[f32; 3]])>,
    /// SunInfo: direction xyz, size, colour xyz, intensity
    pub sun: [f32; 8],
}

impl Geometry<'_> {
    fn desc(&self) -> ffi::ApSceneDesc {
        let (env_w, env_h, env) = match self.env {
            Some((w, h, t)) => (w, h, t.as_ptr() as *const f32),
            None => (0, 0, std::ptr::null()),
        };
        ffi::ApSceneDesc {
            positions: self.positions.as_ptr() as *const f32,
            normals: self.normals.as_ptr() as *const f32,
            num_vertices: self.positions.len() as u32,
            indices: self.indices.as_ptr() as *const u32,
            tri_material: self.tri_material.as_ptr(),
            num_tris: self.indices.len() as u32,
            meshes: self.meshes.as_ptr(),
            num_meshes: self.meshes.len() as u32,
            materials: self.materials.as_ptr(),
            num_materials: self.materials.len() as u32,
            env,
            env_w,
            env_h,
            sun: self.sun,
        }
    }
}

pub struct PathTracerCuda {
    handle: *mut c_void,
    rgba: Vec<u8>,
    /// PathTracerGpuConfig::accum_frames: average still-camera frames
    pub accumulate: bool,
}

// The handle is used by one thread at a time (the node's render thread).
unsafe impl Send for PathTracerCuda {}

impl PathTracerCuda {
    /// PathTracerGpu::new with the reference's default configuration on `device`.
    pub fn new(device: i32) -> Result<Self, String> {
        let mut cfg = ffi::ApFrameConfig::default();
        unsafe { ffi::ap_frame_config_default(&mut cfg) };
        Self::with_config(&cfg, device)
    }

    pub fn with_config(cfg: &ffi::ApFrameConfig, device: i32) -> Result<Self, String> {
        let mut err = 0;
        let handle = unsafe { ffi::ap_create(cfg, device, &mut err) };
        if handle.is_null() {
            return Err(format!("ap_create failed with status {err}"));
        }
        Ok(Self { handle, rgba: Vec::new(), accumulate: false })
    }

    fn status(&self, rc: i32) -> Result<(), String> {
        if rc == ffi::AP_OK {
            Ok(())
        } else {
            let msg = unsafe { CStr::from_ptr(ffi::ap_last_error(self.handle)) };
            Err(format!("appearance-cuda ({rc}): {}", msg.to_string_lossy()))
        }
    }

    /// The base scene (environment, sun and any static geometry).
    pub fn upload_scene(&mut self, scene: &Geometry) -> Result<(), String> {
        let d = scene.desc();
        self.status(unsafe { ffi::ap_scene_upload(self.handle, &d) })
    }

    /// The geometry SpawnModel instantiates by `asset_path`.
    pub fn register_model(&mut self, asset_path: &str, model: &Geometry) -> Result<(), String> {
        let path = CString::new(asset_path).map_err(|e| e.to_string())?;
        let d = model.desc();
        self.status(unsafe { ffi::ap_model_register(self.handle, path.as_ptr(), &d) })
    }

    /// Linear HDR RGB f32 rows (before the reference's tonemap).
    pub fn render_hdr(&mut self, resolution: UVec2, start_row: u32, end_row: u32, out: &mut [f32])
                      -> Result<ffi::ApFrameStats, String> {
        let mut stats = ffi::ApFrameStats::default();
        let rc = unsafe {
            ffi::ap_render_hdr(self.handle, resolution.x, resolution.y, start_row, end_row, out.as_mut_ptr(),
                               std::mem::size_of_val(out), &mut stats)
        };
        self.status(rc).map(|_| stats)
    }
}

impl NodeRenderer for PathTracerCuda {
    fn visible_world_action(&mut self, action: &VisibleWorldActionType) {
        // the (ty, bytes) pair of the wire format (visible_world_action.rs:74-84,110-118)
        let ty: u32 = (*action).into();
        let bytes = action.as_bytes();
        let rc = unsafe { ffi::ap_world_action(self.handle, ty, bytes.as_ptr() as *const c_void, bytes.len()) };
        if let Err(e) = self.status(rc) {
            log::warn!("{e}");
        }
    }

    fn render<F: FnMut(&[u8])>(&mut self, resolution: UVec2, start_row: u32, end_row: u32, mut result_callback: F) {
        let rows = end_row.saturating_sub(start_row) as usize;
        self.rgba.resize(rows * resolution.x as usize * 4, 0);
        let mut stats = ffi::ApFrameStats::default();
        let rc = unsafe {
            ffi::ap_render_rgba8(self.handle, resolution.x, resolution.y, start_row, end_row,
                                 self.accumulate as i32, self.rgba.as_mut_ptr(), self.rgba.len(), &mut stats)
        };
        if let Err(e) = self.status(rc) {
            log::warn!("{e}");
        }
        result_callback(&self.rgba);
    }
}

impl Drop for PathTracerCuda {
    fn drop(&mut self) {
        unsafe { ffi::ap_destroy(self.handle) }
    }
}
