"""Host-side mirror of the reference's renderer interface.

`PathTracer` follows PathTracerGpu (crates/appearance-path-tracer-gpu/src/
lib.rs:247-615) and the NodeRenderer trait it is used through
(crates/appearance-render-loop/src/node.rs:14-25):

    handle_visible_world_action(ty, bytes)     NodeRenderer::visible_world_action
    render(resolution, start_row, end_row, cb) NodeRenderer::render

plus the calls a synthetic-scene host needs (upload_scene, set_camera).  All
work runs in libappearance_cuda.so on the GPU; errors raise RendererError with
the library's message.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _native, presets
from .scenes import Scene, camera_matrices


class RendererError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def config_struct(cfg: dict | None) -> _native.FrameConfig:
    c = _native.FrameConfig()
    _native.load().ap_frame_config_default(ctypes.byref(c))
    for k, v in (cfg or {}).items():
        setattr(c, k, v)
    return c


def scene_desc(scene: Scene):
    """ap_scene_desc for a Scene, and the arrays it points into (keep them alive
    until the upload returns)."""
    keep = dict(pos=np.ascontiguousarray(scene.positions, np.float32),
                nrm=np.ascontiguousarray(scene.normals, np.float32),
                idx=np.ascontiguousarray(scene.indices, np.uint32),
                tm=np.ascontiguousarray(scene.tri_material, np.uint32),
                mesh=np.ascontiguousarray(scene.meshes, np.uint32),
                mat=np.ascontiguousarray(scene.materials, np.float32),
                env=None if scene.env is None else np.ascontiguousarray(scene.env, np.float32))
    d = _native.SceneDesc()
    d.positions, d.normals = _ptr(keep["pos"]), _ptr(keep["nrm"])
    d.num_vertices = keep["pos"].shape[0]
    d.indices, d.tri_material = _ptr(keep["idx"]), _ptr(keep["tm"])
    d.num_tris = keep["idx"].shape[0]
    d.meshes, d.num_meshes = _ptr(keep["mesh"]), keep["mesh"].shape[0]
    d.materials, d.num_materials = _ptr(keep["mat"]), keep["mat"].shape[0]
    if keep["env"] is not None:
        d.env, d.env_h, d.env_w = _ptr(keep["env"]), keep["env"].shape[0], keep["env"].shape[1]
    for i in range(8):
        d.sun[i] = float(scene.sun[i])
    return d, keep


class PathTracer:
    """One renderer instance (one CUDA stream, persistent temporal state)."""

    def __init__(self, config: dict | None = None, device: int = 0):
        self._lib = _native.load()
        err = ctypes.c_int(0)
        self._cfg = config_struct(config if config is not None else presets.FAITHFUL)
        self._h = self._lib.ap_create(ctypes.byref(self._cfg), device, ctypes.byref(err))
        if not self._h:
            raise RendererError(err.value, "ap_create failed (no CUDA device?)")
        self._scene_keep = None
        self._eye = None
        self.last_stats = _native.FrameStats()

    # -- error plumbing
    def _check(self, rc: int):
        if rc != _native.AP_OK:
            raise RendererError(rc, self._lib.ap_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ap_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # -- configuration
    def set_config(self, config: dict):
        self._cfg = config_struct(config)
        self._check(self._lib.ap_set_config(self._h, ctypes.byref(self._cfg)))

    # -- world
    def handle_visible_world_action(self, ty: int, data: bytes):
        """VisibleWorldActionType::from_ty_and_bytes wire format (visible_world_action.rs:87-96)."""
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        self._check(self._lib.ap_world_action(self._h, ty, buf, len(data)))

    @staticmethod
    def camera_update_bytes(transform_col_major, fov_deg: float, near: float, far: float) -> bytes:
        """Packs CameraUpdateData {Mat4, fov, near, far, pad} (visible_world_action.rs:9-15)."""
        m = np.asarray(transform_col_major, np.float32).reshape(16)
        return m.tobytes() + struct.pack("<fffI", fov_deg, near, far, 0)

    def upload_scene(self, scene: Scene):
        d, self._scene_keep = scene_desc(scene)
        self._check(self._lib.ap_scene_upload(self._h, ctypes.byref(d)))

    def register_model(self, asset_path: str, model: Scene):
        """ap_model_register: the geometry SpawnModel instantiates by `asset_path`
        (model space; a glTF file read by appearance_b200.gltf, for example)."""
        d, keep = scene_desc(model)
        self._check(self._lib.ap_model_register(self._h, asset_path.encode(), ctypes.byref(d)))
        del keep

    @staticmethod
    def spawn_model_bytes(transform_col_major, entity_uuid: bytes, asset_path: str) -> bytes:
        """SpawnModelData {Mat4, Uuid, [u8; 256]} (visible_world_action.rs:17-48)."""
        p = asset_path.encode()
        if len(p) > 255 or len(entity_uuid) != 16:
            raise ValueError("asset path of at most 255 bytes and a 16-byte uuid")
        m = np.asarray(transform_col_major, np.float32).reshape(16)
        return m.tobytes() + bytes(entity_uuid) + p + bytes(256 - len(p))

    @staticmethod
    def transform_model_bytes(transform_col_major, entity_uuid: bytes) -> bytes:
        """TransformModelData {Mat4, Uuid} (visible_world_action.rs:50-55)."""
        if len(entity_uuid) != 16:
            raise ValueError("16-byte uuid")
        return np.asarray(transform_col_major, np.float32).reshape(16).tobytes() + bytes(entity_uuid)

    def spawn_model(self, entity_uuid: bytes, asset_path: str, transform_col_major):
        self.handle_visible_world_action(1, self.spawn_model_bytes(transform_col_major, entity_uuid, asset_path))

    def transform_model(self, entity_uuid: bytes, transform_col_major):
        self.handle_visible_world_action(2, self.transform_model_bytes(transform_col_major, entity_uuid))

    def destroy_model(self, entity_uuid: bytes):
        self.handle_visible_world_action(3, bytes(entity_uuid))

    def clear(self):
        self.handle_visible_world_action(4, struct.pack("<I", 0))

    def set_camera_matrices(self, mats: np.ndarray):
        m = np.ascontiguousarray(mats, np.float32).reshape(64)
        self._check(self._lib.ap_set_camera_matrices(self._h, _ptr(m)))

    def set_camera(self, eye, target, fov, near, far, width, height, prev_view_proj=None):
        """Look-at camera; returns this frame's view_proj (float64) for the next frame's motion."""
        mats, vp = camera_matrices(eye, target, fov, near, far, width, height, prev_view_proj)
        self.set_camera_matrices(mats)
        return vp

    # -- rendering
    def render(self, resolution, start_row: int = 0, end_row: int | None = None, result_callback=None,
               out: np.ndarray | None = None) -> np.ndarray:
        """NodeRenderer::render: linear HDR RGB f32 rows [start_row, end_row) of a
        resolution=(width, height) frame.  The callback, when given, receives the
        rows as bytes (the reference passes &[u8]) and the array is returned.
        `out` (C-contiguous float32 of shape (rows, width, 3)) is filled instead
        of a new array; a page-locked one (e.g. from torch's pin_memory) makes
        the device-to-host copy run at full PCIe/C2C speed."""
        w, h = int(resolution[0]), int(resolution[1])
        end_row = h if end_row is None else end_row
        if out is None:
            out = np.empty((max(0, end_row - start_row), w, 3), np.float32)
        elif out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"] or out.shape != (end_row - start_row, w, 3):
            raise ValueError("out must be C-contiguous float32 of shape (rows, width, 3)")
        self._check(self._lib.ap_render_hdr(self._h, w, h, start_row, end_row, _ptr(out), out.nbytes,
                                            ctypes.byref(self.last_stats)))
        if result_callback is not None:
            result_callback(out.tobytes())
        return out

    def attach_radiance_cache(self, cache, prefix_bounces: int = 2, train_stride: int = 16, train_batch: int = 65536,
                              lr: float = 1e-3, train: bool = True):
        """Radiance-cache mode (ap_rc_attach); `cache` None detaches."""
        self._rc = cache
        self._check(self._lib.ap_rc_attach(self._h, None if cache is None else cache._c, prefix_bounces, train_stride,
                                           train_batch, lr, 1 if train else 0))

    def render_rgba8(self, resolution, start_row: int = 0, end_row: int | None = None, accumulate: bool = False,
                     result_callback=None) -> np.ndarray:
        """The reference's byte output: ACES-tonemapped RGBA8 at 64x64-block-swizzled
        positions (rows [start_row, end_row) of the texture)."""
        w, h = int(resolution[0]), int(resolution[1])
        end_row = h if end_row is None else end_row
        out = np.zeros((end_row - start_row, w, 4), np.uint8)
        self._check(self._lib.ap_render_rgba8(self._h, w, h, start_row, end_row, 1 if accumulate else 0, _ptr(out),
                                              out.nbytes, ctypes.byref(self.last_stats)))
        if result_callback is not None:
            result_callback(out.tobytes())
        return out

    def render_device(self, width: int, height: int) -> float:
        """Renders into the device framebuffer only; returns the frame's GPU ms."""
        self._check(self._lib.ap_render_device(self._h, width, height, ctypes.byref(self.last_stats)))
        return self.last_stats.gpu_ms

    def device_framebuffer_ptr(self) -> int:
        return int(self._lib.ap_device_framebuffer(self._h) or 0)

    def trace_rays(self, origins: np.ndarray, dirs: np.ndarray, tmax, any_hit: bool = False) -> np.ndarray:
        """Closest (t, u, v, tri) or any-hit queries; returns (n, 4) uint32 words."""
        n = origins.shape[0]
        o4 = np.zeros((n, 4), np.float32)
        o4[:, :3] = origins
        o4[:, 3] = tmax
        d4 = np.zeros((n, 4), np.float32)
        d4[:, :3] = dirs
        out = np.zeros((n, 4), np.uint32)
        self._check(self._lib.ap_trace_rays(self._h, _ptr(o4), _ptr(d4), n, 1 if any_hit else 0, _ptr(out)))
        return out

    def read_buffer(self, which: int, words: int, pixels: int) -> np.ndarray:
        out = np.zeros((pixels, words), np.uint32)
        self._check(self._lib.ap_read_buffer(self._h, which, _ptr(out), out.nbytes))
        return out

    def profile_frame(self, width: int, height: int, count_visits: bool = False) -> dict:
        """Renders one frame with per-kernel events.  Returns {kind: dict(ms, launches,
        rays, nodes, tris)}; rays/nodes/tris are filled for the traversal kernels
        when count_visits (instrumented kernels, times then not representative)."""
        n = 32
        ms = np.zeros(n, np.float64)
        cnt = np.zeros(n, np.uint32)
        names = (ctypes.c_char_p * n)()
        nk = np.zeros(1, np.uint32)
        visits = np.zeros(3 * n, np.uint64)
        self._check(self._lib.ap_profile_frame(self._h, width, height, _ptr(ms), _ptr(cnt), names, n, _ptr(nk),
                                               1 if count_visits else 0, _ptr(visits),
                                               ctypes.byref(self.last_stats)))
        return {names[i].decode(): dict(ms=float(ms[i]), launches=int(cnt[i]), rays=int(visits[3 * i]),
                                        nodes=int(visits[3 * i + 1]), tris=int(visits[3 * i + 2]))
                for i in range(int(nk[0]))}

    # -- spectral mode (the CPU tracer's estimator, crates/appearance-path-tracer)
    SUN_DIR = (0.0, -1.0, 0.2)  # DistantLight::new in GeometryResources::new (geometry_resources.rs:52-64)
    SUN_RGB = (1.0, 1.0, 0.95)

    def spectral_setup(self, sun_dir=SUN_DIR, sun_rgb=SUN_RGB, sun_scale: float = 100.0, scene_radius: float = 1000.0,
                       env_scale: float = 1.0):
        """Builds the spectral tables of the uploaded scene (ap_spectral_setup)."""
        d = np.asarray(sun_dir, np.float32).reshape(3)
        c = np.asarray(sun_rgb, np.float32).reshape(3)
        self._check(self._lib.ap_spectral_setup(self._h, _ptr(d), _ptr(c), sun_scale, scene_radius, env_scale))

    def render_spectral(self, resolution, spp: int = 1, max_depth: int = 4, seed: int = 0, start_row: int = 0,
                        end_row: int | None = None, to_host: bool = True):
        """Hero-wavelength render: linear sRGB f32 rows [start_row, end_row), mean
        of `spp` paths per pixel (to_host False keeps it on the device and
        returns None; last_stats.gpu_ms holds the kernel time)."""
        w, h = int(resolution[0]), int(resolution[1])
        end_row = h if end_row is None else end_row
        out = np.empty((max(0, end_row - start_row), w, 3), np.float32) if to_host else None
        self._check(self._lib.ap_render_spectral(self._h, w, h, start_row, end_row, spp, max_depth, seed,
                                                 _ptr(out) if to_host else None, out.nbytes if to_host else 0,
                                                 ctypes.byref(self.last_stats)))
        return out

    def profile_spectral(self, resolution, spp: int = 1, max_depth: int = 4, seed: int = 0, start_row: int = 0,
                         end_row: int | None = None) -> dict:
        """render_spectral with instrumented traversal: rays, nodes and triangles
        of the closest-hit and the shadow rays (times not representative)."""
        w, h = int(resolution[0]), int(resolution[1])
        end_row = h if end_row is None else end_row
        v = np.zeros(6, np.uint64)
        self._check(self._lib.ap_profile_spectral(self._h, w, h, start_row, end_row, spp, max_depth, seed, _ptr(v),
                                                  ctypes.byref(self.last_stats)))
        return {"closest": dict(rays=int(v[0]), nodes=int(v[1]), tris=int(v[2])),
                "any": dict(rays=int(v[3]), nodes=int(v[4]), tris=int(v[5]))}

    def bvh_stats(self) -> dict:
        out = np.zeros(8, np.uint32)
        self._check(self._lib.ap_bvh_stats(self._h, _ptr(out)))
        return dict(nodes=int(out[0]), tris=int(out[1]), max_depth=int(out[2]), max_stack=int(out[3]),
                    build_ms=float(out[4:6].view(np.float64)[0]))
