"""ctypes binding of libappearance_cuda.so (include/appearance_cuda.h).

The library is built in-tree by appearance_b200/build.py.  Loading fails with
an exception when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libappearance_cuda.so")

AP_OK, AP_E_INVALID, AP_E_OOM, AP_E_CUDA, AP_E_TIMEOUT, AP_E_UNSUPPORTED, AP_E_NO_SCENE, AP_E_CANCELLED = range(8)

EXPORTS = ["ap_frame_config_default", "ap_create", "ap_destroy", "ap_last_error", "ap_set_config",
           "ap_world_action", "ap_scene_upload", "ap_model_register", "ap_set_camera_matrices", "ap_render_hdr", "ap_render_rgba8", "ap_render_device",
           "ap_device_framebuffer", "ap_trace_rays", "ap_trace_rays_static", "ap_read_buffer", "ap_profile_frame",
           "ap_bvh_stats", "ap_server_create", "ap_server_destroy", "ap_server_last_error", "ap_server_add_scene",
           "ap_server_job_bytes", "ap_server_submit", "ap_server_query", "ap_server_wait", "ap_server_cancel",
           "ap_server_set_batching",
           "ap_server_stats",
           "ap_rc_create", "ap_rc_destroy", "ap_rc_last_error", "ap_rc_set_params", "ap_rc_get_params", "ap_rc_infer",
           "ap_rc_train", "ap_rc_attach", "ap_rc_wait_selftest", "ap_spectral_setup", "ap_render_spectral", "ap_profile_spectral"]

U32, F32, P = ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p


class FrameConfig(ctypes.Structure):
    _fields_ = [("max_bounces", U32), ("sample_count", U32), ("restir_di", U32), ("restir_gi", U32),
                ("svgf", U32), ("firefly_filter", U32), ("taa", U32), ("di_area_samples", U32),
                ("di_bsdf_samples", U32), ("di_temporal_m_factor", F32), ("di_spatial_passes", U32),
                ("di_spatial_samples", U32), ("di_unbiased", U32), ("gi_temporal_m_cap", F32),
                ("gi_spatial_passes", U32), ("gi_spatial_samples", U32), ("gi_unbiased", U32),
                ("svgf_max_history", U32), ("svgf_atrous_passes", U32), ("taa_history_influence", F32)]


class Mesh(ctypes.Structure):
    _fields_ = [("first_vertex", U32), ("num_vertices", U32), ("first_index", U32), ("num_indices", U32),
                ("material_idx", U32), ("emissive", U32)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("positions", P), ("normals", P), ("num_vertices", U32), ("indices", P), ("tri_material", P),
                ("num_tris", U32), ("meshes", P), ("num_meshes", U32), ("materials", P), ("num_materials", U32),
                ("env", P), ("env_w", U32), ("env_h", U32), ("sun", F32 * 8)]


class FrameStats(ctypes.Structure):
    _fields_ = [("gpu_ms", ctypes.c_double), ("extension_rays", ctypes.c_uint64), ("width", U32),
                ("height", U32), ("frame_idx", U32), ("kernel_launches", U32)]


class Job(ctypes.Structure):
    _fields_ = [("scene", U32), ("width", U32), ("height", U32), ("spp", U32), ("max_depth", U32), ("seed", U32),
                ("deadline_ms", U32), ("mats", F32 * 64)]


class JobResult(ctypes.Structure):
    _fields_ = [("queued_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("gpu_ms", ctypes.c_double),
                ("device_bytes", ctypes.c_uint64), ("graph_mode", U32), ("slot", U32), ("batch", U32),
                ("pad", U32)]


_lib = None


def load() -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python appearance_b200/build.py` (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    L.ap_frame_config_default.argtypes = [ctypes.POINTER(FrameConfig)]
    L.ap_create.restype = P
    L.ap_create.argtypes = [ctypes.POINTER(FrameConfig), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.ap_destroy.argtypes = [P]
    L.ap_last_error.restype = ctypes.c_char_p
    L.ap_last_error.argtypes = [P]
    L.ap_set_config.argtypes = [P, ctypes.POINTER(FrameConfig)]
    L.ap_world_action.argtypes = [P, U32, P, ctypes.c_size_t]
    L.ap_scene_upload.argtypes = [P, ctypes.POINTER(SceneDesc)]
    L.ap_model_register.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(SceneDesc)]
    L.ap_set_camera_matrices.argtypes = [P, P]
    L.ap_render_hdr.argtypes = [P, U32, U32, U32, U32, P, ctypes.c_size_t, ctypes.POINTER(FrameStats)]
    L.ap_render_rgba8.argtypes = [P, U32, U32, U32, U32, ctypes.c_int, P, ctypes.c_size_t, ctypes.POINTER(FrameStats)]
    L.ap_render_device.argtypes = [P, U32, U32, ctypes.POINTER(FrameStats)]
    L.ap_device_framebuffer.restype = P
    L.ap_device_framebuffer.argtypes = [P]
    L.ap_trace_rays.argtypes = [P, P, P, U32, ctypes.c_int, P]
    L.ap_trace_rays_static.argtypes = [P, P, P, U32, ctypes.c_int, P]
    L.ap_read_buffer.argtypes = [P, U32, P, ctypes.c_size_t]
    L.ap_bvh_stats.argtypes = [P, P]
    L.ap_rc_wait_selftest.argtypes = [ctypes.c_int, ctypes.c_int, P]
    L.ap_spectral_setup.argtypes = [P, P, P, F32, F32, F32]
    L.ap_render_spectral.argtypes = [P, U32, U32, U32, U32, U32, U32, U32, P, ctypes.c_size_t,
                                     ctypes.POINTER(FrameStats)]
    L.ap_profile_spectral.argtypes = [P, U32, U32, U32, U32, U32, U32, U32, P, ctypes.POINTER(FrameStats)]
    L.ap_profile_frame.argtypes = [P, U32, U32, P, P, P, U32, P, ctypes.c_int, P, ctypes.POINTER(FrameStats)]
    L.ap_server_create.restype = P
    L.ap_server_create.argtypes = [ctypes.POINTER(FrameConfig), ctypes.c_int, ctypes.c_uint64, U32, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int)]
    L.ap_server_destroy.argtypes = [P]
    L.ap_server_last_error.restype = ctypes.c_char_p
    L.ap_server_last_error.argtypes = [P]
    L.ap_server_add_scene.argtypes = [P, ctypes.POINTER(SceneDesc), ctypes.POINTER(U32)]
    L.ap_server_job_bytes.restype = ctypes.c_uint64
    L.ap_server_job_bytes.argtypes = [U32, U32]
    L.ap_server_submit.argtypes = [P, ctypes.POINTER(Job), P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]
    L.ap_server_query.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)]
    L.ap_server_wait.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(JobResult)]
    L.ap_server_cancel.argtypes = [P, ctypes.c_uint64]
    L.ap_server_set_batching.argtypes = [P, U32]
    L.ap_server_stats.argtypes = [P, P]
    L.ap_rc_create.restype = P
    L.ap_rc_create.argtypes = [ctypes.c_int, P, P, U32, ctypes.POINTER(ctypes.c_int)]
    L.ap_rc_destroy.argtypes = [P]
    L.ap_rc_last_error.restype = ctypes.c_char_p
    L.ap_rc_last_error.argtypes = [P]
    L.ap_rc_set_params.argtypes = [P, P, U32]
    L.ap_rc_get_params.argtypes = [P, P, U32]
    L.ap_rc_infer.argtypes = [P, P, U32, P]
    L.ap_rc_train.argtypes = [P, P, P, U32, F32, ctypes.c_int, P, P]
    L.ap_rc_attach.argtypes = [P, P, U32, U32, U32, F32, ctypes.c_int]
    _lib = L
    return L
