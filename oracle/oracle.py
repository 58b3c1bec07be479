"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py load
this module; the shipped library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


class FrameConfig(ctypes.Structure):
    """Same field order as ap_frame_config (include/appearance_cuda.h) plus threads."""
    _fields_ = [(n, t) for n, t in [
        ("max_bounces", ctypes.c_uint32), ("sample_count", ctypes.c_uint32),
        ("restir_di", ctypes.c_uint32), ("restir_gi", ctypes.c_uint32), ("svgf", ctypes.c_uint32),
        ("firefly_filter", ctypes.c_uint32), ("taa", ctypes.c_uint32),
        ("di_area_samples", ctypes.c_uint32), ("di_bsdf_samples", ctypes.c_uint32),
        ("di_temporal_m_factor", ctypes.c_float),
        ("di_spatial_passes", ctypes.c_uint32), ("di_spatial_samples", ctypes.c_uint32),
        ("di_unbiased", ctypes.c_uint32),
        ("gi_temporal_m_cap", ctypes.c_float),
        ("gi_spatial_passes", ctypes.c_uint32), ("gi_spatial_samples", ctypes.c_uint32),
        ("gi_unbiased", ctypes.c_uint32),
        ("svgf_max_history", ctypes.c_uint32), ("svgf_atrous_passes", ctypes.c_uint32),
        ("taa_history_influence", ctypes.c_float),
        ("threads", ctypes.c_uint32)]]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        P, U, F = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float
        L.orc_scene_new.restype = P
        L.orc_scene_new.argtypes = [P, P, U, P, P, U, P, U, P, U, P, U, U, P]
        L.orc_scene_free.argtypes = [P]
        L.orc_closest.argtypes = [P, P, P, U, F, U, P, P]
        L.orc_any.argtypes = [P, P, P, P, U, U, P]
        L.orc_frame_new.restype = P
        L.orc_frame_new.argtypes = [P, U, U, P]
        L.orc_frame_free.argtypes = [P]
        L.orc_frame_render.argtypes = [P, P, P]
        L.orc_frame_buffer.argtypes = [P, U, P]
        L.orc_frame_rays_cast.restype = ctypes.c_uint64
        L.orc_frame_rays_cast.argtypes = [P]
        L.orc_rgb9e5_pack.restype = U
        L.orc_rgb9e5_pack.argtypes = [P]
        L.orc_rgb9e5_unpack.argtypes = [U, P]
        L.orc_oct30_pack.restype = U
        L.orc_oct30_pack.argtypes = [P]
        L.orc_oct30_unpack.argtypes = [U, P]
        for n in ("orc_pcg_hash", "orc_xor_shift"):
            getattr(L, n).restype = U
            getattr(L, n).argtypes = [U]
        L.orc_hash_combine.restype = U
        L.orc_hash_combine.argtypes = [U, U]
        L.orc_disney.argtypes = [P] * 7
        L.orc_detmath.argtypes = [U, P, P, P, U]
        L.orc_resolve_rgba8.argtypes = [P, U, U, U, P, U, P]
        L.orc_spectral_new.restype = P
        L.orc_spectral_new.argtypes = [P, P, P, P, F, F, F, P]
        L.orc_spectral_free.argtypes = [P]
        L.orc_spectral_render.argtypes = [P, P, P, U, U, U, U, U, ctypes.c_int, U, U, P]
        L.orc_two_level_new.restype = P
        L.orc_two_level_new.argtypes = [P, U, P, P, U]
        L.orc_two_level_free.argtypes = [P]
        L.orc_two_level_closest.argtypes = [P, P, P, U, F, U, P]
        L.orc_two_level_any.argtypes = [P, P, P, U, F, U, P]
        L.orc_murmur3_x64_128.argtypes = [P, ctypes.c_size_t, ctypes.c_uint64, P]
        L.orc_zsobol.argtypes = [U, U, U, ctypes.c_uint64, U, U, U, P, U, P]
        L.orc_spectral_cmf.argtypes = [F, P]
        L.orc_spectral_fit.argtypes = [P, P]
        L.orc_spectral_sigmoid.argtypes = [P, F, P]
        L.orc_spectral_wavelength.argtypes = [F, P]
        L.orc_spectral_illuminant_norm.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class OracleScene:
    def __init__(self, scene):
        L = lib()
        self._keep = dict(
            pos=np.ascontiguousarray(scene.positions, np.float32),
            nrm=np.ascontiguousarray(scene.normals, np.float32),
            idx=np.ascontiguousarray(scene.indices, np.uint32),
            tm=np.ascontiguousarray(scene.tri_material, np.uint32),
            mesh=np.ascontiguousarray(scene.meshes, np.uint32),
            mat=np.ascontiguousarray(scene.materials, np.float32),
            env=None if scene.env is None else np.ascontiguousarray(scene.env, np.float32),
            sun=np.ascontiguousarray(scene.sun, np.float32))
        k = self._keep
        env_h, env_w = (0, 0) if k["env"] is None else k["env"].shape[:2]
        self.ptr = L.orc_scene_new(_p(k["pos"]), _p(k["nrm"]), k["pos"].shape[0], _p(k["idx"]), _p(k["tm"]),
                                   k["idx"].shape[0], _p(k["mesh"]), k["mesh"].shape[0], _p(k["mat"]),
                                   k["mat"].shape[0], _p(k["env"]), env_w, env_h, _p(k["sun"]))

    def closest(self, origins, dirs, tmax=1000.0, threads=0):
        n = origins.shape[0]
        out = np.zeros((n, 4), np.float32)
        counts = np.zeros(2, np.uint64)
        lib().orc_closest(self.ptr, _p(np.ascontiguousarray(origins, np.float32)),
                          _p(np.ascontiguousarray(dirs, np.float32)), n, tmax, threads or os.cpu_count(),
                          _p(out), _p(counts))
        return out, counts

    def any(self, origins, dirs, tmax, threads=0):
        n = origins.shape[0]
        out = np.zeros(n, np.uint8)
        lib().orc_any(self.ptr, _p(np.ascontiguousarray(origins, np.float32)),
                      _p(np.ascontiguousarray(dirs, np.float32)), _p(np.ascontiguousarray(tmax, np.float32)),
                      n, threads or os.cpu_count(), _p(out))
        return out

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_scene_free(self.ptr)
            self.ptr = None


class OracleFrame:
    """Persistent frame state (reservoir, G-buffer and SVGF history) of one view."""

    def __init__(self, oscene: OracleScene, width: int, height: int, cfg: dict, threads: int = 0):
        c = FrameConfig(**{k: v for k, v in cfg.items()}, threads=threads or os.cpu_count())
        self.scene = oscene
        self.w, self.h = width, height
        self.ptr = lib().orc_frame_new(oscene.ptr, width, height, ctypes.byref(c))

    def render(self, mats: np.ndarray) -> np.ndarray:
        out = np.zeros((self.h, self.w, 3), np.float32)
        lib().orc_frame_render(self.ptr, _p(np.ascontiguousarray(mats, np.float32)), _p(out))
        return out

    def buffer(self, which: int, words: int) -> np.ndarray:
        out = np.zeros((self.h * self.w, words), np.uint32)
        lib().orc_frame_buffer(self.ptr, which, _p(out))
        return out

    def rays_cast(self) -> int:
        return int(lib().orc_frame_rays_cast(self.ptr))

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_frame_free(self.ptr)
            self.ptr = None


class OracleDisplay:
    """Display resolve state (resolve.wgsl accum_radiance / accum_frame_count):
    `resolve` takes a frame's RGB9E5 radiance words and its camera matrices and
    returns the h x w x 4 RGBA8 texture, accumulating while the camera is still
    (view_proj == prev_view_proj) and `accumulate` is set (lib.rs:349-352)."""

    def __init__(self, width: int, height: int):
        self.w, self.h = width, height
        self.accum = np.zeros((height * width, 4), np.float32)
        self.count = 0

    def resolve(self, radiance_words: np.ndarray, mats: np.ndarray, spp: int, accumulate: bool) -> np.ndarray:
        m = np.asarray(mats, np.float32).reshape(4, 16)
        if not accumulate or not np.array_equal(m[2].view(np.uint32), m[3].view(np.uint32)):
            self.accum[:] = 0.0
            self.count = 0
        out = np.zeros((self.h, self.w, 4), np.uint8)
        lib().orc_resolve_rgba8(_p(np.ascontiguousarray(radiance_words, np.uint32)), self.w, self.h, spp,
                                _p(self.accum), self.count, _p(out))
        self.count += 1
        return out


class OracleSpectral:
    """The spectral mode on the CPU (oracle_spectral.cpp) for one scene; the
    arguments mean what they mean in PathTracer.spectral_setup / render_spectral."""

    def __init__(self, oscene: OracleScene, sun_dir=(0.0, -1.0, 0.2), sun_rgb=(1.0, 1.0, 0.95), sun_scale=100.0,
                 scene_radius=1000.0, env_scale=1.0, two_level=None):
        self.scene = oscene
        self.n_mats = oscene._keep["mat"].shape[0]
        env = oscene._keep["env"]
        self.env_texels = 0 if env is None else env.shape[0] * env.shape[1]
        self.two_level = two_level  # an OracleTwoLevel of the world `oscene` flattens
        self.ptr = lib().orc_spectral_new(oscene.ptr, _p(oscene._keep["nrm"]), _p(np.asarray(sun_dir, np.float32)),
                                          _p(np.asarray(sun_rgb, np.float32)), sun_scale, scene_radius, env_scale,
                                          None if two_level is None else two_level.ptr)

    def render(self, mats: np.ndarray, width: int, height: int, spp: int = 1, max_depth: int = 4, seed: int = 0,
               row0: int = 0, row1: int | None = None, threads: int = 0) -> np.ndarray:
        row1 = height if row1 is None else row1
        m = np.ascontiguousarray(np.asarray(mats, np.float32).reshape(4, 16))
        out = np.zeros((row1 - row0, width, 3), np.float32)
        lib().orc_spectral_render(self.ptr, _p(m[0]), _p(m[1]), width, height, row0, row1, spp, max_depth, seed,
                                  threads or os.cpu_count(), _p(out))
        return out

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_spectral_free(self.ptr)
            self.ptr = None


class OracleTwoLevel:
    """Queries over instances of models (oracle_twolevel.cpp): `models` are
    model-space Scenes, `instances` (model index, column-major 4x4)."""

    def __init__(self, models, instances):
        self.models = [OracleScene(m) for m in models]
        ptrs = (ctypes.c_void_p * len(self.models))(*[m.ptr for m in self.models])
        im = np.ascontiguousarray([i for i, _ in instances], np.uint32)
        mm = np.ascontiguousarray(np.stack([np.asarray(m, np.float32).reshape(16) for _, m in instances]))
        self.ptr = lib().orc_two_level_new(ptrs, len(self.models), _p(im), _p(mm), len(instances))

    def closest(self, origins, dirs, tmax=1e30, threads=0):
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros((o.shape[0], 4), np.uint32)
        lib().orc_two_level_closest(self.ptr, _p(o), _p(d), o.shape[0], tmax, threads or os.cpu_count(), _p(out))
        return out

    def any(self, origins, dirs, tmax, threads=0):
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros(o.shape[0], np.uint8)
        lib().orc_two_level_any(self.ptr, _p(o), _p(d), o.shape[0], tmax, threads or os.cpu_count(), _p(out))
        return out

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_two_level_free(self.ptr)
            self.ptr = None


def murmur3_x64_128(data: bytes, seed: int = 0) -> tuple:
    """MurmurHash3 x64_128 of `data` as (h1, h2)."""
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    out = np.zeros(2, np.uint64)
    lib().orc_murmur3_x64_128(_p(buf), len(data), seed, _p(out))
    return int(out[0]), int(out[1])


def zsobol(res, spp, seed, pixel, sample_idx, kinds) -> np.ndarray:
    """The draws of one ZSobol sample stream (1 = get_1d, 2 = get_2d)."""
    k = np.asarray(kinds, np.uint8)
    out = np.zeros(int(k.astype(np.int64).sum()), np.float32)
    lib().orc_zsobol(res[0], res[1], spp, seed, pixel[0], pixel[1], sample_idx, _p(k), len(k), _p(out))
    return out


def spectral_cmf(lam: float) -> np.ndarray:
    out = np.zeros(4, np.float32)
    lib().orc_spectral_cmf(lam, _p(out))
    return out


def spectral_fit(rgb) -> np.ndarray:
    c = np.zeros(3, np.float32)
    lib().orc_spectral_fit(_p(np.asarray(rgb, np.float32)), _p(c))
    return c


def spectral_sigmoid(coef, lam: float) -> float:
    out = np.zeros(1, np.float32)
    lib().orc_spectral_sigmoid(_p(np.asarray(coef, np.float32)), lam, _p(out))
    return float(out[0])


def spectral_wavelength(u: float):
    out = np.zeros(2, np.float32)
    lib().orc_spectral_wavelength(u, _p(out))
    return float(out[0]), float(out[1])


def spectral_illuminant_norm() -> float:
    return float(lib().orc_spectral_illuminant_norm())


DETMATH = dict(sin=0, cos=1, exp=2, log=3, pow=4, atan2=5, acos=6)


def detmath(fn: str, x, y=None) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    yy = None if y is None else np.ascontiguousarray(y, np.float32)
    out = np.zeros_like(x)
    lib().orc_detmath(DETMATH[fn], _p(x), _p(yy), _p(out), x.size)
    return out


def rgb9e5_pack(rgb) -> int:
    a = np.ascontiguousarray(rgb, np.float32)
    return int(lib().orc_rgb9e5_pack(_p(a)))


def rgb9e5_unpack(d: int) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().orc_rgb9e5_unpack(int(d), _p(out))
    return out


def oct30_pack(v) -> int:
    a = np.ascontiguousarray(v, np.float32)
    return int(lib().orc_oct30_pack(_p(a)))


def oct30_unpack(p: int) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().orc_oct30_unpack(int(p), _p(out))
    return out


def disney(mat, n, wo, wi, r):
    """Disney evaluate (rgb, pdf) and sample (rgb, pdf, wi) at a point with normal n."""
    e = np.zeros(4, np.float32)
    smp = np.zeros(7, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (mat, n, wo, wi, r)]
    lib().orc_disney(*[_p(a) for a in args], _p(e), _p(smp))
    return e, smp
