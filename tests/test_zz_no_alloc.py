"""ap_trace_rays_static, the ray query for callers that may not allocate device
memory (a host that owns the whole device-memory budget, or a thread that
cannot take cudaMalloc's device-wide synchronisation).  Its device staging is a
fixed static array of the library, so it must give exactly the hits of the
allocating entry point ap_trace_rays, call after call, and refuse batches
larger than the array.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from appearance_b200 import PathTracer, _native, presets, scenes

pytestmark = pytest.mark.gpu

STATIC_MAX_RAYS = 65536


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _rays(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    o = np.zeros((n, 4), np.float32)
    o[:, :3] = rng.uniform(lo, hi, (n, 3))
    o[:, 3] = rng.uniform(0.5, 1000.0, n)
    d = np.zeros((n, 4), np.float32)
    v = rng.normal(size=(n, 3))
    d[:, :3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    return o, d


def _call(lib, fn, h, o, d, any_hit):
    out = np.zeros((o.shape[0], 4), np.uint32)
    rc = getattr(lib, fn)(h, _ptr(o), _ptr(d), o.shape[0], any_hit, _ptr(out))
    assert rc == _native.AP_OK, lib.ap_last_error(h).decode()
    return out


def _free_device_bytes():
    # the CUDA runtime the library itself loaded (already mapped in this process)
    rt = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def test_static_scratch_query_matches_allocating_query():
    lib = _native.load()
    sc = scenes.icosphere_field(seed=4, num_spheres=64, num_emissive=4, subdiv=2, box=12.0, env_size=None)
    pt = PathTracer(presets.FAITHFUL)
    pt.upload_scene(sc)
    h = pt._h
    batches = [(STATIC_MAX_RAYS, 0), (40000, 1)]
    rays = [_rays(n, 100 + call, -2.0, 14.0) for call, (n, _) in enumerate(batches)]
    refs = [_call(lib, "ap_trace_rays", h, o, d, any_hit) for (o, d), (_, any_hit) in zip(rays, batches)]
    for call, ((o, d), (n, any_hit), ref) in enumerate(zip(rays, batches, refs)):  # two calls in a row
        free_before = _free_device_bytes()
        got = _call(lib, "ap_trace_rays_static", h, o, d, any_hit)
        free_after = _free_device_bytes()
        assert np.array_equal(got, ref), f"call {call}: {(got != ref).any(1).sum()} rays differ"
        if not any_hit:
            assert (got[:, 3] != 0xFFFFFFFF).mean() > 0.05
        if call > 0:  # the first call may load the library's device code; later calls change nothing
            assert free_after == free_before, f"call {call}: device memory changed by {free_before - free_after} B"


def test_static_scratch_query_rejects_oversized_batches():
    lib = _native.load()
    pt = PathTracer(presets.FAITHFUL)
    pt.upload_scene(scenes.cornell_box())
    o, d = _rays(STATIC_MAX_RAYS + 1, 7, 0.1, 0.9)
    out = np.zeros((o.shape[0], 4), np.uint32)
    rc = lib.ap_trace_rays_static(pt._h, _ptr(o), _ptr(d), o.shape[0], 0, _ptr(out))
    assert rc == _native.AP_E_INVALID
    assert b"static scratch limit" in lib.ap_last_error(pt._h)
