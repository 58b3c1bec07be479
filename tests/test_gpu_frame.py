"""CUDA frame vs the oracle under identical PCG streams.

The arithmetic contract of the path-tracing stages (no contraction, IEEE
division and square root, detmath.h elementary functions, same evaluation
order) makes them a bit-exact function of their inputs: every per-pixel state
buffer (path payload, G-buffer, DI/GI reservoirs, light-sample context, rays)
must be identical to the oracle's, frame after frame, and so must frames
without the SVGF a-trous passes and TAA.  Frames through those passes, whose
kernels use hardware exp and fused multiply-adds, are held to the tolerance
stated in tests/parity.py."""
import os

import numpy as np
import pytest

from appearance_b200 import PathTracer, presets, scenes
from oracle.oracle import OracleFrame, OracleScene
from parity import assert_bits, assert_frame, assert_post_close, rgb9e5_to_rgb, uses_post_tolerance

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BUFFERS = {0: ("radiance", 1, 1), 1: ("payload", 4, 3), 2: ("gbuffer", 8, 6), 3: ("di", 8, 8),
           4: ("gi", 8, 8), 5: ("ctx", 4, 4), 7: ("rays", 4, 4)}


def load_golden_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def compare_state(pt, of, w, h, cfg):
    for which, (name, gw, ow) in BUFFERS.items():
        g = pt.read_buffer(which, gw, w * h)[:, :ow]
        if name == "radiance" and uses_post_tolerance(cfg):  # remodulated output of the denoise chain
            assert_post_close(rgb9e5_to_rgb(g), rgb9e5_to_rgb(of.buffer(which, ow)), name)
        else:
            assert_bits(g, of.buffer(which, ow), name)


@pytest.mark.parametrize("name", ["cornell_plain_32", "spheres_realtime_48x32"])
def test_golden_fixture(name):
    mg = load_golden_module()
    sc, cfg, mats, w, h, images = mg.load_case(name)
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    for f in range(len(mats)):
        pt.set_camera_matrices(mats[f])
        assert_frame(pt.render((w, h)), images[f], cfg, f"{name} frame {f}")


@pytest.mark.parametrize("preset,override", [
    ("plain", dict(sample_count=2)), ("faithful", {}), ("faithful", dict(restir_di=0)),
    ("faithful", dict(di_unbiased=0, gi_unbiased=0)), ("faithful", dict(di_spatial_passes=2)),
    ("realtime", dict(max_bounces=3)), ("realtime_gi_spatial", dict(max_bounces=4, gi_spatial_passes=2)),
])
def test_cornell_sequences_match_oracle(preset, override):
    sc = scenes.cornell_box()
    cfg = dict(presets.PRESETS[preset], **override)
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    of = OracleFrame(OracleScene(sc), 40, 36, cfg)
    cam = scenes.cornell_camera()
    prev = None
    for f in range(3):
        eye = np.asarray(cam["eye"]) + np.array([0.01 * f, -0.005 * f, 0.0])
        mats, prev = scenes.camera_matrices(eye, cam["target"], cam["fov"], cam["near"], cam["far"], 40, 36, prev)
        pt.set_camera_matrices(mats)
        assert_frame(pt.render((40, 36)), of.render(mats), cfg, f"{preset} frame {f}")
    compare_state(pt, of, 40, 36, cfg)


@pytest.mark.parametrize("w,h", [(1, 1), (17, 9), (64, 3), (3, 70), (129, 65)])
def test_ragged_resolutions(w, h):
    sc = scenes.icosphere_field(seed=2, num_spheres=32, num_emissive=4, subdiv=2, box=10.0, env_size=(32, 16))
    cfg = dict(presets.REALTIME_GI_SPATIAL, max_bounces=3)
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    of = OracleFrame(OracleScene(sc), w, h, cfg)
    path = scenes.camera_spline(seed=2, frames=8, box=10.0)
    prev = None
    for f in range(2):
        mats, prev = scenes.camera_matrices(path[f][0], path[f][1], 60.0, 0.01, 500.0, w, h, prev)
        pt.set_camera_matrices(mats)
        assert_frame(pt.render((w, h)), of.render(mats), cfg, f"{w}x{h} frame {f}")
    compare_state(pt, of, w, h, cfg)


def test_benchmark_scene_small_view():
    """The full 1.31M-triangle benchmark scene and preset at 96x54, 3 frames."""
    sc = scenes.icosphere_field(seed=0, env_size=(512, 256))
    cfg = dict(presets.REALTIME)
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    of = OracleFrame(OracleScene(sc), 96, 54, cfg)
    path = scenes.camera_spline(seed=0, frames=64)
    prev = None
    for f in range(3):
        mats, prev = scenes.camera_matrices(path[f][0], path[f][1], 60.0, 0.01, 1000.0, 96, 54, prev)
        pt.set_camera_matrices(mats)
        assert_frame(pt.render((96, 54)), of.render(mats), cfg, f"benchmark scene frame {f}")
    compare_state(pt, of, 96, 54, cfg)


def test_row_range_is_a_crop():
    sc = scenes.cornell_box()
    cam = scenes.cornell_camera()
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], 48, 40)
    a = PathTracer(presets.PLAIN)
    a.upload_scene(sc)
    a.set_camera_matrices(mats)
    full = a.render((48, 40))
    b = PathTracer(presets.PLAIN)
    b.upload_scene(sc)
    b.set_camera_matrices(mats)
    assert_bits(b.render((48, 40), 7, 29), full[7:29], "row range")


@pytest.mark.parametrize("accumulate", [False, True])
def test_rgba8_display_output_matches_oracle(accumulate):
    """ap_render_rgba8 (the reference's byte output): ACES fit, accumulation
    while the camera is still, 64x64-block-swizzled RGBA8, bit-exact."""
    from oracle.oracle import OracleDisplay
    sc = scenes.cornell_box()
    cfg = dict(presets.PRESETS["faithful"])
    w, h = 128, 96  # one full and one partial block row: swizzled positions past the texture are dropped
    cam = scenes.cornell_camera()
    eye, tgt = np.array(cam["eye"]), np.array(cam["target"])
    args = (cam["fov"], cam["near"], cam["far"], w, h)
    m0, vp0 = scenes.camera_matrices(eye, tgt, *args, None)  # prev == current: a still camera
    moved, vp1 = scenes.camera_matrices(eye + np.array([0.01, 0.0, 0.0]), tgt, *args, vp0)
    still, _ = scenes.camera_matrices(eye + np.array([0.01, 0.0, 0.0]), tgt, *args, vp1)
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    of = OracleFrame(OracleScene(sc), w, h, cfg)
    disp = OracleDisplay(w, h)
    for m in (m0, m0, m0, moved, still, still):
        m = np.array(m, np.float32)
        pt.set_camera_matrices(m)
        img = pt.render_rgba8((w, h), accumulate=accumulate)
        of.render(m)
        ref = disp.resolve(of.buffer(0, 1)[:, 0], m, cfg["sample_count"], accumulate)
        assert np.array_equal(img, ref)
    part = pt.render_rgba8((w, h), start_row=32, end_row=80, accumulate=accumulate)
    assert part.shape == (48, w, 4)


def test_render_into_caller_buffer():
    sc = scenes.cornell_box()
    cam = scenes.cornell_camera()
    w, h = 40, 24
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], w, h)
    a = PathTracer(presets.PLAIN)
    a.upload_scene(sc)
    a.set_camera_matrices(mats)
    b = PathTracer(presets.PLAIN)
    b.upload_scene(sc)
    b.set_camera_matrices(mats)
    import torch
    out = torch.empty((h, w, 3), dtype=torch.float32, pin_memory=True).numpy()
    ref = a.render((w, h))
    got = b.render((w, h), out=out)
    assert got is out
    assert_bits(out, ref, "pinned caller buffer")
    part = np.zeros((7, w, 3), np.float32)
    b.set_camera_matrices(mats)
    with pytest.raises(ValueError):
        b.render((w, h), 3, 12, out=part)
    a.close()
    b.close()


def test_second_stream_frames_equal_one_stream_frames():
    """A render traces the DI shadow rays of every bounce but the last on the
    handle's second stream, beside the next bounce's extension; a profiled frame
    runs every launch on one stream.  Both orders leave every per-path state
    buffer bit-identical, frame after frame (320x180, the benchmark scene and
    preset)."""
    sc = scenes.icosphere_field(seed=0, env_size=(512, 256))
    w, h = 320, 180
    path = scenes.camera_spline(seed=0, frames=64)
    a = PathTracer(dict(presets.REALTIME))
    b = PathTracer(dict(presets.REALTIME))
    a.upload_scene(sc)
    b.upload_scene(sc)
    prev = None
    for f in range(3):
        mats, prev = scenes.camera_matrices(path[f][0], path[f][1], 60.0, 0.01, 1000.0, w, h, prev)
        a.set_camera_matrices(mats)
        b.set_camera_matrices(mats)
        a.render_device(w, h)
        b.profile_frame(w, h)
        for which, (name, gw, _) in BUFFERS.items():
            assert_bits(a.read_buffer(which, gw, w * h), b.read_buffer(which, gw, w * h), f"{name} frame {f}")
    assert a.last_stats.extension_rays == b.last_stats.extension_rays
