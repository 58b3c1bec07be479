"""Radiance-cache benchmark: the plain full-depth tracer against the same
estimator with paths ended at a short prefix by the online-trained cache.

For each scene: device time per frame at 1920x1080 (1 spp, depth 8) of the
plain tracer and of cache mode (inference + training included); and at
480x270 an equal-time study: both methods average frames (1 spp each) from a
fixed camera, and their relMSE = mean((x - ref)^2 / (ref^2 + 0.01)) against a
4096-spp full-depth reference accumulated in float64 on the host is tracked
against accumulated device time.  Reported: relMSE at equal time, and the time
the plain tracer needs to reach the cache's relMSE.

    python -m appearance_b200.rc_bench [--scenes cornell,field] [--budget-ms 400] [--study-size 480x270]
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import PathTracer, presets, scenes
from .radiance_cache import RadianceCache

PLAIN = dict(presets.PLAIN, max_bounces=8, sample_count=1)


def rel_mse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def scene_setup(name, w, h):
    if name == "cornell":
        sc = scenes.cornell_box()
        cam = scenes.cornell_camera()
        mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], w, h, None)
    else:
        sc = scenes.icosphere_field(seed=0)
        eye, tgt = scenes.camera_spline(seed=0, frames=64)[5]
        mats, _ = scenes.camera_matrices(eye, tgt, 60.0, 0.01, 1000.0, w, h, None)
    lo = sc.positions.min(0) - 0.05 * (sc.positions.max(0) - sc.positions.min(0))
    hi = sc.positions.max(0) + 0.05 * (sc.positions.max(0) - sc.positions.min(0))
    return sc, mats, lo, hi


def tracer(sc, mats, cfg):
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    pt.set_camera_matrices(mats)
    return pt


def frame_ms(sc, mats, w, h, cache_prefix=None, lo=None, hi=None, frames=8, warm=40):
    pt = tracer(sc, mats, PLAIN)
    rc = None
    if cache_prefix is not None:
        rc = RadianceCache(lo, hi, seed=1)
        pt.attach_radiance_cache(rc, prefix_bounces=cache_prefix, train_stride=16, train_batch=65536, lr=1e-3)
    for _ in range(warm):
        pt.render_device(w, h)
    ms = [pt.render_device(w, h) for _ in range(frames)]
    pt.close()
    if rc is not None:
        rc.close()
    return float(np.median(ms))


def quality_curve(pt, w, h, ref, budget_ms, max_frames=4000):
    acc = np.zeros((h, w, 3))
    t, k, curve = 0.0, 0, []
    while t < budget_ms and k < max_frames:
        acc += pt.render((w, h))
        t += pt.last_stats.gpu_ms
        k += 1
        if k in (1, 2, 4) or k % 8 == 0:
            curve.append((t, rel_mse(acc / k, ref)))
    curve.append((t, rel_mse(acc / k, ref)))
    return curve


def time_to(curve, target):
    for t, e in curve:
        if e <= target:
            return t
    return None


def study(name, budget_ms, warm_frames, w=480, h=270):
    sc, mats, lo, hi = scene_setup(name, w, h)
    pt = tracer(sc, mats, dict(PLAIN, sample_count=16))
    ref = np.zeros((h, w, 3))
    for _ in range(256):  # 4096 spp, float64 accumulation
        ref += pt.render((w, h))
    ref /= 256
    pt.close()
    out = {}
    pt = tracer(sc, mats, PLAIN)
    # the plain tracer runs on to 4x the budget, so that the time it needs to
    # reach the cache's relMSE is measured rather than cut off at the budget
    out["plain"] = quality_curve(pt, w, h, ref, 4.0 * budget_ms)
    pt.close()
    for prefix in (2, 1):
        rc = RadianceCache(lo, hi, seed=1)
        pt = tracer(sc, mats, PLAIN)
        pt.attach_radiance_cache(rc, prefix_bounces=prefix, train_stride=16, train_batch=65536, lr=1e-3)
        train_ms = 0.0
        for _ in range(warm_frames):  # online training before the timed accumulation
            pt.render((w, h))
            train_ms += pt.last_stats.gpu_ms
        out[f"cache_prefix{prefix}"] = quality_curve(pt, w, h, ref, budget_ms)
        out[f"cache_prefix{prefix}_warmup_ms"] = train_ms
        pt.close()
        rc.close()
    res = {"resolution": [w, h], "budget_ms": budget_ms, "warm_frames": warm_frames,
           "reference": "4096 spp full depth, float64 accumulation"}
    at_budget = [(t, e) for t, e in out["plain"] if t <= budget_ms] or out["plain"][:1]
    e_plain = at_budget[-1][1]
    res["plain"] = {"relmse_at_budget": e_plain, "frames_ms": at_budget[-1][0],
                    "relmse_at_4x_budget": out["plain"][-1][1], "frames_ms_4x": out["plain"][-1][0]}
    for prefix in (2, 1):
        cur = out[f"cache_prefix{prefix}"]
        e = cur[-1][1]
        t_plain = time_to(out["plain"], e)
        warm = out[f"cache_prefix{prefix}_warmup_ms"]
        # equal total time with the warm-up counted: the cache's relMSE after
        # (budget - warm-up) ms of accumulation against the plain relMSE at the budget
        e_cache_eq = next((ec for tc, ec in reversed(cur) if tc <= budget_ms - warm), None)
        res[f"cache_prefix{prefix}"] = {
            "relmse_at_budget": e, "warmup_training_ms": warm,
            "plain_time_to_same_relmse_ms": t_plain,
            "time_ratio_cache_over_plain": (cur[-1][0] / t_plain) if t_plain else None,
            "time_ratio_with_warmup": ((cur[-1][0] + warm) / t_plain) if t_plain else None,
            "relmse_ratio_at_equal_time": e / e_plain,
            "relmse_ratio_at_equal_time_with_warmup": (e_cache_eq / e_plain) if e_cache_eq is not None else None}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m appearance_b200.rc_bench")
    ap.add_argument("--scenes", default="cornell,field")
    ap.add_argument("--budget-ms", type=float, default=400.0)
    ap.add_argument("--warm-frames", type=int, default=200)
    ap.add_argument("--study-size", default="480x270", help="resolution of the equal-time study, WxH")
    ap.add_argument("--skip-frame-ms", action="store_true", help="only the equal-time study")
    a = ap.parse_args(argv)
    sw, sh = (int(v) for v in a.study_size.split("x"))
    result = {"metric": "radiance cache vs plain full-depth tracer", "config": {
        "mlp": "144 -> 4x64 ReLU -> 3 exp, FP16 weights/activations, FP32 accumulation (tcgen05)",
        "training": "2^16 suffix vertices per frame from 1/16 of the pixels, Adam lr 1e-3, relative L2",
        "plain": "1 spp, depth 8, RIS next-event estimation, no reuse or denoising"}}
    for name in a.scenes.split(","):
        w, h = 1920, 1080
        r = {}
        if not a.skip_frame_ms:
            sc, mats, lo, hi = scene_setup(name, w, h)
            r["frame_ms_1080p"] = {"plain": frame_ms(sc, mats, w, h),
                                   "cache_prefix2": frame_ms(sc, mats, w, h, 2, lo, hi),
                                   "cache_prefix1": frame_ms(sc, mats, w, h, 1, lo, hi)}
        r[f"equal_time_{sw}x{sh}"] = study(name, a.budget_ms, a.warm_frames, sw, sh)
        result[name] = r
        print(json.dumps({name: r}), flush=True)
    print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
