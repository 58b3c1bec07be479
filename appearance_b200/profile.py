"""Per-kernel device times and the HBM roofline of the frame's kernels.

Algorithmic bytes (what `achieved` is computed from):
  traversal (extend, trace_closest, trace_any): per ray 48 B (ray 32 + hit 16)
      + 80 B per wide-BVH node visited + 36 B per triangle tested (3 x f32x3),
      with node and triangle counts taken from an instrumented pass of the same
      frame setup (same BVH, same kind of rays);
  a-trous: 40 B per pixel per iteration (radiance 12 + variance 4 + normal 4 +
      depth 4 in, radiance 12 + variance 4 out);
  SVGF temporal: 88 B per pixel; TAA: 52 B per pixel.
"""
from __future__ import annotations

TRAVERSAL = ("extend", "trace_closest", "trace_any")

# DRAM bytes (read + write) per ray of the queue traversal kernels, from one
# ncu capture of every traversal launch of a 960x540 benchmark frame divided by
# that frame's ray count (`python -m appearance_b200.profile --visits`); used
# as the measured `traffic` of a full frame, scaled by its ray count.
NCU_DRAM_BYTES_PER_RAY = {"trace_any": 136.4, "trace_closest": 152.7}
PER_PIXEL_BYTES = {"atrous": 40.0, "svgf_temporal": 88.0, "taa": 52.0}


def traversal_bytes(rays: int, nodes: int, tris: int) -> float:
    return 48.0 * rays + 80.0 * nodes + 36.0 * tris


def kernel_rooflines(timing: dict, counts: dict, pixels: int, peak_gbs: float) -> dict:
    out = {}
    for k, t in timing.items():
        ms = t["ms"]
        if ms <= 0:
            continue
        if k in TRAVERSAL and counts.get(k, {}).get("rays", 0) > 0:
            c = counts[k]
            # scale the instrumented frame's work to this frame's ray count
            per_ray = traversal_bytes(c["rays"], c["nodes"], c["tris"]) / c["rays"]
            rays = c["rays"]
            byts = per_ray * rays
            out[k] = dict(ms=ms, bytes=byts, achieved_gbs=byts / (ms * 1e-3) / 1e9, bytes_per_ray=per_ray,
                          rays=rays, nodes_per_ray=c["nodes"] / c["rays"], tris_per_ray=c["tris"] / c["rays"])
        elif k in PER_PIXEL_BYTES:
            iters = t["launches"]
            byts = PER_PIXEL_BYTES[k] * pixels * iters
            out[k] = dict(ms=ms, bytes=byts, achieved_gbs=byts / (ms * 1e-3) / 1e9)
        if k in out:
            out[k]["frac"] = out[k]["achieved_gbs"] / peak_gbs
    return out


def frame_roofline(pt, scene, path, cfg, width: int, height: int, peak) -> dict:
    """Runs one instrumented frame (visit counts) and one timed frame with
    per-kernel events, both continuing the renderer's frame sequence."""
    peak_gbs, peak_kind = peak
    counts = pt.profile_frame(width, height, count_visits=True)
    timing = pt.profile_frame(width, height)
    launches = pt.last_stats.kernel_launches
    total = sum(v["ms"] for v in timing.values())
    roofs = kernel_rooflines(timing, counts, width * height, peak_gbs)
    dominant = max(timing, key=lambda k: timing[k]["ms"])
    # the reported roofline is the most time-consuming kernel that has an
    # algorithmic byte count (the traversal kernels or a denoiser stencil)
    best = max(roofs, key=lambda k: roofs[k]["ms"]) if roofs else None
    res = {
        "kernels_ms": {k: round(v["ms"], 4) for k, v in sorted(timing.items(), key=lambda kv: -kv[1]["ms"])
                       if v["ms"] > 0},
        "kernels_share": {k: round(v["ms"] / total, 4) for k, v in timing.items() if v["ms"] > 0},
        "dominant_kernel": dominant,
        "gpu_launches_per_step": launches,
    }
    if best:
        r = roofs[best]
        traffic = None
        if best in NCU_DRAM_BYTES_PER_RAY and "rays" in r:
            traffic = NCU_DRAM_BYTES_PER_RAY[best] * r["rays"]
        res["roofline"] = {"kernel": best, "bound": "hbm", "achieved": round(r["achieved_gbs"], 2),
                           "peak": peak_gbs, "unit": "GB/s", "frac": round(r["frac"], 4), "traffic": traffic,
                           "traffic_note": "DRAM bytes per frame of this kernel kind: ncu bytes/ray of a 960x540 "
                                           "frame x this frame's rays" if traffic else None,
                           "peak_source": peak_kind,
                           "algorithmic_bytes_per_frame": r["bytes"]}
        if "bytes_per_ray" in r:
            res["roofline"].update(rays=r["rays"], bytes_per_ray=round(r["bytes_per_ray"], 1),
                                   nodes_per_ray=round(r["nodes_per_ray"], 2), tris_per_ray=round(r["tris_per_ray"], 2))
    res["kernel_rooflines"] = {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                               for k, v in roofs.items()}
    return res


def _frames_cli(argv=None):
    """Renders frames of the benchmark workload (seeded 1.31M-triangle
    icosphere field, seeded camera spline) on cuda:0 and prints each frame's
    device time; the fixed command that profiler captures run."""
    import argparse

    from . import PathTracer, presets, scenes
    ap = argparse.ArgumentParser(prog="python -m appearance_b200.profile")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--preset", default="realtime", choices=sorted(presets.PRESETS))
    ap.add_argument("--kernels", action="store_true", help="also print per-kernel times of one more frame")
    ap.add_argument("--visits", action="store_true",
                    help="also print rays, BVH nodes and triangles per traversal kind of one more (instrumented) frame")
    a = ap.parse_args(argv)
    scene = scenes.icosphere_field(seed=0)
    path = scenes.camera_spline(seed=0, frames=64)
    pt = PathTracer(presets.PRESETS[a.preset])
    pt.upload_scene(scene)
    prev = None
    f = 0
    for f in range(a.frames):
        eye, tgt = path[f % len(path)]
        mats, prev = scenes.camera_matrices(eye, tgt, 60.0, 0.01, 1000.0, a.width, a.height, prev)
        pt.set_camera_matrices(mats)
        ms = pt.render_device(a.width, a.height)
        print(f"frame {f} {a.width}x{a.height} {ms:.3f} ms launches {pt.last_stats.kernel_launches}", flush=True)
    if a.kernels:
        eye, tgt = path[(f + 1) % len(path)]
        mats, prev = scenes.camera_matrices(eye, tgt, 60.0, 0.01, 1000.0, a.width, a.height, prev)
        pt.set_camera_matrices(mats)
        prof = pt.profile_frame(a.width, a.height)
        tot = sum(v["ms"] for v in prof.values())
        for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"]):
            if v["ms"] > 0:
                print(f"  {k:16s} {v['ms']:9.3f} ms {v['launches']:4d} launches {100 * v['ms'] / tot:5.1f}%")
        print(f"total {tot:.3f} ms")
        f += 1
    if a.visits:
        eye, tgt = path[(f + 1) % len(path)]
        mats, prev = scenes.camera_matrices(eye, tgt, 60.0, 0.01, 1000.0, a.width, a.height, prev)
        pt.set_camera_matrices(mats)
        prof = pt.profile_frame(a.width, a.height, count_visits=True)
        for k in TRAVERSAL:
            v = prof.get(k, {})
            if v.get("rays"):
                print(f"  visits {k:14s} rays {v['rays']} nodes {v['nodes']} tris {v['tris']} "
                      f"bytes/ray {traversal_bytes(v['rays'], v['nodes'], v['tris']) / v['rays']:.1f}")
    pt.close()


if __name__ == "__main__":
    _frames_cli()
