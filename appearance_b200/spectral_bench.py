"""Spectral-mode benchmark on the procedural city (10.0M world triangles on a
2 km grid, emissive windows, sky environment): by default the instanced city
(4096 instances of 64 building models, placed by world actions and traced
through the two-level BVH), or (`--flat`) 4096 distinct buildings in one
world-space BVH;
hero-wavelength paths of depth 16 at 4096 x 4096 and 64 spp, rendered in row
bands, timed on the device.  Reports Msamples/s, Mrays/s and rays per sample;
with --quality also the relMSE of the 64-spp image on the centre 1024 x 1024
crop against a high-spp reference of that crop accumulated in float64; with
--cache the same for the radiance-cache mode (paths ended at their first
bounce's hit in the online-trained cache).

The CPU figure beside it (the oracle's restatement of the same integrator on
all host threads over a band of rows at 1 spp) is taken by bench.py.

    python -m appearance_b200.spectral_bench [--lots 64] [--size 4096] [--spp 64] [--flat [--cache]]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import PathTracer, presets, scenes

SUN = dict(sun_dir=(0.0, -1.0, 0.2), sun_rgb=(1.0, 1.0, 0.95), sun_scale=100.0)


def setup(lots: int, size: int, instanced: bool):
    """The city (a Scene, or (base, models, instances)) and camera matrices."""
    t0 = time.perf_counter()
    extent = 2000.0 * lots / 64
    sc = scenes.city_instanced(lots=lots, extent=extent) if instanced else scenes.city(lots=lots, extent=extent)
    gen_s = time.perf_counter() - t0
    cam = scenes.city_camera(extent)
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], 0.5, 5000.0, size, size, None)
    return sc, mats, gen_s


def load_world(pt, sc, instanced: bool):
    """Uploads the city: the flat Scene, or the base scene plus the models
    spawned by SpawnModel world actions (ap_model_register first)."""
    if not instanced:
        pt.upload_scene(sc)
        return
    base, models, instances = sc
    pt.upload_scene(base)
    for k, m in enumerate(models):
        pt.register_model(f"city/building{k}.glb", m)
    for i, (k, m16) in enumerate(instances):
        pt.spawn_model(i.to_bytes(16, "little"), f"city/building{k}.glb", m16)


def rel_mse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def render_bands(pt, size, spp, depth, seed, band, to_host=False):
    """The image in row bands; returns (image or None, device ms, rays)."""
    img = np.empty((size, size, 3), np.float32) if to_host else None
    ms, rays = 0.0, 0
    for r0 in range(0, size, band):
        r1 = min(size, r0 + band)
        out = pt.render_spectral((size, size), spp=spp, max_depth=depth, seed=seed, start_row=r0, end_row=r1,
                                 to_host=to_host)
        if to_host:
            img[r0:r1] = out
        ms += pt.last_stats.gpu_ms
        rays += int(pt.last_stats.extension_rays)
    return img, ms, rays


def measure(lots=64, size=4096, spp=64, depth=16, band=4096, repeats=1, quality=False, ref_spp=4096,
            cache=False, cache_prefix=1, keep_scene=None, instanced=True) -> dict:
    """The measurements above as a dict; `keep_scene` (a dict), when given,
    receives the scene, camera matrices and light parameters for a caller's
    own comparison run.  The radiance-cache mode takes the flat city."""
    if instanced and cache:
        raise ValueError("the radiance-cache mode renders flat scenes")
    sc, mats, gen_s = setup(lots, size, instanced)
    pt = PathTracer(presets.PLAIN)
    t0 = time.perf_counter()
    load_world(pt, sc, instanced)
    pt.set_camera_matrices(mats)
    radius = 0.75 * 2000.0 * lots / 64
    pt.spectral_setup(scene_radius=radius, **SUN)  # builds the world's BVHs
    upload_s = time.perf_counter() - t0
    render_bands(pt, size, min(spp, 4), depth, 1, band)  # warm-up at a few samples
    runs = []
    for rep in range(repeats):
        _, ms, rays = render_bands(pt, size, spp, depth, 100 + rep, band)
        runs.append((ms, rays, pt.last_stats.kernel_launches))
    ms = float(np.median([r[0] for r in runs]))
    rays = runs[0][1]
    samples = size * size * spp
    if instanced:
        base, models, instances = sc
        world_tris = base.num_tris + sum(models[k].num_tris for k, _ in instances)
        desc = (f"instanced city: {len(instances)} instances of {len(models)} building models "
                f"({sum(m.num_tris for m in models)} model triangles, {world_tris} world triangles), two-level BVH")
    else:
        world_tris = sc.num_tris
        desc = f"city of {lots}x{lots} distinct buildings, {world_tris} triangles, one world-space BVH"
    res = {"metric": "spectral Msamples/s", "value": samples / (ms * 1e3), "unit": "Msamples/s",
           "frame_ms": ms, "rays": rays, "rays_per_sample": rays / samples, "mrays_per_s": rays / (ms * 1e3),
           "workload": f"{desc}, {size}x{size} x {spp} spp, depth {depth}, 4 wavelengths, "
                       f"wavefront in bands of {band} rows",
           "kernel_launches_per_band": runs[0][2], "scene_gen_s": gen_s, "upload_and_bvh_s": upload_s}
    if not instanced:
        res["bvh"] = pt.bvh_stats()
    # traversal work per ray from the instrumented kernels on one sample per pixel
    v = pt.profile_spectral((size, size), spp=1, max_depth=depth, seed=100)
    trav = {}
    total_bytes = 0.0
    for kind in ("closest", "any"):
        r = max(v[kind]["rays"], 1)
        n, t = v[kind]["nodes"] / r, v[kind]["tris"] / r
        # ray 32 + hit 16, 80 B per node, 36 B per triangle; the two-level form
        # reads 64 B of instance record per instance entered, counted as nodes
        # here (the instrumented kernels count TLAS and BLAS nodes alike)
        b = 48.0 + 80.0 * n + 36.0 * t
        trav[kind] = {"nodes_per_ray": n, "tris_per_ray": t, "bytes_per_ray": b,
                      "ray_share": v[kind]["rays"] / max(v["closest"]["rays"] + v["any"]["rays"], 1)}
        total_bytes += b * trav[kind]["ray_share"]
    trav["algorithmic_gbs_over_image_time"] = total_bytes * rays / (ms * 1e-3) / 1e9
    res["traversal"] = trav
    c0, c1 = size // 2 - size // 8, size // 2 + size // 8  # centre crop rows/cols (1024 of 4096)
    if quality:
        img, _, _ = render_bands(pt, size, spp, depth, 100, band, to_host=True)
        ref = np.zeros((c1 - c0, c1 - c0, 3), np.float64)
        chunk, done, seed = 256, 0, 10_000
        while done < ref_spp:
            k = min(chunk, ref_spp - done)
            out = pt.render_spectral((size, size), spp=k, max_depth=depth, seed=seed, start_row=c0, end_row=c1)
            ref += out[:, c0:c1].astype(np.float64) * k
            done += k
            seed += 1
        ref /= ref_spp
        res["quality"] = {"crop": [c0, c1], "ref_spp": ref_spp,
                          "relmse_crop": rel_mse(img[c0:c1, c0:c1].astype(np.float64), ref),
                          "mean_crop": ref.mean(axis=(0, 1)).tolist()}
    if cache:
        # radiance-cache mode: paths end at their prefix-th hit in the online-trained
        # cache; 1/16 of the pixels per pass trace full paths and train it
        from .radiance_cache import RadianceCache
        ext = sc.positions.max(0) - sc.positions.min(0)  # the flat city
        rc = RadianceCache(sc.positions.min(0) - 0.02 * ext, sc.positions.max(0) + 0.02 * ext, seed=1)
        pt.attach_radiance_cache(rc, prefix_bounces=cache_prefix, train_stride=16, train_batch=65536, lr=1e-3)
        warm_ms = render_bands(pt, size, 8, depth, 7, band)[1]  # 8 passes of online training first
        _, ms_c, rays_c = render_bands(pt, size, spp, depth, 100, band)
        res["cache"] = {"value": samples / (ms_c * 1e3), "unit": "Msamples/s", "frame_ms": ms_c,
                        "rays_per_sample": rays_c / samples, "prefix": cache_prefix, "warmup_ms": warm_ms,
                        "training": "65536 suffix vertices per sample pass from 1/16 of the pixels, Adam lr 1e-3"}
        if quality:
            img_c, _, _ = render_bands(pt, size, spp, depth, 100, band, to_host=True)
            res["cache"]["relmse_crop"] = rel_mse(img_c[c0:c1, c0:c1].astype(np.float64), ref)
        pt.attach_radiance_cache(None)
        rc.close()
    pt.close()
    if keep_scene is not None:
        keep_scene.update(scene=sc, mats=mats, light=dict(scene_radius=radius, **SUN), size=size, depth=depth,
                          instanced=instanced)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m appearance_b200.spectral_bench")
    ap.add_argument("--lots", type=int, default=64)
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--depth", type=int, default=16)
    ap.add_argument("--band", type=int, default=4096, help="rows per launch sequence")
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--quality", action="store_true", help="relMSE of the crop against a high-spp reference")
    ap.add_argument("--ref-spp", type=int, default=4096)
    ap.add_argument("--cache", action="store_true", help="also run the radiance-cache mode")
    ap.add_argument("--cache-prefix", type=int, default=1)
    ap.add_argument("--flat", action="store_true", help="distinct buildings in one world-space BVH (the cache needs it)")
    a = ap.parse_args(argv)
    res = measure(a.lots, a.size, a.spp, a.depth, a.band, a.repeats, a.quality, a.ref_spp, a.cache, a.cache_prefix,
                  instanced=not a.flat)
    print(json.dumps(res), flush=True)
    return res


if __name__ == "__main__":
    main()
