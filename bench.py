"""Benchmark of the real-time path-tracing frame on B200.

Workload (one step = one frame): the seeded 1,310,722-triangle icosphere field
(1024 icospheres x 1280 triangles + ground quad, 64 emissive spheres, 2048x1024
procedural sky), 1920x1080, 1 spp, depth 8, ReSTIR DI (32 area candidates,
temporal M cap 20x, 5-neighbour spatial), ReSTIR GI (temporal and one unbiased
5-neighbour spatial pass), firefly filter, SVGF (5 a-trous passes), TAA,
camera moving along a 64-frame seeded spline.  Metric: Msamples/s (= pixels x spp / frame time).

  value   device time of the frames (CUDA events on the renderer's stream),
          scene and frame state resident in HBM.
  e2e     the same camera frames again through the public C ABI call
          ap_render_hdr with a host output buffer (page-locked, allocated
          once): per frame the camera goes host->device and the 1920x1080 RGB
          f32 framebuffer comes back device->host.

Run with torchrun for N>1: every rank renders its own independent replica of
the job (the frame does not shard), so scaling is weak and value sums ranks.
`--impl reference` times the CPU restatement of the reference frame (the
reference itself is Rust/WGSL on wgpu and cannot run here) on all host cores,
on the same 1920x1080 frames of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_FULL, H_FULL = 1920, 1080
CPU_W, CPU_H = W_FULL, H_FULL  # CPU samples: the same frames of the same workload
CPU_TIMED_FRAMES = 2
PRESET = "realtime_gi_spatial"
METRIC = "Msamples/s (1080p ReSTIR+SVGF+TAA frame, 1.31M-tri scene)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-baseline", type=int, default=1, help="time the CPU oracle sample (rank 0, N=1)")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_workload():
    from appearance_b200 import scenes
    scene = scenes.icosphere_field(seed=0)
    path = scenes.camera_spline(seed=0, frames=64)
    return scene, path


def frame_mats(path, f, prev, w, h):
    from appearance_b200 import scenes
    eye, tgt = path[f % len(path)]
    return scenes.camera_matrices(eye, tgt, 60.0, 0.01, 1000.0, w, h, prev)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(scene, path, cfg) -> dict:
    """The CPU oracle (restatement of the reference frame) on a bounded sample:
    the same scene, preset, camera path and resolution, 1 warm + 2 timed
    frames, all host threads."""
    from oracle.oracle import OracleFrame, OracleScene
    w, h = CPU_W, CPU_H
    osc = OracleScene(scene)
    fr = OracleFrame(osc, w, h, cfg, threads=os.cpu_count())
    prev = None
    mats, prev = frame_mats(path, 0, prev, w, h)
    fr.render(mats)  # builds nothing new; first frame warms the history
    t0 = time.perf_counter()
    frames = CPU_TIMED_FRAMES
    for f in range(1, 1 + frames):
        mats, prev = frame_mats(path, f, prev, w, h)
        fr.render(mats)
    dt = time.perf_counter() - t0
    return {"value": w * h * frames / dt / 1e6, "unit": "Msamples/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle (CPU restatement of the reference frame), same scene/preset, {w}x{h}, "
                      f"{frames} timed frames after 1 warm frame, {os.cpu_count()} threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from appearance_b200 import presets
    scene, path = build_workload()
    from oracle.oracle import OracleFrame, OracleScene
    w, h = CPU_W, CPU_H
    osc = OracleScene(scene)
    fr = OracleFrame(osc, w, h, presets.PRESETS[PRESET], threads=os.cpu_count())
    prev = None
    for f in range(args.warmup):
        mats, prev = frame_mats(path, f, prev, w, h)
        fr.render(mats)
    t0 = time.perf_counter()
    for f in range(args.warmup, args.warmup + args.steps):
        mats, prev = frame_mats(path, f, prev, w, h)
        fr.render(mats)
    dt = time.perf_counter() - t0
    v = w * h * args.steps / dt / 1e6
    sample = (f"CPU restatement of the reference frame (the reference is Rust+WGSL on wgpu/Vulkan ray queries and "
              f"cannot run here), same scene/preset at {w}x{h} per step, {os.cpu_count()} threads")
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "Msamples/s", "n_gpus": world,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic (seeded icosphere field)",
                      "config": {"workload": "icosphere-field-1.31M-tris 1920x1080 realtime frame", "width": w,
                                 "height": h, "spp": 1, "preset": PRESET},
                      "cpu_baseline": {"value": v, "unit": "Msamples/s", "cores": os.cpu_count(), "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": v, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from appearance_b200 import PathTracer, presets, replicas
    scene, path = build_workload()
    cfg = dict(presets.PRESETS[PRESET])
    pt = PathTracer(cfg, device=local)
    pt.upload_scene(scene)
    bvh = pt.bvh_stats()
    P = W_FULL * H_FULL

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # warm-up
    prev = None
    f = replicas.replica_first_frame(rank)  # each replica renders its own stretch of the camera path
    for _ in range(args.warmup):
        mats, prev = frame_mats(path, f, prev, W_FULL, H_FULL)
        pt.set_camera_matrices(mats)
        pt.render_device(W_FULL, H_FULL)
        f += 1
    # timed device-resident frames; the output (24.9 MB) exceeds nothing in L2 reuse terms:
    # every frame rewrites ~1 GB of per-pixel state, far beyond the 126 MB L2.
    clocks = ClockSampler(local)
    f0, prev0 = f, prev  # the e2e pass below renders the same camera frames
    barrier()
    clocks.start()
    gpu_ms = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        mats, prev = frame_mats(path, f, prev, W_FULL, H_FULL)
        pt.set_camera_matrices(mats)
        gpu_ms.append(pt.render_device(W_FULL, H_FULL))
        f += 1
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    dev_s = sum(gpu_ms) / 1e3
    # end-to-end through ap_render_hdr with a host output buffer
    barrier()
    # the caller's output buffer: page-locked host memory, allocated once
    out = torch.empty((H_FULL, W_FULL, 3), dtype=torch.float32, pin_memory=True).numpy()
    e2e_t = []
    f, prev = f0, prev0
    for _ in range(args.steps):
        mats, prev = frame_mats(path, f, prev, W_FULL, H_FULL)
        t1 = time.perf_counter()
        pt.set_camera_matrices(mats)
        pt.render((W_FULL, H_FULL), out=out)
        e2e_t.append(time.perf_counter() - t1)
        f += 1
    barrier()
    e2e_s = sum(e2e_t)
    e2e_frames = len(e2e_t)
    # the slowest rank's times; the job's samples over them
    dev_s, e2e_s, wall = replicas.max_over_ranks([dev_s, e2e_s, wall], world, device="cuda")
    if rank == 0:
        value = replicas.job_throughput(P * args.steps, world, dev_s) / 1e6
        e2e = replicas.job_throughput(P * e2e_frames, world, e2e_s) / 1e6
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded icosphere field, procedural sky, seeded camera spline)",
            "config": {"workload": "icosphere-field-1.31M-tris 1920x1080 realtime frame", "width": W_FULL,
                       "height": H_FULL, "spp": 1, "depth": cfg["max_bounces"], "preset": PRESET,
                       "gi_spatial_passes": cfg["gi_spatial_passes"],
                       "parallelism": f"replicas x{world}", "l2": "inputs+state ~1 GB/frame > 126 MB L2",
                       "bvh": bvh},
            "frame_ms": {"median": statistics.median(gpu_ms), "min": min(gpu_ms), "max": max(gpu_ms)},
            "wall_ms_per_step": wall * 1e3 / args.steps,
            "e2e": {"value": e2e, "unit": "Msamples/s", "h2d_bytes_per_step": 256,
                    "d2h_bytes_per_step": int(out.nbytes)},
            "clocks": clk,
            "gpu_launches": None,
        }
        details = measure_details(pt, scene, path, cfg)
        line.update(details)
        line["gpu_launches"] = int(details["gpu_launches_per_step"]) * args.steps
        if world == 1 and args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(scene, path, cfg)
        if world == 1:  # the other configurations are single-GPU cases, measured on one GPU only
            cpu = bool(args.cpu_baseline)
            line["configs"] = {"cornell_512_16spp_depth5": cornell_config(cpu),
                               "city_spectral_4096_64spp_depth16": city_spectral_config(cpu),
                               "serving_mixed_jobs": serving_config(),
                               "radiance_cache_cornell_480x270": radiance_cache_config()}
        print(json.dumps(line), flush=True)
    pt.close()
    if world > 1:
        dist.destroy_process_group()


def cornell_config(cpu: bool) -> dict:
    """The plain CPU-comparable configuration: the seeded Cornell box at
    512x512, 16 spp, depth 5, RIS next-event estimation without reuse or
    denoising.  Device time of 5 frames after 2 warm-up frames; the CPU oracle
    of the same estimator on a 256x256 render (same scene, spp and depth,
    all host threads) beside it."""
    from appearance_b200 import PathTracer, presets, scenes
    cfg = dict(presets.PLAIN)
    w = h = 512
    sc = scenes.cornell_box()
    cam = scenes.cornell_camera()
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], w, h, None)
    pt = PathTracer(cfg)
    pt.upload_scene(sc)
    pt.set_camera_matrices(mats)
    for _ in range(2):
        pt.render_device(w, h)
    ms = [pt.render_device(w, h) for _ in range(5)]
    pt.close()
    samples = w * h * cfg["sample_count"]
    out = {"workload": "cornell box 512x512, 16 spp, depth 5, plain estimator", "triangles": int(sc.num_tris),
           "frame_ms": statistics.median(ms), "value": samples / (statistics.median(ms) * 1e-3) / 1e6,
           "unit": "Msamples/s"}
    if cpu:
        from oracle.oracle import OracleFrame, OracleScene
        cw = ch = 256
        cm, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], cw, ch, None)
        fr = OracleFrame(OracleScene(sc), cw, ch, cfg, threads=os.cpu_count())
        t0 = time.perf_counter()
        fr.render(cm)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": cw * ch * cfg["sample_count"] / dt / 1e6, "unit": "Msamples/s",
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": f"oracle, same scene and estimator at {cw}x{ch}, 16 spp, depth 5, 1 frame"}
    return out


def radiance_cache_config() -> dict:
    """The radiance cache against the plain full-depth tracer (1 spp, depth 8)
    on the Cornell box at 480x270: both accumulate frames from a fixed camera
    for 400 ms of device time and are scored by relMSE against a 4096-spp
    full-depth reference; the cache first trains online for 100 frames, and
    the ratios with that warm-up included are reported beside those without."""
    from appearance_b200 import rc_bench
    r = rc_bench.study("cornell", budget_ms=400.0, warm_frames=100)
    out = {"workload": "cornell box 480x270, 1 spp frames, depth 8, cache prefix 1 and 2 bounces",
           "budget_ms": r["budget_ms"], "plain": r["plain"]}
    for k in ("cache_prefix1", "cache_prefix2"):
        out[k] = r[k]
    return out


def serving_config() -> dict:
    """The render-serving loop (ap_server_*): 96 seeded jobs of mixed
    resolution (256^2 .. 1920x1080), spp (1 .. 64) and scene (resident
    icosphere fields of 0.1M, 1M, 2M and 4M triangles), Poisson arrivals at
    200 jobs/s (far above what one GPU completes: latency there is queueing),
    then the same list at 60 % of the completion rate seen there (a load the
    server sustains: latency is the loop's), and the 200 jobs/s list on a
    one-job-at-a-time server.  Latency is submit -> result in host memory."""
    from appearance_b200 import serve
    r = serve.run_benchmark(n_jobs=96, rates=(200.0,), sustained_fraction=0.6, serial=True)
    over, sus = r["server"][0], r["server"][1]
    keep = ("rate", "jobs", "p50_ms", "p99_ms", "mean_ms", "msamples_per_s", "wall_s", "mean_queued_ms", "mean_gpu_ms")
    return {"workload": "96 mixed jobs (4 resident scenes 0.1M-4M triangles, 256^2-1080p, 1-64 spp, depth 8)",
            "unit": "Msamples/s", "value": over["msamples_per_s"],
            "overload": {k: over[k] for k in keep}, "sustained": {k: sus[k] for k in keep},
            "serial": {k: r["serial"][k] for k in keep}, "throughput_vs_serial": r["throughput_vs_serial"],
            "server_stats": r["stats"]}


def city_spectral_config(cpu: bool) -> dict:
    """The large spectral configuration: the seeded instanced city (4096
    instances of 64 box-building models on a 2 km grid, 10.0M world triangles,
    emissive windows, sky environment) placed by world actions and traced
    through the two-level BVH, hero-wavelength paths (4 wavelengths in 360-830
    nm, RGB-to-spectrum albedos and emitters), depth 16, 4096x4096 at 64 spp:
    one warm-up image at 4 spp, then one timed image (device time).  Beside
    it the flat city (4096 distinct buildings, one world-space BVH) plain and
    in radiance-cache mode (`cache`: paths ended at their first bounce's hit in
    the online-trained cache, after 8 training passes).  The CPU oracle of the
    same integrator renders 64 full-width rows of the instanced city at 1 spp."""
    from appearance_b200 import scenes, spectral_bench
    kept = {}
    res = spectral_bench.measure(instanced=True, keep_scene=kept if cpu else None)
    flat = spectral_bench.measure(instanced=False, cache=True, quality=True, ref_spp=1024)
    res["flat_city"] = {k: flat[k] for k in ("value", "unit", "frame_ms", "rays_per_sample", "workload", "traversal")}
    res["cache"] = dict(flat["cache"])
    # relMSE of the 1024x1024 centre crop against a 1024-spp plain render of it;
    # the plain time to the cache's relMSE assumes relMSE ~ 1/spp (variance)
    e_plain, e_cache = flat["quality"]["relmse_crop"], flat["cache"]["relmse_crop"]
    t_plain_eq = flat["frame_ms"] * e_plain / e_cache
    res["cache"].update(relmse_plain=e_plain, relmse_cache=e_cache, reference_spp=1024,
                        plain_time_to_cache_relmse_ms=t_plain_eq,
                        time_ratio=(flat["cache"]["frame_ms"] + flat["cache"]["warmup_ms"]) / t_plain_eq)
    if cpu:
        from oracle.oracle import OracleScene, OracleSpectral, OracleTwoLevel
        rows, size, threads = 64, kept["size"], os.cpu_count()
        base, models, instances = kept["scene"]
        eye = np.eye(4, dtype=np.float32).reshape(16)
        tl = OracleTwoLevel([base] + list(models), [(0, eye)] + [(k + 1, m) for k, m in instances])
        osp = OracleSpectral(OracleScene(scenes.flatten_world(base, models, instances)), two_level=tl,
                             **kept["light"])
        r0 = size // 2 - rows // 2
        t0 = time.perf_counter()
        osp.render(kept["mats"], size, size, spp=1, max_depth=kept["depth"], seed=100, row0=r0, row1=r0 + rows,
                   threads=threads)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": rows * size / dt / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
                               "sample": f"oracle, rows {r0}..{r0 + rows} of the {size}^2 image (full width) at 1 spp, "
                                         f"{dt:.1f} s"}
    return res


def measure_details(pt, scene, path, cfg) -> dict:
    """Per-kernel device times and the roofline of the dominant kernel (filled in
    by appearance_b200.profile)."""
    from appearance_b200 import profile
    return profile.frame_roofline(pt, scene, path, cfg, W_FULL, H_FULL, peaks())


if __name__ == "__main__":
    main()
