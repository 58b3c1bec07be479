"""Render-serving loop: the host side of the ap_server_* entry points
(include/appearance_cuda.h), and the serving benchmark.

`RenderServer` keeps scenes resident on one GPU and runs submitted jobs of
mixed resolution, samples per pixel and scene concurrently, admitting them in
arrival order as device memory and execution slots free up (the native
dispatcher in csrc/serve.cu does the work).  It takes the role of the
reference's frame farm (crates/appearance-render-loop/src/host.rs:250-505,
node.rs:27-147), where a node renders one request at a time.

Benchmark (`python -m appearance_b200.serve`): Poisson arrivals, resolutions
{256^2, 512^2, 1024^2, 1920x1080} with probabilities (0.4, 0.3, 0.2, 0.1), spp
uniform in {1, 4, 16, 64}, depth 8, scenes drawn uniformly from resident
icosphere fields of the requested triangle counts.  It reports p50/p99 job
latency (submit -> result in host memory) and aggregate Msamples/s, for the
concurrent server and for serial execution (one job at a time) of the same
job list.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import threading
import time

import numpy as np

from . import _native, presets, scenes
from .renderer import RendererError, config_struct, scene_desc

RESOLUTIONS = [(256, 256), (512, 512), (1024, 1024), (1920, 1080)]
RES_PROBS = [0.4, 0.3, 0.2, 0.1]
SPPS = [1, 4, 16, 64]
TRIS_PER_SPHERE = 1280

# the serving frame: the plain estimator (RIS next-event estimation + BSDF
# continuation), no temporal reuse or denoising across independent jobs
SERVE_CONFIG = dict(presets.PLAIN, max_bounces=8, sample_count=1)


class RenderServer:
    def __init__(self, config: dict | None = None, device: int = 0, hbm_budget: float = 150e9,
                 max_inflight: int = 4, use_graphs: bool = True):
        self._lib = _native.load()
        self._cfg = config_struct(config if config is not None else SERVE_CONFIG)
        err = ctypes.c_int(0)
        self._s = self._lib.ap_server_create(ctypes.byref(self._cfg), device, int(hbm_budget), max_inflight,
                                             1 if use_graphs else 0, ctypes.byref(err))
        if not self._s:
            raise RendererError(err.value, "ap_server_create failed")
        self._outs = {}

    def _check(self, rc):
        if rc != _native.AP_OK:
            raise RendererError(rc, self._lib.ap_server_last_error(self._s).decode())

    def close(self):
        if getattr(self, "_s", None):
            self._lib.ap_server_destroy(self._s)
            self._s = None

    def __del__(self):
        self.close()

    def add_scene(self, scene) -> int:
        d, keep = scene_desc(scene)
        sid = ctypes.c_uint32(0)
        self._check(self._lib.ap_server_add_scene(self._s, ctypes.byref(d), ctypes.byref(sid)))
        del keep
        return sid.value

    @staticmethod
    def job_bytes(width: int, height: int) -> int:
        return int(_native.load().ap_server_job_bytes(width, height))

    def submit(self, scene: int, width: int, height: int, spp: int, max_depth: int, seed: int, mats,
               out: np.ndarray | None = None, deadline_ms: int = 0) -> int:
        """Queues a job and returns its ticket.  `out` (float32, height x width x 3)
        receives the result; page-locked memory avoids one host copy.  A job
        still queued `deadline_ms` after submission (0: no deadline) is not
        started and its wait raises with AP_E_TIMEOUT."""
        j = _native.Job()
        j.scene, j.width, j.height, j.spp, j.max_depth, j.seed = scene, width, height, spp, max_depth, seed
        j.deadline_ms = deadline_ms
        m = np.ascontiguousarray(mats, np.float32).reshape(64)
        for i in range(64):
            j.mats[i] = float(m[i])
        if out is None:
            out = np.empty((height, width, 3), np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size >= width * height * 3
        t = ctypes.c_uint64(0)
        self._check(self._lib.ap_server_submit(self._s, ctypes.byref(j), out.ctypes.data_as(ctypes.c_void_p),
                                               out.nbytes, ctypes.byref(t)))
        self._outs[t.value] = out
        return t.value

    def done(self, ticket: int) -> bool:
        d = ctypes.c_int(0)
        self._check(self._lib.ap_server_query(self._s, ticket, ctypes.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int):
        """Blocks until the job is done; returns (image, timing dict)."""
        r = _native.JobResult()
        out = self._outs.pop(ticket)
        self._check(self._lib.ap_server_wait(self._s, ticket, ctypes.byref(r)))
        return out, dict(queued_ms=r.queued_ms, total_ms=r.total_ms, gpu_ms=r.gpu_ms, device_bytes=r.device_bytes,
                         graph_mode=r.graph_mode, slot=r.slot, batch=r.batch)

    def set_batching(self, max_batch: int):
        """ap_server_set_batching: the largest batch of same-shape jobs admitted
        together (1 runs every job on its own)."""
        self._check(self._lib.ap_server_set_batching(self._s, max_batch))

    def cancel(self, ticket: int):
        """ap_server_cancel: a queued job is dropped; one on the GPU finishes its
        launches; either way its wait raises with AP_E_CANCELLED."""
        self._check(self._lib.ap_server_cancel(self._s, ticket))

    def stats(self) -> dict:
        a = np.zeros(8, np.uint64)
        self._check(self._lib.ap_server_stats(self._s, a.ctypes.data_as(ctypes.c_void_p)))
        keys = ["completed", "in_flight", "queued", "device_bytes", "peak_device_bytes", "scene_bytes",
                "graphs_instantiated", "graphs_updated"]
        return {k: int(v) for k, v in zip(keys, a)}


def serving_jobs(n_jobs: int, rate: float, n_scenes: int, seed: int = 0, depth: int = 8):
    """The job list of the serving workload: seeded Poisson arrival times
    (seconds from the start), resolution, spp, scene and PCG frame index."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n_jobs)
    t = np.cumsum(gaps) - gaps[0]
    res = rng.choice(len(RESOLUTIONS), n_jobs, p=RES_PROBS)
    spp = rng.choice(SPPS, n_jobs)
    sc = rng.integers(0, n_scenes, n_jobs)
    view = rng.integers(0, 64, n_jobs)
    return [dict(arrival=float(t[i]), width=RESOLUTIONS[res[i]][0], height=RESOLUTIONS[res[i]][1], spp=int(spp[i]),
                 depth=depth, scene=int(sc[i]), view=int(view[i]), seed=i) for i in range(n_jobs)]


def job_mats(job, paths):
    eye, tgt = paths[job["scene"]][job["view"]]
    mats, _ = scenes.camera_matrices(eye, tgt, 60.0, 0.01, 1000.0, job["width"], job["height"], None)
    return mats


def run_jobs(server: RenderServer, jobs, paths, realtime: bool = True, pinned=None):
    """Submits the jobs at their arrival times (or all at once) and collects
    each job's timing.  Returns (per-job results, wall seconds)."""
    tickets = [None] * len(jobs)
    results = [None] * len(jobs)

    def waiter():
        for i in range(len(jobs)):
            while tickets[i] is None:
                time.sleep(0.0002)
            _, r = server.wait(tickets[i])
            results[i] = r

    th = threading.Thread(target=waiter)
    th.start()
    t0 = time.perf_counter()
    for i, j in enumerate(jobs):
        if realtime:
            delay = j["arrival"] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
        out = None if pinned is None else pinned(j)
        tickets[i] = server.submit(j["scene"], j["width"], j["height"], j["spp"], j["depth"], j["seed"],
                                   job_mats(j, paths), out)
    th.join()
    wall = time.perf_counter() - t0
    return results, wall


def summarise(jobs, results, wall):
    lat = sorted(r["total_ms"] for r in results)
    batches = [r.get("batch", 1) for r in results]
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    q = lambda p: lat[min(len(lat) - 1, int(round(p * (len(lat) - 1))))]
    return dict(jobs=len(jobs), p50_ms=q(0.5), p99_ms=q(0.99), mean_ms=statistics.mean(lat),
                msamples_per_s=samples / wall / 1e6, wall_s=wall,
                mean_queued_ms=statistics.mean(r["queued_ms"] for r in results),
                mean_batch=statistics.mean(batches), batched_jobs=sum(1 for b in batches if b > 1),
                mean_gpu_ms=statistics.mean(r["gpu_ms"] for r in results))


def run_benchmark(n_jobs: int = 200, rates=(200.0,), scene_tris=(100000, 1000000, 2000000, 4000000),
                  budget_gb: float = 150.0, slots: int = 4, graphs: bool = True, serial: bool = True,
                  sustained_fraction: float = 0.0, seed: int = 0) -> dict:
    """The serving benchmark: the same seeded job list submitted at each
    Poisson rate in `rates` (jobs/s) to a concurrent server, and, with
    `sustained_fraction` > 0, once more at that fraction of the job rate the
    server completed at the first rate (a load it sustains, so that latency is
    the loop's and not queueing); with `serial`, the list at the first rate to
    a one-job-at-a-time server as well."""
    import torch  # page-locked result buffers
    t = time.perf_counter()
    field = [scenes.icosphere_field(seed=k, num_spheres=max(1, round(n / TRIS_PER_SPHERE)),
                                    num_emissive=max(1, round(n / TRIS_PER_SPHERE) // 16)) for k, n in enumerate(scene_tris)]
    paths = [scenes.camera_spline(seed=k, frames=64) for k in range(len(scene_tris))]
    gen_s = time.perf_counter() - t

    def pinned(j):
        return torch.empty((j["height"], j["width"], 3), dtype=torch.float32, pin_memory=True).numpy()

    out = dict(workload=dict(jobs=n_jobs, rates=list(rates), scene_tris=[int(f.num_tris) for f in field],
                             budget_gb=budget_gb, slots=slots, graphs=bool(graphs), depth=8, spp=SPPS,
                             resolutions=RESOLUTIONS, res_probs=RES_PROBS, scene_gen_s=gen_s))
    warm = [dict(j, arrival=0.0) for j in serving_jobs(8, 1.0, len(scene_tris), seed=seed + 99)]

    def server(max_inflight, use_graphs, max_batch=8):
        srv = RenderServer(SERVE_CONFIG, hbm_budget=budget_gb * 1e9, max_inflight=max_inflight, use_graphs=use_graphs)
        srv.set_batching(max_batch)
        for f in field:
            srv.add_scene(f)
        run_jobs(srv, warm, paths, realtime=False, pinned=pinned)  # one job per class, untimed
        return srv

    t = time.perf_counter()
    srv = server(slots, bool(graphs))
    out["workload"]["scene_upload_s"] = time.perf_counter() - t
    runs = []
    for rate in rates:
        jobs = serving_jobs(n_jobs, rate, len(scene_tris), seed=seed)
        res, wall = run_jobs(srv, jobs, paths, realtime=True, pinned=pinned)
        runs.append(dict(rate=rate, **summarise(jobs, res, wall)))
    if sustained_fraction > 0:
        first = runs[0]
        rate = sustained_fraction * first["jobs"] / first["wall_s"]
        jobs = serving_jobs(n_jobs, rate, len(scene_tris), seed=seed)
        res, wall = run_jobs(srv, jobs, paths, realtime=True, pinned=pinned)
        runs.append(dict(rate=rate, sustained=True, **summarise(jobs, res, wall)))
    out["server"] = runs
    out["stats"] = srv.stats()
    srv.close()
    if serial:
        ser = server(1, False, max_batch=1)
        jobs = serving_jobs(n_jobs, rates[0], len(scene_tris), seed=seed)
        res, wall = run_jobs(ser, jobs, paths, realtime=True, pinned=pinned)
        out["serial"] = dict(rate=rates[0], **summarise(jobs, res, wall))
        ser.close()
        out["throughput_vs_serial"] = runs[0]["msamples_per_s"] / out["serial"]["msamples_per_s"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m appearance_b200.serve")
    ap.add_argument("--jobs", type=int, default=200)
    ap.add_argument("--rate", type=float, default=200.0, help="Poisson arrival rate (jobs/s)")
    ap.add_argument("--sustained", type=float, default=0.6,
                    help="also run at this fraction of the completion rate seen at --rate (0: off)")
    ap.add_argument("--scene-tris", default="100000,1000000,2000000,4000000")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--graphs", type=int, default=1)
    ap.add_argument("--serial", type=int, default=1, help="also run the jobs one at a time")
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    out = run_benchmark(a.jobs, (a.rate,), [int(x) for x in a.scene_tris.split(",")], a.budget_gb, a.slots,
                        bool(a.graphs), bool(a.serial), a.sustained, a.seed)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
