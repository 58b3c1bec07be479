"""Render-serving loop on the GPU: a job's result equals the single-renderer
frame with the same inputs, and is the same alone and in a mix of concurrent
jobs (with and without CUDA graphs); admission respects the memory budget."""
import numpy as np
import pytest

from appearance_b200 import PathTracer, RendererError, scenes
from appearance_b200.serve import SERVE_CONFIG, RenderServer

pytestmark = pytest.mark.gpu


def small_scene(seed):
    return scenes.icosphere_field(seed=seed, num_spheres=24, num_emissive=3, subdiv=2, box=8.0, env_size=(32, 16))


def mats_for(seed, view, w, h):
    eye, tgt = scenes.camera_spline(seed=seed, frames=16, box=8.0)[view]
    return scenes.camera_matrices(eye, tgt, 60.0, 0.01, 500.0, w, h, None)[0]


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


CFG = dict(SERVE_CONFIG, max_bounces=3)
MIX = [(0, 96, 64, 2, 3, 5), (1, 40, 30, 8, 3, 6), (1, 128, 72, 1, 2, 7), (0, 17, 9, 4, 3, 8),
       (1, 64, 64, 16, 1, 9), (0, 33, 21, 3, 3, 10), (1, 200, 120, 1, 3, 11)]


@pytest.mark.parametrize("graphs", [False, True])
def test_job_equals_frame_and_is_same_alone_and_in_mix(graphs):
    scs = [small_scene(0), small_scene(1)]
    w, h, spp, depth = 64, 48, 4, 3
    m = mats_for(0, 3, w, h)
    pt = PathTracer(dict(CFG, sample_count=spp, max_bounces=depth))
    pt.upload_scene(scs[0])
    pt.set_camera_matrices(m)
    ref = pt.render((w, h))  # frame 0 of a fresh renderer: PCG frame index 0
    pt.close()
    srv = RenderServer(CFG, hbm_budget=8e9, max_inflight=4, use_graphs=graphs)
    ids = [srv.add_scene(s) for s in scs]
    alone, info = srv.wait(srv.submit(ids[0], w, h, spp, depth, 0, m))
    assert same_bits(alone, ref)
    assert info["graph_mode"] == (1 if graphs else 0)
    # the same job among others of mixed scene, size, spp and depth, all in flight together
    tickets = []
    for k, (sc, ww, hh, s, d, seed) in enumerate(MIX):
        if k == 3:
            tickets.append(("target", srv.submit(ids[0], w, h, spp, depth, 0, m)))
        tickets.append((k, srv.submit(ids[sc], ww, hh, s, d, seed, mats_for(sc, k, ww, hh))))
    outs = {key: srv.wait(t)[0] for key, t in tickets}
    assert same_bits(outs["target"], alone)
    for k, (sc, ww, hh, s, d, seed) in enumerate(MIX):
        assert outs[k].shape == (hh, ww, 3) and np.isfinite(outs[k]).all()
    # each mixed job alone gives the same image as in the mix
    for k in (0, 4, 6):
        sc, ww, hh, s, d, seed = MIX[k]
        img, _ = srv.wait(srv.submit(ids[sc], ww, hh, s, d, seed, mats_for(sc, k, ww, hh)))
        assert same_bits(img, outs[k])
    st = srv.stats()
    assert st["completed"] >= 12 and st["in_flight"] == 0 and st["queued"] == 0
    srv.close()


def test_graph_updated_in_place_for_same_shape():
    srv = RenderServer(CFG, hbm_budget=8e9, max_inflight=1, use_graphs=True)
    sid = srv.add_scene(small_scene(0))
    modes = [srv.wait(srv.submit(sid, 48, 32, 2, 3, k, mats_for(0, k, 48, 32)))[1]["graph_mode"] for k in range(3)]
    assert modes == [1, 2, 2]
    assert srv.stats()["graphs_updated"] == 2
    # another scene and resolution with the same samples and depth: the same
    # launch sequence, updated in place, and the image of a graph-less run
    sid1 = srv.add_scene(small_scene(1))
    img, info = srv.wait(srv.submit(sid1, 64, 40, 2, 3, 7, mats_for(1, 7, 64, 40)))
    assert info["graph_mode"] == 2
    plain = RenderServer(CFG, hbm_budget=8e9, max_inflight=1, use_graphs=False)
    pid = [plain.add_scene(small_scene(k)) for k in range(2)][1]
    ref, _ = plain.wait(plain.submit(pid, 64, 40, 2, 3, 7, mats_for(1, 7, 64, 40)))
    assert same_bits(img, ref)
    plain.close()
    srv.close()


def test_admission_respects_the_budget():
    probe = RenderServer(CFG, hbm_budget=8e9, max_inflight=1)
    probe.add_scene(small_scene(0))
    scene_bytes = probe.stats()["scene_bytes"]
    probe.close()
    job = RenderServer.job_bytes(256, 256)
    budget = scene_bytes + int(1.5 * job)  # room for one such job at a time
    srv = RenderServer(CFG, hbm_budget=budget, max_inflight=4, use_graphs=False)
    sid = srv.add_scene(small_scene(0))
    ts = [srv.submit(sid, 256, 256, 1, 2, k, mats_for(0, k, 256, 256)) for k in range(4)]
    for t in ts:
        srv.wait(t)
    st = srv.stats()
    assert st["peak_device_bytes"] <= budget
    assert st["peak_device_bytes"] >= scene_bytes + job
    # a job that cannot fit even alone fails cleanly
    with pytest.raises(RendererError):
        srv.wait(srv.submit(sid, 1024, 1024, 1, 1, 0, mats_for(0, 0, 1024, 1024)))
    srv.close()


def test_faults_fail_their_own_job_only():
    """Host-side fault injection on the serving loop (no GPU fault): a job
    cancelled while queued, a job whose deadline passes in the queue, a job
    naming an unknown scene, and a job too large for the device-memory budget
    each fail with their own status, while the jobs around them complete with
    the images they give alone."""
    from appearance_b200 import _native
    sc = small_scene(0)
    srv = RenderServer(CFG, hbm_budget=2e9, max_inflight=1, use_graphs=False)
    sid = srv.add_scene(sc)
    w, h = 96, 64
    m = mats_for(0, 2, w, h)
    ref, _ = srv.wait(srv.submit(sid, w, h, 2, 3, 4, m))  # the image of the probe job alone
    # one slot: a long job occupies it while the others queue behind
    long_t = srv.submit(sid, 512, 512, 64, 3, 1, mats_for(0, 5, 512, 512))
    dropped = srv.submit(sid, w, h, 2, 3, 4, m)
    late = srv.submit(sid, w, h, 2, 3, 4, m, deadline_ms=1)
    probe = srv.submit(sid, w, h, 2, 3, 4, m)
    srv.cancel(dropped)
    with pytest.raises(RendererError) as e:  # a corrupted scene id is refused at submission
        srv.submit(sid + 7, w, h, 2, 3, 4, m)
    assert e.value.code == _native.AP_E_INVALID
    srv.wait(long_t)
    with pytest.raises(RendererError) as e:
        srv.wait(dropped)
    assert e.value.code == _native.AP_E_CANCELLED
    with pytest.raises(RendererError) as e:
        srv.wait(late)
    assert e.value.code == _native.AP_E_TIMEOUT
    img, _ = srv.wait(probe)
    assert same_bits(img, ref)
    # a job larger than the whole budget fails alone; the next job still runs
    big_w = big_h = 4096
    assert RenderServer.job_bytes(big_w, big_h) > 2e9
    big = srv.submit(sid, big_w, big_h, 1, 3, 4, mats_for(0, 1, big_w, big_h))
    after = srv.submit(sid, w, h, 2, 3, 4, m)
    with pytest.raises(RendererError) as e:
        srv.wait(big)
    assert e.value.code == _native.AP_E_OOM
    img, _ = srv.wait(after)
    assert same_bits(img, ref)
    # cancelling a finished or unknown ticket
    with pytest.raises(RendererError):
        srv.cancel(123456789)
    srv.close()


@pytest.mark.parametrize("graphs", [False, True])
def test_batched_jobs_equal_their_alone_results(graphs):
    """Jobs of the same spp and depth queued together run as one launch
    sequence (shared traversal launches over all their ray queues); each
    result is bit for bit the one the job has on a server that runs every job
    on its own.  The batch mixes scenes, sizes (one of a single pixel),
    cameras and seeds."""
    scs = [small_scene(0), small_scene(1)]
    jobs = [(0, 64, 48, 11), (1, 40, 30, 12), (0, 1, 1, 13), (1, 96, 20, 14), (0, 33, 65, 15), (1, 64, 48, 16)]
    spp, depth = 2, 3
    alone = RenderServer(CFG, hbm_budget=8e9, max_inflight=1, use_graphs=False)
    alone.set_batching(1)
    ids = [alone.add_scene(s) for s in scs]
    refs = []
    for sc, w, h, seed in jobs:
        img, info = alone.wait(alone.submit(ids[sc], w, h, spp, depth, seed, mats_for(sc, seed % 16, w, h)))
        assert info["batch"] == 1
        refs.append(img)
    alone.close()
    srv = RenderServer(CFG, hbm_budget=8e9, max_inflight=1, use_graphs=graphs)
    ids = [srv.add_scene(s) for s in scs]
    # a long job first holds the only slot, so the others queue up and are admitted together
    blocker = srv.submit(ids[0], 256, 256, 16, depth, 1, mats_for(0, 1, 256, 256))
    tickets = [srv.submit(ids[sc], w, h, spp, depth, seed, mats_for(sc, seed % 16, w, h)) for sc, w, h, seed in jobs]
    srv.wait(blocker)
    batches = []
    for t, ref in zip(tickets, refs):
        img, info = srv.wait(t)
        assert same_bits(img, ref)
        batches.append(info["batch"])
    assert max(batches) > 1, batches
    st = srv.stats()
    assert st["in_flight"] == 0 and st["queued"] == 0
    srv.close()
