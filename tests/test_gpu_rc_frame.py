"""Radiance-cache mode of the frame: what the trained network gains.

Against a high-sample full-depth reference of the Cornell box, paths cut after
their first bounce lose the light of their longer suffixes (about 15 % of the
image in this estimator, which carries little light past the second bounce);
the same 1-bounce prefix ended with the online-trained cache recovers most of
it.  Both are averaged over the same number of frames and samples."""
import numpy as np
import pytest

from appearance_b200 import PathTracer, presets, scenes
from appearance_b200.radiance_cache import RadianceCache

pytestmark = pytest.mark.gpu
W, H = 96, 64


def rel_mse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def average(pt, frames):
    acc = np.zeros((H, W, 3))
    for _ in range(frames):
        acc += pt.render((W, H))
    return acc / frames


def test_trained_cache_beats_truncation():
    sc = scenes.cornell_box()  # closed box: multiple bounces carry much of the light
    cam = scenes.cornell_camera()
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], W, H, None)
    plain = dict(presets.PLAIN, max_bounces=8, sample_count=16)

    def tracer(cfg):
        pt = PathTracer(cfg)
        pt.upload_scene(sc)
        pt.set_camera_matrices(mats)
        return pt

    pt = tracer(plain)
    ref = average(pt, 128)  # 2048 spp, full depth
    pt.close()

    pt = tracer(dict(plain, max_bounces=1))
    cut = average(pt, 32)
    pt.close()

    rc = RadianceCache([-0.05, -0.05, -0.05], [1.05, 1.05, 1.05], seed=1)
    pt = tracer(plain)
    pt.attach_radiance_cache(rc, prefix_bounces=1, train_stride=4, train_batch=16384, lr=5e-3)
    average(pt, 150)  # online training
    cached = average(pt, 32)
    pt.close()
    rc.close()

    e_cut, e_cached = rel_mse(cut, ref), rel_mse(cached, ref)
    print(f"relMSE truncated {e_cut:.5f} cached {e_cached:.5f}; mean ref {ref.mean():.4f} cut {cut.mean():.4f} "
          f"cached {cached.mean():.4f}")
    assert np.isfinite(cached).all()
    assert cut.mean() < 0.9 * ref.mean()  # truncation loses light here
    assert abs(cached.mean() - ref.mean()) < 0.5 * abs(cut.mean() - ref.mean())
    assert e_cached < 0.6 * e_cut


def test_ray_queries_between_cached_frames_leave_the_cache_state_intact():
    """A batch ray query that grows the handle's query scratch must not touch
    the radiance cache's frame state: the frames after it equal the frames of
    the same sequence without the query."""
    sc = scenes.cornell_box()
    cam = scenes.cornell_camera()
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], W, H, None)
    cfg = dict(presets.PLAIN, max_bounces=4, sample_count=2)
    rng = np.random.default_rng(3)
    o = rng.uniform(0.1, 0.9, (4096, 3)).astype(np.float32)
    d = rng.normal(size=(4096, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)

    def run(with_query):
        rc = RadianceCache([-0.05, -0.05, -0.05], [1.05, 1.05, 1.05], seed=2)
        pt = PathTracer(cfg)
        pt.upload_scene(sc)
        pt.set_camera_matrices(mats)
        # training on: the batch and the gradient sums are assembled in a fixed
        # order, so the whole sequence is reproducible bit for bit
        pt.attach_radiance_cache(rc, prefix_bounces=1, train_stride=4, train_batch=4096, lr=5e-3)
        frames = [pt.render((W, H))]
        if with_query:
            pt.trace_rays(o[:16], d[:16], 100.0)
            pt.trace_rays(o, d, 100.0)  # larger than before: the query scratch grows
        frames += [pt.render((W, H)) for _ in range(3)]
        pt.close()
        rc.close()
        return frames

    a, b = run(False), run(True)
    for i, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"frame {i} differs"


def test_online_training_is_reproducible():
    """Two runs of the same cached frame sequence from the same initial
    network give the same frames and the same trained weights, bit for bit:
    the training batch takes its records in slot order (a prefix-sum
    compaction) and each step's gradient is the CTAs' rows added in a fixed
    order.  The spectral mode's training, over several sample passes, too."""
    sc = scenes.cornell_box()
    cam = scenes.cornell_camera()
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], W, H, None)

    def frames_run():
        rc = RadianceCache([-0.05, -0.05, -0.05], [1.05, 1.05, 1.05], seed=4)
        pt = PathTracer(dict(presets.PLAIN, max_bounces=8, sample_count=2))
        pt.upload_scene(sc)
        pt.set_camera_matrices(mats)
        pt.attach_radiance_cache(rc, prefix_bounces=1, train_stride=4, train_batch=4096, lr=5e-3)
        out = [pt.render((W, H)) for _ in range(12)]
        params = rc.params()
        pt.close()
        rc.close()
        return out, params

    def spectral_run():
        rc = RadianceCache([-0.05, -0.05, -0.05], [1.05, 1.05, 1.05], seed=5)
        pt = PathTracer(presets.PLAIN)
        pt.upload_scene(sc)
        pt.set_camera_matrices(mats)
        pt.spectral_setup(sun_scale=0.0, scene_radius=10.0)
        pt.attach_radiance_cache(rc, prefix_bounces=1, train_stride=4, train_batch=8192, lr=5e-3)
        img = pt.render_spectral((W, H), spp=8, max_depth=8, seed=1)
        params = rc.params()
        pt.close()
        rc.close()
        return img, params

    (fa, pa), (fb, pb) = frames_run(), frames_run()
    for i, (x, y) in enumerate(zip(fa, fb)):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"frame {i} differs"
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32)), "trained weights differ"
    (ia, qa), (ib, qb) = spectral_run(), spectral_run()
    assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32)), "spectral image differs"
    assert np.array_equal(qa.view(np.uint32), qb.view(np.uint32)), "spectral-trained weights differ"
