"""Two-level traversal on the GPU (ap_trace_rays over a world of spawned
instances: a TLAS over per-model BLAS, rays mapped to object space, as the
reference's TLAS of BLAS instances) against the oracle's own two-level
queries: closest hits (t, u, v, triangle id) and any-hit answers bit for bit,
up to the instanced city of the large spectral configuration (4096 instances
of 64 building models, 10.0M world triangles)."""
import numpy as np
import pytest

from appearance_b200 import PathTracer, presets, scenes
from oracle.oracle import OracleTwoLevel

pytestmark = pytest.mark.gpu
IDENTITY = np.eye(4, dtype=np.float32).reshape(16)


def world(pt, base, models, instances):
    pt.upload_scene(base)
    for k, m in enumerate(models):
        pt.register_model(f"models/{k}.glb", m)
    for i, (k, m16) in enumerate(instances):
        pt.spawn_model(i.to_bytes(16, "little"), f"models/{k}.glb", m16)
    return OracleTwoLevel([base] + list(models), [(0, IDENTITY)] + [(k + 1, m16) for k, m16 in instances])


def compare(pt, orc, o, d, tmax, what):
    got = pt.trace_rays(o, d, tmax)
    ref = orc.closest(o, d, tmax)
    bad = (got != ref).any(1)
    assert not bad.any(), f"{what}: {bad.sum()} of {len(o)} closest hits differ, e.g. {got[bad][:2]} vs {ref[bad][:2]}"
    hit = got[:, 3] != 0xFFFFFFFF
    ga = pt.trace_rays(o, d, tmax, any_hit=True)[:, 0].astype(np.uint8)
    ra = orc.any(o, d, tmax)
    assert np.array_equal(ga, ra), f"{what}: {(ga != ra).sum()} any-hit answers differ"
    return hit.mean()


def random_transform(rng, box):
    a, b = rng.uniform(0, 2 * np.pi, 2)
    ca, sa, cb, sb = np.cos(a), np.sin(a), np.cos(b), np.sin(b)
    r = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]]) @ np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    m = np.eye(4)
    m[:3, :3] = r * rng.uniform(0.3, 1.5, 3)[None, :]  # non-uniform scale
    m[:3, 3] = rng.uniform(-box, box, 3)
    return m.astype(np.float32).T.reshape(16).copy()


def test_instances_of_models_match_the_oracle():
    rng = np.random.default_rng(11)
    base = scenes.cornell_box()
    models = [scenes.icosphere_field(seed=s, num_spheres=4, num_emissive=1, subdiv=2, box=0.6, env_size=None)
              for s in (1, 2, 3)]
    instances = [(int(rng.integers(0, 3)), random_transform(rng, 2.0)) for _ in range(40)]
    pt = PathTracer(presets.PLAIN)
    orc = world(pt, base, models, instances)
    n = 40000
    o = rng.uniform(-3.0, 3.0, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    assert compare(pt, orc, o, d, 1e30, "random rays") > 0.2
    # rays toward instance centres, short segments for the any-hit form
    targets = np.stack([np.asarray(m, np.float32).reshape(4, 4)[3, :3] for _, m in instances])
    t = targets[rng.integers(0, len(targets), n)] + rng.normal(scale=0.05, size=(n, 3)).astype(np.float32)
    d2 = t - o
    d2 = (d2 / np.linalg.norm(d2, axis=1, keepdims=True)).astype(np.float32)
    assert compare(pt, orc, o, d2, 1e30, "rays at instances") > 0.5
    compare(pt, orc, o, d2, 1.5, "short rays")
    # moving an instance moves its hits
    pt.transform_model((0).to_bytes(16, "little"), random_transform(rng, 2.0))
    pt.close()


def test_instanced_city_matches_the_oracle():
    base, models, instances = scenes.city_instanced(env_size=None)
    pt = PathTracer(presets.PLAIN)
    orc = world(pt, base, models, instances)
    cam = scenes.city_camera()
    w, h = 256, 192
    mats = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], 0.5, 5000.0, w, h, None)[0]
    inv_view, inv_proj = np.asarray(mats, np.float64).reshape(4, 4, 4)[0].T, np.asarray(mats).reshape(4, 4, 4)[1].T
    ys, xs = np.mgrid[0:h, 0:w]
    ndc = np.stack([(xs + 0.5) / w * 2 - 1, -((ys + 0.5) / h * 2 - 1), np.ones_like(xs, float), np.ones_like(xs, float)], -1)
    tgt = ndc.reshape(-1, 4) @ inv_proj.T
    dirs = np.concatenate([tgt[:, :3] / np.linalg.norm(tgt[:, :3], axis=1, keepdims=True),
                           np.zeros((w * h, 1))], 1) @ inv_view.T
    d = (dirs[:, :3] / np.linalg.norm(dirs[:, :3], axis=1, keepdims=True)).astype(np.float32)
    o = np.repeat(np.asarray(cam["eye"], np.float32)[None], w * h, 0)
    assert compare(pt, orc, o, d, 1e30, "city camera rays") > 0.5
    rng = np.random.default_rng(5)
    n = 30000
    o2 = np.stack([rng.uniform(-1000, 1000, n), rng.uniform(1, 150, n), rng.uniform(-1000, 1000, n)], 1).astype(np.float32)
    d2 = rng.normal(size=(n, 3))
    d2[:, 1] = -np.abs(d2[:, 1])
    d2 = (d2 / np.linalg.norm(d2, axis=1, keepdims=True)).astype(np.float32)
    compare(pt, orc, o2, d2, 1e30, "city random rays")
    compare(pt, orc, o2, d2, 40.0, "city short rays")
    pt.close()


def _spectral_pair(base, models, instances, mats, w, h, light, spp, depth, seed):
    from oracle.oracle import OracleScene, OracleSpectral
    from test_world_cpu import compose_many
    pt = PathTracer(presets.PLAIN)
    tl = world(pt, base, models, instances)
    pt.set_camera_matrices(mats)
    pt.spectral_setup(**light)
    img = pt.render_spectral((w, h), spp=spp, max_depth=depth, seed=seed)
    pt.close()
    flat = compose_many(base, models, instances)
    ref = OracleSpectral(OracleScene(flat), two_level=tl, **light).render(mats, w, h, spp=spp, max_depth=depth,
                                                                         seed=seed)
    return img, ref


def test_spectral_over_instances_matches_the_oracle():
    """The spectral mode over a world of instances (two-level traversal, normals
    through the instance transforms) against the oracle tracing the same
    two-level form and shading from the flattened world."""
    from parity import assert_spectral_close
    rng = np.random.default_rng(4)
    base = scenes.cornell_box()
    models = [scenes.icosphere_field(seed=s, num_spheres=3, num_emissive=1, subdiv=2, box=0.3, env_size=None)
              for s in (6, 7)]
    models[1].materials[:, 3] = 1.0  # gold
    instances = [(int(rng.integers(0, 2)), random_transform(rng, 0.35)) for _ in range(12)]
    for k, m in instances:
        m[12:15] += 0.5  # inside the box
    cam = scenes.cornell_camera()
    w, h = 64, 48
    mats = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], 0.01, 100.0, w, h, None)[0]
    img, ref = _spectral_pair(base, models, instances, mats, w, h, dict(sun_scale=0.0, scene_radius=10.0), 2, 6, 3)
    assert img.mean() > 0.0
    assert_spectral_close(img, ref, "instances spp=2 depth=6")


def test_spectral_instanced_city_matches_the_oracle():
    from parity import assert_spectral_close
    base, models, instances = scenes.city_instanced(env_size=(512, 256))
    cam = scenes.city_camera()
    w = h = 64
    mats = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], 0.5, 5000.0, w, h, None)[0]
    light = dict(sun_dir=(0.0, -1.0, 0.2), sun_rgb=(1.0, 1.0, 0.95), sun_scale=100.0, scene_radius=1500.0)
    img, ref = _spectral_pair(base, models, instances, mats, w, h, light, 2, 16, 3)
    assert img.mean() > 0.0
    assert_spectral_close(img, ref, "instanced city 64x64 spp=2 depth=16")
