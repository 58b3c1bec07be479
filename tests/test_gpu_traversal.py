"""CUDA wide-BVH traversal vs the oracle: closest-hit triangle ids, t and
barycentrics bit-exact; any-hit agreement; degenerate rays.  The closest hit is
defined as the minimum of (t, triangle id) over the watertight test, so the
comparison has no tie tolerance: ties are resolved identically by rule."""
import numpy as np
import pytest

from appearance_b200 import PathTracer, presets, scenes
from oracle.oracle import OracleScene

pytestmark = pytest.mark.gpu


def rand_rays(n, lo, hi, seed):
    r = np.random.default_rng(seed)
    o = r.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = r.normal(size=(n, 3))
    return o, (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def check_closest(pt, osc, o, d, tmax=1000.0):
    g = pt.trace_rays(o, d, tmax)
    c, _ = osc.closest(o, d, tmax)
    c = c.view(np.uint32)
    assert np.array_equal(g[:, 3], c[:, 3]), f"{(g[:, 3] != c[:, 3]).sum()} triangle ids differ"
    hit = c[:, 3] != 0xFFFFFFFF
    assert np.array_equal(g[hit, :3], c[hit, :3])
    return hit.mean()


@pytest.fixture(scope="module")
def cornell():
    sc = scenes.cornell_box()
    pt = PathTracer(presets.FAITHFUL)
    pt.upload_scene(sc)
    return pt, OracleScene(sc), sc


@pytest.fixture(scope="module")
def field():
    sc = scenes.icosphere_field(seed=1, num_spheres=128, num_emissive=8, env_size=None)
    pt = PathTracer(presets.FAITHFUL)
    pt.upload_scene(sc)
    return pt, OracleScene(sc), sc


def test_cornell_random_rays(cornell):
    pt, osc, _ = cornell
    o, d = rand_rays(200000, 0.01, 0.99, 1)
    assert check_closest(pt, osc, o, d) > 0.5  # the room is open at z = 1


def test_field_random_rays(field):
    pt, osc, _ = field
    o, d = rand_rays(300000, -5.0, 45.0, 2)
    assert check_closest(pt, osc, o, d) > 0.1


def test_field_camera_rays(field):
    pt, osc, _ = field
    w, h = 320, 180
    mats, _ = scenes.camera_matrices((60, 30, 70), (20, 5, 20), 60.0, 0.01, 1000.0, w, h)
    iv, ip = (mats[i].reshape(4, 4).T.astype(np.float64) for i in range(2))
    ys, xs = np.mgrid[0:h, 0:w]
    t = np.stack([(xs + 0.5) / w * 2 - 1, -((ys + 0.5) / h * 2 - 1), np.ones_like(xs), np.ones_like(xs)], -1) @ ip.T
    d = t[..., :3] / np.linalg.norm(t[..., :3], axis=-1, keepdims=True) @ iv[:3, :3].T
    o = np.broadcast_to(iv[:3, 3], d.shape)
    check_closest(pt, osc, o.reshape(-1, 3).astype(np.float32), d.reshape(-1, 3).astype(np.float32))


def test_degenerate_rays(cornell):
    """Axis-aligned directions (zero components), origins on vertices, edges and
    the shared diagonal of a quad, and rays grazing a wall plane."""
    pt, osc, sc = cornell
    axes = np.concatenate([np.eye(3), -np.eye(3)]).astype(np.float32)
    pts = np.concatenate([sc.positions, (sc.positions[:-1] + sc.positions[1:]) / 2,
                          np.array([[0.5, 0.5, 0.5], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5], [0.25, 0.25, 0.0]])]).astype(np.float32)
    o = np.repeat(pts, len(axes), 0)
    d = np.tile(axes, (len(pts), 1))
    check_closest(pt, osc, o, d)
    # the Cornell floor quad's diagonal: rays straight down onto it
    s = np.linspace(0.01, 0.99, 997, dtype=np.float32)
    o2 = np.stack([s, np.full_like(s, 0.5), 1.0 - s], -1)
    check_closest(pt, osc, o2, np.tile(np.array([[0, -1, 0]], np.float32), (len(s), 1)))
    # grazing: in the plane of the back wall
    o3 = np.stack([s, np.full_like(s, 0.3), np.zeros_like(s)], -1)
    check_closest(pt, osc, o3, np.tile(np.array([[0, 1, 0]], np.float32), (len(s), 1)))


def test_any_hit_matches(field):
    pt, osc, _ = field
    o, d = rand_rays(200000, -5.0, 45.0, 3)
    tmax = np.random.default_rng(4).uniform(0.0, 30.0, len(o)).astype(np.float32)
    g = pt.trace_rays(o, d, tmax, any_hit=True)[:, 0]
    c = osc.any(o, d, tmax)
    assert np.array_equal(g.astype(np.uint8), c)


def test_full_size_scene_bit_exact():
    """The 1,310,722-triangle benchmark scene, 500k rays from the benchmark camera path."""
    sc = scenes.icosphere_field(seed=0, env_size=None)
    pt = PathTracer(presets.REALTIME)
    pt.upload_scene(sc)
    st = pt.bvh_stats()
    assert st["tris"] == sc.num_tris and st["max_stack"] <= 96
    osc = OracleScene(sc)
    eye, tgt = scenes.camera_spline(seed=0, frames=64)[5]
    rng = np.random.default_rng(5)
    n = 500000
    o = np.tile(np.asarray(eye, np.float32), (n, 1))
    d = (np.asarray(tgt) - np.asarray(eye))[None] + rng.normal(scale=15.0, size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    check_closest(pt, osc, o, d)
