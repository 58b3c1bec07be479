"""World actions on the GPU (SpawnModel / TransformModel / DestroyModel /
Clear through ap_world_action, models from ap_model_register): the frames a
handle renders after them equal, bit for bit, the frames of the same world
uploaded in one piece (base scene plus the instances flattened with the rule
restated in tests/test_world_cpu.py), and the spectral mode sees the same
world (in its two-level form)."""
import numpy as np
import pytest

from appearance_b200 import PathTracer, gltf, presets, scenes
from appearance_b200.renderer import RendererError
from parity import assert_bits, assert_spectral_close
from test_world_cpu import compose

pytestmark = pytest.mark.gpu
W, H = 64, 48


def col_major(m4):
    return np.asarray(m4, np.float32).T.reshape(16)


def trs(t, angle_y, s):
    c, sn = np.cos(angle_y), np.sin(angle_y)
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = np.array([[c, 0, sn], [0, 1, 0], [-sn, 0, c]], np.float32) * np.float32(s)
    m[:3, 3] = t
    return col_major(m)


def setup(tmp_path):
    base = scenes.cornell_box()
    sph = scenes.icosphere_field(seed=9, num_spheres=3, num_emissive=1, subdiv=2, box=0.3, env_size=None)
    path = tmp_path / "spheres.glb"
    gltf.save_glb(str(path), sph)
    model = gltf.load(str(path))
    cam = scenes.cornell_camera()
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], W, H)
    return base, model, mats


def frames(pt, mats, n=2):
    out = []
    for _ in range(n):
        pt.set_camera_matrices(mats)
        out.append(pt.render((W, H)))
    return out


def reference_frames(base, model, transforms, mats, cfg, n=2, skip=0):
    """Frames skip .. skip + n - 1 of a fresh handle with the composed world
    (a world action keeps the handle's frame sequence going, so the frame
    index, and with it the sample streams, continues across it)."""
    pt = PathTracer(cfg)
    pt.upload_scene(compose(base, model, transforms))
    frames(pt, mats, skip)
    out = frames(pt, mats, n)
    pt.close()
    return out


def test_spawn_transform_destroy_equal_flattened_uploads(tmp_path):
    base, model, mats = setup(tmp_path)
    cfg = dict(presets.PLAIN, sample_count=2, max_bounces=3)
    u1, u2 = bytes(range(16)), bytes(range(16, 32))
    t1, t2 = trs([0.3, 0.05, 0.3], 0.4, 1.0), trs([0.6, 0.2, 0.5], -1.1, 0.7)
    pt = PathTracer(cfg)
    pt.upload_scene(base)
    pt.register_model("models/spheres.glb", model)
    pt.spawn_model(u1, "models/spheres.glb", t1)
    pt.spawn_model(u2, "models/spheres.glb", t2)
    for a, b in zip(frames(pt, mats), reference_frames(base, model, [t1, t2], mats, cfg)):
        assert_bits(a, b, "two instances")
    t1b = trs([0.25, 0.1, 0.55], 1.3, 1.2)
    pt.transform_model(u1, t1b)
    for a, b in zip(frames(pt, mats), reference_frames(base, model, [t1b, t2], mats, cfg, skip=2)):
        assert_bits(a, b, "after TransformModel")
    pt.destroy_model(u1)
    for a, b in zip(frames(pt, mats), reference_frames(base, model, [t2], mats, cfg, skip=4)):
        assert_bits(a, b, "after DestroyModel")
    pt.destroy_model(u1)  # unknown entity: ignored, as the reference's map remove
    with pytest.raises(RendererError):
        pt.transform_model(u1, t1)  # unknown entity
    with pytest.raises(RendererError):
        pt.spawn_model(bytes(16), "models/missing.glb", t1)
    pt.clear()
    with pytest.raises(RendererError):
        pt.render((W, H))  # Clear dropped the whole world
    pt.close()


def test_spectral_mode_sees_spawned_instances(tmp_path):
    base, model, mats = setup(tmp_path)
    t1 = trs([0.4, 0.1, 0.4], 0.7, 1.0)
    light = dict(sun_scale=0.0, scene_radius=10.0)
    a = PathTracer(presets.PLAIN)
    a.upload_scene(base)
    a.register_model("m", model)
    a.spawn_model(bytes(range(16)), "m", t1)
    a.set_camera_matrices(mats)
    a.spectral_setup(**light)
    img = a.render_spectral((W, H), spp=2, max_depth=4, seed=1)
    b = PathTracer(presets.PLAIN)
    b.upload_scene(compose(base, model, [t1]))
    b.set_camera_matrices(mats)
    b.spectral_setup(**light)
    ref = b.render_spectral((W, H), spp=2, max_depth=4, seed=1)
    # the world of instances renders through its two-level form (hits in
    # object space, normals through the instance transform), the upload
    # through the flattened world: the same estimator within the spectral
    # tolerance
    assert_spectral_close(img, ref, "spectral world")
    a.close()
    b.close()
