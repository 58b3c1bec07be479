"""Host-side logic: scene generators, camera matrices, presets."""
import math

import numpy as np

from appearance_b200 import presets, scenes


def test_cornell_counts():
    sc = scenes.cornell_box()
    assert sc.num_tris == 36  # 5 walls x 2 + 2 boxes x 12 + 2 light triangles
    assert sc.meshes.shape == (2, 6)
    assert sc.meshes[1, 5] == 1 and sc.meshes[0, 5] == 0
    light = sc.materials[sc.meshes[1, 4]]
    assert np.allclose(light[5:8], [17, 12, 4])


def test_icosphere_field_counts():
    v, f = scenes.icosphere(3)
    assert f.shape[0] == 1280 and v.shape[0] == 642
    sc = scenes.icosphere_field(seed=0, env_size=(64, 32))
    assert sc.num_tris == 1024 * 1280 + 2
    assert int(sc.meshes[:, 5].sum()) == 64
    assert np.allclose(np.linalg.norm(sc.normals, axis=1), 1.0, atol=1e-5)
    again = scenes.icosphere_field(seed=0, env_size=(64, 32))
    assert np.array_equal(sc.positions, again.positions)


def test_sky_env_peak():
    env = scenes.sky_env(256, 128, sun_sigma=0.05)
    assert env.shape == (128, 256, 3)
    assert env.max() > 1e3 and env.min() >= 0


def test_camera_matrices_inverse_and_projection():
    mats, vp = scenes.camera_matrices((1, 2, 3), (0, 0, 0), 40.0, 0.01, 100.0, 64, 48)
    iv, ip, vpm = (mats[i].reshape(4, 4).T.astype(np.float64) for i in range(3))
    view = np.linalg.inv(iv)
    proj = np.linalg.inv(ip)
    assert np.allclose(proj @ view, vpm, atol=1e-5)
    # the eye maps to the origin of view space, the target onto the -z axis
    e = view @ np.array([1, 2, 3, 1.0])
    assert np.allclose(e[:3], 0, atol=1e-5)
    t = view @ np.array([0, 0, 0, 1.0])
    assert abs(t[0]) < 1e-5 and abs(t[1]) < 1e-5 and t[2] < 0
    assert math.isclose(proj[1, 1], 1 / math.tan(math.radians(20)), rel_tol=1e-6)


def test_presets_consistent():
    assert presets.PLAIN["sample_count"] == 16 and presets.PLAIN["max_bounces"] == 5
    assert presets.REALTIME["di_area_samples"] == 32 and presets.REALTIME["max_bounces"] == 8
    for p in presets.PRESETS.values():
        assert set(p) == set(presets.FAITHFUL)
