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


def test_city_counts_and_layout():
    sc = scenes.city(seed=0, lots=8, extent=250.0, num_emissive_tris=200, env_size=(64, 32))
    per_building = 12 + 2 * 4 * 16 * 19  # box + two triangles per window, 16 x 19 windows per facade
    assert per_building == 2444
    assert sc.num_tris == 64 * per_building + 2
    emissive = sc.meshes[sc.meshes[:, 5] == 1]
    assert int(emissive[:, 3].sum()) // 3 == 200
    for m in emissive:  # emitters: radiance U[1, 20] x (1, 0.8, 0.55)
        r = sc.materials[m[4]][5:8]
        assert 1.0 <= r[0] <= 20.0 and np.isclose(r[1], 0.8 * r[0]) and np.isclose(r[2], 0.55 * r[0])
    # buildings stay inside their lots and under 200 m
    lo, hi = sc.positions.min(0), sc.positions.max(0)
    assert hi[1] <= 200.0 + 1e-3 and lo[1] >= -1e-3
    assert np.all(np.abs(sc.positions[:, [0, 2]]) <= 0.55 * 250.0 + 1e-3)
    assert np.allclose(np.linalg.norm(sc.normals, axis=1), 1.0, atol=1e-5)
    again = scenes.city(seed=0, lots=8, extent=250.0, num_emissive_tris=200, env_size=(64, 32))
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
