"""World-action support on the CPU: the glTF 2.0 reader (models for
SpawnModel), the wire sizes of the world actions, and the world-space
flattening rule the library applies (restated here in numpy; the GPU tests
check the library against it)."""
import base64
import json
import struct

import numpy as np

from appearance_b200 import gltf, scenes
from appearance_b200.renderer import PathTracer


def test_glb_round_trip(tmp_path):
    sc = scenes.icosphere_field(seed=5, num_spheres=6, num_emissive=2, subdiv=1, box=4.0, env_size=None)
    sc.materials[1, 8] = 0.5
    p = tmp_path / "m.glb"
    gltf.save_glb(str(p), sc)
    back = gltf.load(str(p))
    np.testing.assert_array_equal(back.positions, sc.positions)
    np.testing.assert_array_equal(back.normals, sc.normals)
    np.testing.assert_array_equal(back.indices, sc.indices)
    np.testing.assert_array_equal(back.meshes[:, :5], sc.meshes[:, :5])
    np.testing.assert_array_equal(back.meshes[:, 5], (sc.materials[sc.meshes[:, 4], 5:8] > 0).any(1))
    for k in (slice(0, 3), 3, 4, slice(5, 8), 8):
        np.testing.assert_allclose(back.materials[:, k], sc.materials[:, k], rtol=1e-6)
    np.testing.assert_allclose(back.materials[:, 9], sc.materials[:, 9], rtol=1e-6)  # eta = 1 / ior


def test_gltf_node_transforms_and_defaults(tmp_path):
    # one triangle, referenced by a child node under a translated, scaled parent;
    # no normals (computed), default material
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    buf = pos.tobytes()
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0]}],
           "nodes": [{"translation": [10, 0, 0], "scale": [2, 2, 2], "children": [1]},
                     {"rotation": [0, 0, 0.7071067811865476, 0.7071067811865476], "mesh": 0}],
           "meshes": [{"primitives": [{"attributes": {"POSITION": 0}}]}],
           "accessors": [{"bufferView": 0, "componentType": 5126, "count": 3, "type": "VEC3"}],
           "bufferViews": [{"buffer": 0, "byteLength": len(buf)}],
           "buffers": [{"byteLength": len(buf), "uri": "data:application/octet-stream;base64,"
                        + base64.b64encode(buf).decode()}]}
    p = tmp_path / "t.gltf"
    p.write_text(json.dumps(doc))
    m = gltf.load(str(p))
    # rotate 90 degrees about z, then scale 2, then translate 10 in x
    np.testing.assert_allclose(m.positions, [[10, 0, 0], [10, 2, 0], [8, 0, 0]], atol=1e-5)
    np.testing.assert_allclose(m.normals, [[0, 0, 1]] * 3, atol=1e-6)
    # no glTF material: the reference's Material::default()
    np.testing.assert_array_equal(m.materials, scenes.material()[None, :])


def test_world_action_wire_sizes():
    u = bytes(range(16))
    s = PathTracer.spawn_model_bytes(np.eye(4), u, "models/box.glb")
    assert len(s) == 336 and s[64:80] == u and s[80:94] == b"models/box.glb" and s[94:] == bytes(242)
    t = PathTracer.transform_model_bytes(np.eye(4), u)
    assert len(t) == 80 and t[64:] == u
    assert struct.unpack("<16f", s[:64]) == tuple(np.eye(4, dtype=np.float32).reshape(16))


def compose(base, model, transforms):
    """base + instances of `model`, as World::flatten lays them out."""
    return scenes.flatten_world(base, [model], [(0, m16) for m16 in transforms])


def test_flatten_rule_moves_points_and_keeps_normals_unit():
    model = scenes.icosphere_field(seed=1, num_spheres=2, num_emissive=0, subdiv=1, box=2.0, env_size=None)
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = [[0, -2, 0], [2, 0, 0], [0, 0, 3]]
    m[:3, 3] = [1, 2, 3]
    p, n = scenes.flatten_instance(model, m.T.reshape(16))  # column-major
    ref = model.positions.astype(np.float64) @ m[:3, :3].T.astype(np.float64) + m[:3, 3]
    np.testing.assert_allclose(p, ref, rtol=1e-6, atol=1e-5)
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-6)
    nref = model.normals.astype(np.float64) @ np.linalg.inv(m[:3, :3].astype(np.float64))
    nref /= np.linalg.norm(nref, axis=1, keepdims=True)
    np.testing.assert_allclose(n, nref, atol=1e-6)


def test_two_level_oracle_with_identity_instances_equals_the_flat_oracle():
    from oracle.oracle import OracleScene, OracleTwoLevel
    a = scenes.cornell_box()
    b = scenes.icosphere_field(seed=3, num_spheres=5, num_emissive=1, subdiv=1, box=0.8, env_size=None)
    eye = np.eye(4, dtype=np.float32).reshape(16)
    two = OracleTwoLevel([a, b], [(0, eye), (1, eye)])
    flat = OracleScene(compose(a, b, [eye]))
    rng = np.random.default_rng(2)
    o = rng.uniform(-0.5, 1.5, (4000, 3)).astype(np.float32)
    d = rng.normal(size=(4000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    got = two.closest(o, d, 1000.0)
    ref, _ = flat.closest(o, d, 1000.0)
    assert np.array_equal(got, ref.view(np.uint32))
    assert (got[:, 3] != 0xFFFFFFFF).mean() > 0.3
    np.testing.assert_array_equal(two.any(o, d, 0.7), flat.any(o, d, np.full(len(o), 0.7, np.float32)))




def compose_many(base, models, instances):
    return scenes.flatten_world(base, models, instances)
