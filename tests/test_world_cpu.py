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


def flatten_instance(model, m16):
    """One instance in world space with the library's arithmetic (world.cpp):
    positions m * (p, 1) summed left to right in float32; normals by the
    inverse transpose of the upper 3x3 (cofactors over the determinant in
    double, rounded to float), renormalised in float32."""
    m = np.asarray(m16, np.float32).reshape(16)
    f = np.float32
    x, y, z = (model.positions[:, k].astype(f) for k in range(3))
    pos = np.stack([((m[r] * x + m[4 + r] * y) + m[8 + r] * z) + m[12 + r] for r in range(3)], 1).astype(f)
    a = [[float(m[4 * c + r]) for r in range(3)] for c in range(3)]
    det = (a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) - a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2])
           + a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]))
    nt = np.zeros((3, 3), f)
    for r in range(3):
        for k in range(3):
            r1, r2, k1, k2 = (r + 1) % 3, (r + 2) % 3, (k + 1) % 3, (k + 2) % 3
            nt[r, k] = f((a[k1][r1] * a[k2][r2] - a[k2][r1] * a[k1][r2]) / det)
    nx, ny, nz = (model.normals[:, k].astype(f) for k in range(3))
    n = np.stack([(nt[r, 0] * nx + nt[r, 1] * ny) + nt[r, 2] * nz for r in range(3)], 1).astype(f)
    ln = np.sqrt((n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]).astype(f)
    s = np.where(ln > 0, f(1.0) / np.where(ln > 0, ln, f(1.0)), f(0.0)).astype(f)
    return pos, (n * s[:, None]).astype(f)


def compose(base, model, transforms):
    """base + instances of `model`, as World::flatten lays them out."""
    pos, nrm, idx, tm, meshes = [base.positions], [base.normals], [base.indices], [base.tri_material], list(base.meshes)
    mats = [base.materials, model.materials]
    mat0 = base.materials.shape[0]
    nv, nt = base.positions.shape[0], base.indices.shape[0]
    for m16 in transforms:
        p, n = flatten_instance(model, m16)
        pos.append(p)
        nrm.append(n)
        idx.append(model.indices)
        tm.append(model.tri_material)
        for fv, cnt, fi, ni, mi, em in model.meshes:
            meshes.append((fv + nv, cnt, fi + 3 * nt, ni, mi + mat0, em))
        nv += model.positions.shape[0]
        nt += model.indices.shape[0]
    return scenes.Scene(positions=np.concatenate(pos), normals=np.concatenate(nrm), indices=np.concatenate(idx),
                        tri_material=np.concatenate(tm), meshes=np.asarray(meshes, np.uint32),
                        materials=np.concatenate(mats).astype(np.float32), env=base.env, sun=base.sun)


def test_flatten_rule_moves_points_and_keeps_normals_unit():
    model = scenes.icosphere_field(seed=1, num_spheres=2, num_emissive=0, subdiv=1, box=2.0, env_size=None)
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = [[0, -2, 0], [2, 0, 0], [0, 0, 3]]
    m[:3, 3] = [1, 2, 3]
    p, n = flatten_instance(model, m.T.reshape(16))  # column-major
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
    """base + instances of several models (model index, column-major 4x4) in
    World::flatten's layout (a model's materials appended at its first use)."""
    pos, nrm, idx, tm, meshes = [base.positions], [base.normals], [base.indices], [base.tri_material], list(base.meshes)
    mats = [base.materials]
    mat_base = {}
    nmat = base.materials.shape[0]
    nv, nt = base.positions.shape[0], base.indices.shape[0]
    for k, m16 in instances:
        model = models[k]
        if k not in mat_base:
            mat_base[k] = nmat
            mats.append(model.materials)
            nmat += model.materials.shape[0]
        p, n = flatten_instance(model, m16)
        pos.append(p)
        nrm.append(n)
        idx.append(model.indices)
        tm.append(model.tri_material)
        for fv, cnt, fi, ni, mi, em in model.meshes:
            meshes.append((fv + nv, cnt, fi + 3 * nt, ni, mi + mat_base[k], em))
        nv += model.positions.shape[0]
        nt += model.indices.shape[0]
    return scenes.Scene(positions=np.concatenate(pos), normals=np.concatenate(nrm), indices=np.concatenate(idx),
                        tri_material=np.concatenate(tm), meshes=np.asarray(meshes, np.uint32),
                        materials=np.concatenate(mats).astype(np.float32), env=base.env, sun=base.sun)
