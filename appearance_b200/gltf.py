"""glTF 2.0 models (.gltf with embedded or external buffers, or .glb) as the
model-space Scene that ap_model_register takes.

The reference loads its models with the `gltf` crate
(crates/appearance-model/src/asset.rs): every mesh primitive of the scene's
node tree becomes geometry under its node's accumulated transform
(rebuild_tlas_rec, crates/appearance-path-tracer-gpu/src/scene_resources/
mod.rs:159-216), and each glTF material fills a Material record
(asset.rs:195-260): base colour, metallic, roughness, emission times the
emissive strength, transmission, eta = 1 / ior (1.5 by default), volume
absorption, specular, clearcoat.  This module reads the same fields with its
own parser; textures are not read (the synthetic scenes carry constant
material parameters).  Triangle primitives only (mode 4).
"""
from __future__ import annotations

import base64
import json
import os
import struct

import numpy as np

from .scenes import Scene, material

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_COUNT = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


def _read(path: str):
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] == b"glTF":  # binary container: header, JSON chunk, optional BIN chunk
        _, _, length = struct.unpack_from("<III", data, 0)
        off, doc, binary = 12, None, None
        while off < length:
            clen, ctype = struct.unpack_from("<II", data, off)
            chunk = data[off + 8:off + 8 + clen]
            if ctype == 0x4E4F534A:
                doc = json.loads(chunk.decode("utf-8"))
            elif ctype == 0x004E4942:
                binary = chunk
            off += 8 + clen
        return doc, binary
    return json.loads(data.decode("utf-8")), None


def _buffers(doc, binary, base_dir):
    out = []
    for i, b in enumerate(doc.get("buffers", [])):
        uri = b.get("uri")
        if uri is None:
            if binary is None or i != 0:
                raise ValueError("glTF buffer without data")
            out.append(binary)
        elif uri.startswith("data:"):
            out.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            with open(os.path.join(base_dir, uri), "rb") as f:
                out.append(f.read())
    return out


def _accessor(doc, buffers, idx):
    a = doc["accessors"][idx]
    dt, n = np.dtype(_COMPONENT[a["componentType"]]), _COUNT[a["type"]]
    count = a["count"]
    if "bufferView" not in a:
        return np.zeros((count, n), dt)
    bv = doc["bufferViews"][a["bufferView"]]
    buf = buffers[bv["buffer"]]
    start = bv.get("byteOffset", 0) + a.get("byteOffset", 0)
    stride = bv.get("byteStride", 0) or dt.itemsize * n
    rows = np.ndarray((count, n), dt, buffer=buf, offset=start, strides=(stride, dt.itemsize))
    return np.array(rows)


def _node_matrix(node) -> np.ndarray:
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).T  # column-major in the file
    t = np.asarray(node.get("translation", [0, 0, 0]), np.float64)
    x, y, z, w = node.get("rotation", [0, 0, 0, 1])
    s = np.asarray(node.get("scale", [1, 1, 1]), np.float64)
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    m = np.eye(4)
    m[:3, :3] = r * s[None, :]
    m[:3, 3] = t
    return m


def _material(m: dict) -> np.ndarray:
    pbr = m.get("pbrMetallicRoughness", {})
    ext = m.get("extensions", {})
    emission = np.asarray(m.get("emissiveFactor", [0, 0, 0]), np.float32)
    emission = emission * ext.get("KHR_materials_emissive_strength", {}).get("emissiveStrength", 1.0)
    absorption = (0.0, 0.0, 0.0)
    if "KHR_materials_volume" in ext:
        v = ext["KHR_materials_volume"]
        dist = v.get("attenuationDistance", float("inf"))
        absorption = tuple((1.0 - np.asarray(v.get("attenuationColor", [1, 1, 1]), np.float64)) / dist)
    spec = ext.get("KHR_materials_specular", {})
    cc = ext.get("KHR_materials_clearcoat", {})
    return material(color=tuple(pbr.get("baseColorFactor", [1, 1, 1, 1])[:3]),
                    metallic=pbr.get("metallicFactor", 1.0), roughness=pbr.get("roughnessFactor", 1.0),
                    emission=tuple(emission), absorption=absorption,
                    transmission=ext.get("KHR_materials_transmission", {}).get("transmissionFactor", 0.0),
                    eta=1.0 / ext.get("KHR_materials_ior", {}).get("ior", 1.5),
                    specular=spec.get("specularFactor", 0.0),
                    specular_tint=tuple(spec.get("specularColorFactor", [1, 1, 1])),
                    clearcoat=cc.get("clearcoatFactor", 0.0),
                    clearcoat_roughness=cc.get("clearcoatRoughnessFactor", 0.0),
                    alpha_cutoff=m.get("alphaCutoff", 0.5) if m.get("alphaMode") == "MASK" else 0.0)


def _vertex_normals(pos: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals for primitives that carry none."""
    p = pos.astype(np.float64)
    fn = np.cross(p[idx[:, 1]] - p[idx[:, 0]], p[idx[:, 2]] - p[idx[:, 0]])
    n = np.zeros_like(p)
    for k in range(3):
        np.add.at(n, idx[:, k], fn)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    return np.where(ln > 0, n / np.maximum(ln, 1e-300), [0.0, 1.0, 0.0])


def load(path: str) -> Scene:
    """The model at `path` in model space: one mesh per triangle primitive."""
    doc, binary = _read(path)
    buffers = _buffers(doc, binary, os.path.dirname(os.path.abspath(path)))
    mats = [_material(m) for m in doc.get("materials", [])] or [material()]
    pos_l, nrm_l, idx_l, tm_l, meshes = [], [], [], [], []
    nv = nt = 0
    scene = doc.get("scenes", [{}])[doc.get("scene", 0)] if doc.get("scenes") else {"nodes": []}
    stack = [(n, np.eye(4)) for n in reversed(scene.get("nodes", []))]
    while stack:
        ni, parent = stack.pop()
        node = doc["nodes"][ni]
        m = parent @ _node_matrix(node)
        for c in reversed(node.get("children", [])):
            stack.append((c, m))
        if "mesh" not in node:
            continue
        nrm_m = np.linalg.inv(m[:3, :3]).T
        for prim in doc["meshes"][node["mesh"]]["primitives"]:
            if prim.get("mode", 4) != 4:
                continue
            attrs = prim["attributes"]
            pos = _accessor(doc, buffers, attrs["POSITION"]).astype(np.float64)
            idx = (_accessor(doc, buffers, prim["indices"]).reshape(-1, 3).astype(np.uint32) if "indices" in prim
                   else np.arange(pos.shape[0], dtype=np.uint32).reshape(-1, 3))
            nrm = (_accessor(doc, buffers, attrs["NORMAL"]).astype(np.float64) if "NORMAL" in attrs
                   else _vertex_normals(pos, idx))
            pw = pos @ m[:3, :3].T + m[:3, 3]
            nw = nrm @ nrm_m.T
            nw /= np.maximum(np.linalg.norm(nw, axis=1, keepdims=True), 1e-300)
            mi = prim.get("material", 0)
            if mi >= len(mats):
                mi = 0
            emissive = bool(np.any(mats[mi][5:8] > 0))
            meshes.append((nv, pw.shape[0], 3 * nt, 3 * idx.shape[0], mi, 1 if emissive else 0))
            pos_l.append(pw.astype(np.float32))
            nrm_l.append(nw.astype(np.float32))
            idx_l.append(idx)
            tm_l.append(np.zeros(idx.shape[0], np.uint32))
            nv += pw.shape[0]
            nt += idx.shape[0]
    if not meshes:
        raise ValueError(f"{path}: no triangle primitives")
    return Scene(positions=np.concatenate(pos_l), normals=np.concatenate(nrm_l), indices=np.concatenate(idx_l),
                 tri_material=np.concatenate(tm_l), meshes=np.asarray(meshes, np.uint32),
                 materials=np.stack(mats).astype(np.float32), env=None, sun=np.zeros(8, np.float32))


def save_glb(path: str, scene: Scene) -> None:
    """Writes a Scene's meshes as a .glb (one node and primitive per mesh,
    constant materials); the inverse of load for these fields."""
    blobs, views, accessors, meshes, nodes = [], [], [], [], []

    def add(arr, target, ctype, typ):
        raw = np.ascontiguousarray(arr).tobytes()
        off = sum(len(b) for b in blobs)
        blobs.append(raw + bytes((-len(raw)) % 4))
        views.append({"buffer": 0, "byteOffset": off, "byteLength": len(raw), "target": target})
        acc = {"bufferView": len(views) - 1, "componentType": ctype, "count": int(arr.shape[0]), "type": typ}
        if typ == "VEC3" and ctype == 5126:
            acc["min"] = [float(v) for v in arr.min(0)]
            acc["max"] = [float(v) for v in arr.max(0)]
        accessors.append(acc)
        return len(accessors) - 1

    for fv, nvx, fi, ni, mi, _ in scene.meshes:
        p = add(scene.positions[fv:fv + nvx], 34962, 5126, "VEC3")
        n = add(scene.normals[fv:fv + nvx], 34962, 5126, "VEC3")
        ix = add(scene.indices[fi // 3:(fi + ni) // 3].reshape(-1), 34963, 5125, "SCALAR")
        meshes.append({"primitives": [{"attributes": {"POSITION": p, "NORMAL": n}, "indices": ix,
                                       "material": int(mi)}]})
        nodes.append({"mesh": len(meshes) - 1})
    mats = []
    for m in scene.materials:
        mats.append({"pbrMetallicRoughness": {"baseColorFactor": [float(m[0]), float(m[1]), float(m[2]), 1.0],
                                              "metallicFactor": float(m[3]), "roughnessFactor": float(m[4])},
                     "emissiveFactor": [float(v) for v in m[5:8]],
                     "extensions": {"KHR_materials_transmission": {"transmissionFactor": float(m[8])},
                                    "KHR_materials_ior": {"ior": float(1.0 / m[9]) if m[9] else 1.5}}})
    binary = b"".join(blobs)
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": list(range(len(nodes)))}],
           "nodes": nodes, "meshes": meshes, "materials": mats, "accessors": accessors, "bufferViews": views,
           "buffers": [{"byteLength": len(binary)}]}
    js = json.dumps(doc).encode()
    js += b" " * ((-len(js)) % 4)
    out = struct.pack("<III", 0x46546C67, 2, 12 + 8 + len(js) + 8 + len(binary))
    out += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(binary), 0x004E4942) + binary
    with open(path, "wb") as f:
        f.write(out)
