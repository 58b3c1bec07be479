"""Seeded synthetic scenes, environment maps and camera matrices.

The reference loads glTF assets (crates/appearance-model/src/asset.rs); the
benchmarks here use procedural scenes instead, generated deterministically from
a seed so that every run, the CUDA path and the CPU oracle see the same bytes.

A scene is a flat, instance-major list of meshes (each mesh is one
VertexPoolSlice of the reference, crates/appearance-path-tracer-gpu/assets/
shaders/shared/vertex_pool.wgsl:3-12) with world-space positions and normals,
per-triangle material indices relative to the mesh's first material, and Disney
material records in the order of ap_material (include/appearance_cuda.h).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# ap_material field offsets (26 float32 per material)
MAT_FLOATS = 26
_OFF = dict(color=0, metallic=3, roughness=4, emission=5, transmission=8, eta=9,
            subsurface=10, absorption=11, specular=14, specular_tint=15,
            anisotropic=18, sheen=19, sheen_tint=20, clearcoat=23,
            clearcoat_roughness=24, alpha_cutoff=25)


def material(color=(1.0, 1.0, 1.0), metallic=0.0, roughness=0.5, emission=(0.0, 0.0, 0.0),
             transmission=0.0, eta=1.0 / 1.5, subsurface=0.0, absorption=(0.0, 0.0, 0.0),
             specular=0.0, specular_tint=(1.0, 1.0, 1.0), anisotropic=0.0, sheen=0.0,
             sheen_tint=(0.0, 0.0, 0.0), clearcoat=0.0, clearcoat_roughness=0.0,
             alpha_cutoff=0.0) -> np.ndarray:
    """One material record; defaults follow Material::default()
    (crates/appearance-model/src/material.rs:42-76)."""
    m = np.zeros(MAT_FLOATS, np.float32)
    vals = dict(color=color, metallic=metallic, roughness=roughness, emission=emission,
                transmission=transmission, eta=eta, subsurface=subsurface, absorption=absorption,
                specular=specular, specular_tint=specular_tint, anisotropic=anisotropic,
                sheen=sheen, sheen_tint=sheen_tint, clearcoat=clearcoat,
                clearcoat_roughness=clearcoat_roughness, alpha_cutoff=alpha_cutoff)
    for k, v in vals.items():
        v = np.atleast_1d(np.asarray(v, np.float32))
        m[_OFF[k]:_OFF[k] + v.size] = v
    return m


@dataclasses.dataclass
class Scene:
    positions: np.ndarray      # (V, 3) float32, world space
    normals: np.ndarray        # (V, 3) float32, world space, unit length
    indices: np.ndarray        # (T, 3) uint32, relative to the mesh's first vertex
    tri_material: np.ndarray   # (T,) uint32, relative to the mesh's material_idx
    meshes: np.ndarray         # (M, 6) uint32: first_vertex, num_vertices, first_index,
                               #                num_indices, material_idx, emissive
    materials: np.ndarray      # (K, 26) float32
    env: np.ndarray | None     # (H, W, 3) float32 equirect, or None for black
    sun: np.ndarray            # (8,) float32: direction xyz, size, color xyz, intensity

    @property
    def num_tris(self) -> int:
        return int(self.indices.shape[0])


class _Builder:
    def __init__(self):
        self.pos, self.nrm, self.idx, self.tmat, self.meshes, self.mats = [], [], [], [], [], []
        self.nv = 0
        self.nt = 0

    def add_material(self, m: np.ndarray) -> int:
        self.mats.append(m)
        return len(self.mats) - 1

    def add_mesh(self, pos, nrm, idx, tri_mat, material_idx, emissive):
        pos = np.asarray(pos, np.float32).reshape(-1, 3)
        nrm = np.asarray(nrm, np.float32).reshape(-1, 3)
        idx = np.asarray(idx, np.uint32).reshape(-1, 3)
        self.meshes.append((self.nv, pos.shape[0], 3 * self.nt, 3 * idx.shape[0], material_idx,
                            1 if emissive else 0))
        self.pos.append(pos)
        self.nrm.append(nrm)
        self.idx.append(idx)
        self.tmat.append(np.asarray(tri_mat, np.uint32).reshape(-1))
        self.nv += pos.shape[0]
        self.nt += idx.shape[0]

    def finish(self, env, sun) -> Scene:
        return Scene(np.concatenate(self.pos), np.concatenate(self.nrm), np.concatenate(self.idx),
                     np.concatenate(self.tmat), np.asarray(self.meshes, np.uint32),
                     np.stack(self.mats).astype(np.float32), env, np.asarray(sun, np.float32))


def _quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3); flat normal = normalize(cross(p1-p0, p2-p0))."""
    p = np.array([p0, p1, p2, p3], np.float64)
    n = np.cross(p[1] - p[0], p[2] - p[0])
    n /= np.linalg.norm(n)
    return p, np.repeat(n[None], 4, 0), np.array([[0, 1, 2], [0, 2, 3]])


def _box(center, size, angle_deg):
    """Axis box of `size` rotated about +y, resting on y=0; 12 triangles, outward normals."""
    sx, sy, sz = size
    a = math.radians(angle_deg)
    rot = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    c = np.array([center[0], 0.0, center[1]])
    corners = lambda pts: (np.array(pts) * [sx / 2, sy, sz / 2]) @ rot.T + c
    faces = [  # each as four corners counter-clockwise seen from outside
        [(-1, 0, 1), (1, 0, 1), (1, 1, 1), (-1, 1, 1)],      # +z
        [(1, 0, -1), (-1, 0, -1), (-1, 1, -1), (1, 1, -1)],  # -z
        [(1, 0, 1), (1, 0, -1), (1, 1, -1), (1, 1, 1)],      # +x
        [(-1, 0, -1), (-1, 0, 1), (-1, 1, 1), (-1, 1, -1)],  # -x
        [(-1, 1, 1), (1, 1, 1), (1, 1, -1), (-1, 1, -1)],    # +y
        [(-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1)],    # -y
    ]
    P, N, I = [], [], []
    for f in faces:
        p, n, i = _quad(*corners(f))
        I.append(i + 4 * len(P))
        P.append(p)
        N.append(n)
    return np.concatenate(P), np.concatenate(N), np.concatenate(I)


def cornell_box(seed: int = 0) -> Scene:
    """Unit-room Cornell box: 5 wall quads, a short (0.3^3, -18 deg) and a tall
    (0.3x0.6x0.3, +15 deg) box, a 0.25x0.25 ceiling light of radiance (17,12,4);
    Lambertian Disney materials (roughness 1, metallic 0, specular 0).  The seed
    only jitters nothing (the layout is fixed) but is kept for the generator API."""
    del seed
    b = _Builder()
    red = b.add_material(material(color=(0.63, 0.065, 0.05), roughness=1.0))
    green = b.add_material(material(color=(0.14, 0.45, 0.091), roughness=1.0))
    white = b.add_material(material(color=(0.725, 0.725, 0.725), roughness=1.0))
    light = b.add_material(material(color=(0.78, 0.78, 0.78), roughness=1.0, emission=(17.0, 12.0, 4.0)))
    P, N, I, M = [], [], [], []

    def put(p, n, i, m):
        I.append(i + sum(x.shape[0] for x in P))
        P.append(p)
        N.append(n)
        M.append(np.full(i.shape[0], m, np.uint32))

    # front (z = 1) open; normals point into the room
    put(*_quad((0, 0, 1), (1, 0, 1), (1, 0, 0), (0, 0, 0)), white)   # floor, +y
    put(*_quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)), white)   # ceiling, -y
    put(*_quad((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)), white)   # back, +z
    put(*_quad((0, 0, 1), (0, 0, 0), (0, 1, 0), (0, 1, 1)), red)     # left, +x
    put(*_quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)), green)   # right, -x
    put(*_box((0.66, 0.40), (0.3, 0.3, 0.3), -18.0), white)
    put(*_box((0.33, 0.27), (0.3, 0.6, 0.3), 15.0), white)
    b.add_mesh(np.concatenate(P), np.concatenate(N), np.concatenate(I), np.concatenate(M) - red, red, False)
    y = 0.999
    lp, ln, li = _quad((0.375, y, 0.375), (0.625, y, 0.375), (0.625, y, 0.625), (0.375, y, 0.625))
    b.add_mesh(lp, ln, li, np.zeros(2, np.uint32), light, True)
    sun = np.array([0.0, -1.0, 0.0, 0.5, 1.0, 1.0, 1.0, 0.0], np.float32)
    return b.finish(None, sun)


def cornell_camera():
    """Pinhole looking down -z into the open front; 40 degree vertical fov."""
    return dict(eye=(0.5, 0.5, 0.5 + 0.5 / math.tan(math.radians(20.0)) + 0.02), target=(0.5, 0.5, 0.0),
                fov=40.0, near=0.001, far=100.0)


def icosphere(subdiv: int):
    """Unit icosphere; subdiv=3 gives 20 * 4^3 = 1280 triangles, 642 vertices."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    for _ in range(subdiv):
        cache = {}
        new_faces = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    return np.array(verts), np.array(faces, np.uint32)


def sky_env(width: int = 2048, height: int = 1024, sun_elevation_deg: float = 40.0,
            sun_azimuth_deg: float = 30.0, sun_peak: float = 1e4, sun_sigma: float = 0.01) -> np.ndarray:
    """Equirect HDR environment: zenith-to-horizon sky gradient, dark ground and a
    Gaussian sun lobe of the given peak.  Texel (x, y) covers the direction that
    unit_vector_to_panorama_coords (assets/shaders/math.wgsl:101-106) maps to
    ((x + 0.5) / width, (y + 0.5) / height)."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    phi = u * 2.0 * np.pi - np.pi              # atan2(z, x)
    theta = v * np.pi                           # acos(y)
    st = np.sin(theta)[:, None]
    d = np.stack([np.cos(phi)[None, :] * st, np.broadcast_to(np.cos(theta)[:, None], (height, width)),
                  np.sin(phi)[None, :] * st], -1)
    up = d[..., 1]
    zenith = np.array([0.25, 0.45, 1.0])
    horizon = np.array([0.9, 0.9, 1.0])
    ground = np.array([0.12, 0.1, 0.08])
    tsky = np.clip(up, 0.0, 1.0)[..., None] ** 0.5
    sky = horizon * (1 - tsky) + zenith * tsky
    img = np.where(up[..., None] >= 0.0, sky, ground * np.clip(1.0 + up[..., None], 0.0, 1.0))
    el, az = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sdir = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    ang = np.arccos(np.clip(d @ sdir, -1.0, 1.0))
    img = img + (sun_peak * np.exp(-0.5 * (ang / sun_sigma) ** 2))[..., None] * np.array([1.0, 0.95, 0.85])
    return img.astype(np.float32)


def icosphere_field(seed: int = 0, num_spheres: int = 1024, num_emissive: int = 64, subdiv: int = 3,
                    box: float = 40.0, env_size=(2048, 1024)) -> Scene:
    """1024 icospheres (1280 triangles each) with centres U[0,box]^3, radius
    log-uniform in [0.2, 2], per-sphere Disney materials (baseColor U[0.05,0.95]^3,
    metallic Bernoulli(0.3), roughness U[0.05,1], specular 0.5, clearcoat
    Bernoulli(0.2)), `num_emissive` of them emissive with radiance U[5,50]^3, on a
    2-triangle ground plane, lit by the sky_env environment."""
    rng = np.random.default_rng(seed)
    uv, uf = icosphere(subdiv)
    b = _Builder()
    centers = rng.uniform(0.0, box, size=(num_spheres, 3))
    radii = np.exp(rng.uniform(math.log(0.2), math.log(2.0), size=num_spheres))
    colors = rng.uniform(0.05, 0.95, size=(num_spheres, 3))
    metallic = (rng.uniform(size=num_spheres) < 0.3).astype(np.float32)
    rough = rng.uniform(0.05, 1.0, size=num_spheres)
    clear = (rng.uniform(size=num_spheres) < 0.2).astype(np.float32)
    emissive = np.zeros(num_spheres, bool)
    emissive[rng.choice(num_spheres, size=num_emissive, replace=False)] = True
    radiance = rng.uniform(5.0, 50.0, size=(num_spheres, 3))
    for i in range(num_spheres):
        m = b.add_material(material(color=colors[i], metallic=float(metallic[i]), roughness=float(rough[i]),
                                    specular=0.5, clearcoat=float(clear[i]),
                                    emission=radiance[i] if emissive[i] else (0.0, 0.0, 0.0)))
        b.add_mesh(uv * radii[i] + centers[i], uv, uf, np.zeros(uf.shape[0], np.uint32), m, bool(emissive[i]))
    g = b.add_material(material(color=(0.5, 0.5, 0.5), roughness=0.8))
    e = 100.0
    gp, gn, gi = _quad((-e, 0.0, box + e), (box + e, 0.0, box + e), (box + e, 0.0, -e), (-e, 0.0, -e))
    b.add_mesh(gp, gn, gi, np.zeros(2, np.uint32), g, False)
    env = sky_env(*env_size) if env_size else None
    sun = np.array([0.0, -1.0, 0.0, 0.5, 1.0, 1.0, 1.0, 0.0], np.float32)
    return b.finish(env, sun)


def city(seed: int = 0, lots: int = 64, extent: float = 2000.0, cols: int = 16, rows: int = 19,
         num_emissive_tris: int = 10000, env_size=(2048, 1024)) -> Scene:
    """Procedural city: a lots x lots grid of box buildings over extent x extent
    metres (64 x 64 on 2 km by default), footprint U[0.4, 0.85] of the lot per
    side, height log-uniform in [5, 200] m, facade colour U[0.2, 0.8]^3 (diffuse).
    Every facade carries a cols x rows grid of window quads 5 cm in front of it
    (cell fill U[0.5, 0.8] per building; mirror-like metallic grey), so a
    building has 12 + 8 cols rows triangles (2444 by default; 10.0M triangles
    over 4096 buildings).  num_emissive_tris / 2 windows drawn uniformly over the
    city are emitters of radiance U[1, 20] x (1, 0.8, 0.55), grouped per building
    into emissive meshes; a 1.1 x extent ground quad and the sky_env
    environment complete the scene.  Each building is its own mesh (flattened
    at upload like every instance)."""
    rng = np.random.default_rng(seed)
    nb = lots * lots
    lot = extent / lots
    gx, gz = np.meshgrid(np.arange(lots), np.arange(lots), indexing="ij")
    cx = (gx.reshape(-1) + 0.5) * lot - extent / 2
    cz = (gz.reshape(-1) + 0.5) * lot - extent / 2
    sx = rng.uniform(0.4, 0.85, nb) * lot
    sz = rng.uniform(0.4, 0.85, nb) * lot
    cx = cx + rng.uniform(-0.5, 0.5, nb) * (lot - sx) * 0.9
    cz = cz + rng.uniform(-0.5, 0.5, nb) * (lot - sz) * 0.9
    height = np.exp(rng.uniform(math.log(5.0), math.log(200.0), nb))
    facade = rng.uniform(0.2, 0.8, (nb, 3))
    fill = rng.uniform(0.5, 0.8, (nb, 2))
    nwin = 4 * cols * rows
    emit_flat = rng.choice(nb * nwin, size=num_emissive_tris // 2, replace=False)
    emissive = np.zeros(nb * nwin, bool)
    emissive[emit_flat] = True
    emissive = emissive.reshape(nb, nwin)
    radiance = rng.uniform(1.0, 20.0, nb * nwin).reshape(nb, nwin)

    # window corners of all buildings: facade f spans corner a -> b at the base,
    # outward normal n; window (c, r) covers the middle fill fraction of its cell
    hx, hz = sx / 2, sz / 2
    fac = [  # (start xz, end xz, normal xz) in units of the half extents
        ((-1, 1), (1, 1), (0, 1)), ((1, -1), (-1, -1), (0, -1)), ((1, 1), (1, -1), (1, 0)), ((-1, -1), (-1, 1), (-1, 0))]
    c_idx, r_idx = np.meshgrid(np.arange(cols), np.arange(rows), indexing="ij")
    c_idx, r_idx = c_idx.reshape(-1), r_idx.reshape(-1)
    win_p = np.zeros((nb, 4, cols * rows, 4, 3), np.float64)
    win_n = np.zeros((nb, 4, 3), np.float64)
    for f, ((ax, az), (bx, bz), (nx, nz)) in enumerate(fac):
        a = np.stack([cx + ax * hx, np.zeros(nb), cz + az * hz], -1)
        b_ = np.stack([cx + bx * hx, np.zeros(nb), cz + bz * hz], -1)
        n = np.array([nx, 0.0, nz])
        win_n[:, f] = n
        u0 = (c_idx[None] + 0.5 - fill[:, :1] / 2) / cols
        u1 = (c_idx[None] + 0.5 + fill[:, :1] / 2) / cols
        v0 = (r_idx[None] + 0.5 - fill[:, 1:] / 2) / rows * height[:, None]
        v1 = (r_idx[None] + 0.5 + fill[:, 1:] / 2) / rows * height[:, None]
        along = (b_ - a)[:, None, :]
        base = a[:, None, :] + 0.05 * n
        up = np.array([0.0, 1.0, 0.0])
        for k, (uu, vv) in enumerate(((u0, v0), (u1, v0), (u1, v1), (u0, v1))):
            win_p[:, f, :, k] = base + uu[..., None] * along + vv[..., None] * up
    win_p = win_p.reshape(nb, nwin, 4, 3).astype(np.float32)
    quad_i = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)

    b = _Builder()
    glass = material(color=(0.55, 0.6, 0.65), metallic=1.0, roughness=0.1)
    for i in range(nb):
        box_p, box_n, box_i = _box((cx[i], cz[i]), (sx[i], height[i], sz[i]), 0.0)
        keep = ~emissive[i]
        wp = win_p[i, keep].reshape(-1, 3)
        wn = np.repeat(np.repeat(win_n[i], cols * rows, 0)[keep], 4, 0)
        nk = int(keep.sum())
        wi = (quad_i[None] + 4 * np.arange(nk, dtype=np.uint32)[:, None, None]).reshape(-1, 3) + box_p.shape[0]
        m = b.add_material(material(color=facade[i], roughness=0.9))
        b.add_material(glass)
        tm = np.concatenate([np.zeros(12, np.uint32), np.ones(2 * nk, np.uint32)])
        b.add_mesh(np.concatenate([box_p, wp]), np.concatenate([box_n, wn]), np.concatenate([box_i, wi]), tm, m,
                   False)
        ne = int(emissive[i].sum())
        if ne:
            ep = win_p[i, emissive[i]].reshape(-1, 3)
            en = np.repeat(np.repeat(win_n[i], cols * rows, 0)[emissive[i]], 4, 0)
            ei = (quad_i[None] + 4 * np.arange(ne, dtype=np.uint32)[:, None, None]).reshape(-1, 3)
            first = None
            for r in radiance[i, emissive[i]]:
                k = b.add_material(material(color=(0.8, 0.8, 0.8), roughness=1.0,
                                            emission=(r, 0.8 * r, 0.55 * r)))
                first = k if first is None else first
            b.add_mesh(ep, en, ei, np.repeat(np.arange(ne, dtype=np.uint32), 2), first, True)
    g = b.add_material(material(color=(0.3, 0.3, 0.3), roughness=0.9))
    e = 0.55 * extent
    gp, gn, gi = _quad((-e, 0.0, e), (e, 0.0, e), (e, 0.0, -e), (-e, 0.0, -e))
    b.add_mesh(gp, gn, gi, np.zeros(2, np.uint32), g, False)
    env = sky_env(*env_size) if env_size else None
    sun = np.array([0.3, -1.0, 0.2, 0.5, 1.0, 1.0, 0.95, 0.0], np.float32)
    return b.finish(env, sun)


def city_instanced(seed: int = 0, lots: int = 64, extent: float = 2000.0, variants: int = 64,
                   emissive_windows: int = 4, env_size=(2048, 1024)):
    """The procedural city as instances: `variants` building models (each one
    lot of `city`, with its window grid and `emissive_windows` emissive
    windows, built in lot-local coordinates), placed on the lots x lots grid
    by a translation and a rotation by a multiple of 90 degrees.  With the
    defaults 4096 instances of 64 models: 10.0M world triangles from 156k
    model triangles.  Returns (base, models, instances): the base scene (the
    ground quad, the sky and the sun), the model Scenes, and (model index,
    column-major 4x4 transform) per instance."""
    rng = np.random.default_rng(seed)
    lot = extent / lots
    models = []
    for k in range(variants):
        m = city(seed=seed * 1000 + k + 1, lots=1, extent=lot, num_emissive_tris=2 * emissive_windows, env_size=None)
        keep = m.meshes.shape[0] - 1  # drop the lot's ground quad (the last mesh)
        last_tri = int(m.meshes[keep, 2]) // 3
        last_vtx = int(m.meshes[keep, 0])
        models.append(Scene(positions=m.positions[:last_vtx], normals=m.normals[:last_vtx],
                            indices=m.indices[:last_tri], tri_material=m.tri_material[:last_tri],
                            meshes=m.meshes[:keep].copy(), materials=m.materials[:-1].copy(), env=None,
                            sun=np.zeros(8, np.float32)))
    gx, gz = np.meshgrid(np.arange(lots), np.arange(lots), indexing="ij")
    cx = (gx.reshape(-1) + 0.5) * lot - extent / 2
    cz = (gz.reshape(-1) + 0.5) * lot - extent / 2
    which = rng.integers(0, variants, lots * lots)
    turn = rng.integers(0, 4, lots * lots)
    instances = []
    for i in range(lots * lots):
        c, s = [(1, 0), (0, 1), (-1, 0), (0, -1)][turn[i]]
        t = np.eye(4, dtype=np.float32)
        t[:3, :3] = [[c, 0, s], [0, 1, 0], [-s, 0, c]]
        t[:3, 3] = [cx[i], 0.0, cz[i]]
        instances.append((int(which[i]), t.T.reshape(16).copy()))
    b = _Builder()
    g = b.add_material(material(color=(0.3, 0.3, 0.3), roughness=0.9))
    e = 0.55 * extent
    gp, gn, gi = _quad((-e, 0.0, e), (e, 0.0, e), (e, 0.0, -e), (-e, 0.0, -e))
    b.add_mesh(gp, gn, gi, np.zeros(2, np.uint32), g, False)
    env = sky_env(*env_size) if env_size else None
    sun = np.array([0.3, -1.0, 0.2, 0.5, 1.0, 1.0, 0.95, 0.0], np.float32)
    return b.finish(env, sun), models, instances


def flatten_instance(model, m16):
    """One instance in world space with the library's arithmetic (World::flatten,
    csrc/world.cpp):
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



def flatten_world(base, models, instances):
    """The world of a base scene and instances of models (model index,
    column-major 4x4) as one Scene, in the layout of the library's World::flatten
    (csrc/world.cpp): base first, then each instance's meshes in order, a
    model's materials appended at its first use; the same float32 arithmetic,
    so that the flattened upload equals the world the library builds."""
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
    return Scene(positions=np.concatenate(pos), normals=np.concatenate(nrm), indices=np.concatenate(idx),
                        tri_material=np.concatenate(tm), meshes=np.asarray(meshes, np.uint32),
                        materials=np.concatenate(mats).astype(np.float32), env=base.env, sun=base.sun)


def city_camera(extent: float = 2000.0):
    """Elevated view over the city towards its centre."""
    return dict(eye=(-0.42 * extent, 0.12 * extent, -0.42 * extent), target=(0.0, 20.0, 0.0), fov=50.0)


def camera_spline(seed: int = 0, frames: int = 64, box: float = 40.0):
    """Closed Catmull-Rom spline through 8 seeded control points circling the
    field; returns `frames` (eye, target) pairs."""
    rng = np.random.default_rng(seed + 1000)
    k = 8
    ang = np.linspace(0.0, 2.0 * np.pi, k, endpoint=False) + rng.uniform(-0.2, 0.2, k)
    rad = rng.uniform(0.9, 1.2, k) * box
    ctrl = np.stack([box / 2 + rad * np.cos(ang), rng.uniform(0.25, 0.6, k) * box,
                     box / 2 + rad * np.sin(ang)], -1)
    out = []
    for f in range(frames):
        s = f / frames * k
        i = int(s)
        t = s - i
        p0, p1, p2, p3 = (ctrl[(i + j) % k] for j in (-1, 0, 1, 2))
        eye = 0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t * t +
                     (-p0 + 3 * p1 - 3 * p2 + p3) * t ** 3)
        out.append((tuple(eye), (box / 2, box * 0.2, box / 2)))
    return out


# --------------------------------------------------------------------------
# Camera matrices: glam's perspective_rh and look_to_rh
# (crates/appearance-camera/src/lib.rs:124-136; appearance-transform get_view_matrix),
# computed in float64 and rounded once to float32.

def perspective_rh(fov_y_deg, aspect, near, far):
    f = 1.0 / math.tan(0.5 * math.radians(fov_y_deg))
    r = far / (near - far)
    m = np.zeros((4, 4))
    m[0, 0] = f / aspect
    m[1, 1] = f
    m[2, 2] = r
    m[3, 2] = -1.0
    m[2, 3] = r * near
    return m


def look_at_rh(eye, target, up=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, u, -f
    m[0, 3], m[1, 3], m[2, 3] = -s @ eye, -u @ eye, f @ eye
    return m


def camera_matrices(eye, target, fov, near, far, width, height, prev=None):
    """Returns float32 (4, 16) column-major: inv_view, inv_proj, view_proj, prev_view_proj.
    `prev` is the previous frame's view_proj (float64 4x4) or None (no motion)."""
    view = look_at_rh(eye, target)
    proj = perspective_rh(fov, width / height, near, far)
    vp = proj @ view
    pvp = vp if prev is None else prev
    mats = [np.linalg.inv(view), np.linalg.inv(proj), vp, pvp]
    return np.stack([m.T.reshape(16) for m in mats]).astype(np.float32), vp
