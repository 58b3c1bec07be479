"""Generates the frozen fixtures in this folder from the CPU oracle.

The reference (Rust + WGSL on wgpu/Vulkan ray queries) cannot be built or run
here, so these fixtures freeze the oracle's own output: CPU tests check that
the oracle still reproduces them, GPU tests check the CUDA path against them.
Each fixture stores its exact inputs (scene arrays, camera matrices) next to
the images, because numpy's transcendental functions may round differently in
the last place on another CPU and would regenerate a slightly different scene.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from appearance_b200 import presets, scenes  # noqa: E402
from oracle.oracle import OracleFrame, OracleScene  # noqa: E402


def small_sphere_scene():
    return scenes.icosphere_field(seed=3, num_spheres=48, num_emissive=6, subdiv=2, box=12.0, env_size=(64, 32))


def cornell_case():
    sc = scenes.cornell_box()
    cam = scenes.cornell_camera()
    w = h = 32
    mats, _ = scenes.camera_matrices(cam["eye"], cam["target"], cam["fov"], cam["near"], cam["far"], w, h)
    cfg = dict(presets.PLAIN, sample_count=4)
    return sc, cfg, [mats], w, h


def spheres_case():
    sc = small_sphere_scene()
    w, h = 48, 32
    cfg = dict(presets.REALTIME_GI_SPATIAL, max_bounces=4)
    path = scenes.camera_spline(seed=3, frames=16, box=12.0)
    mats_list, prev = [], None
    for f in range(3):
        eye, tgt = path[f]
        mats, prev = scenes.camera_matrices(eye, tgt, 60.0, 0.01, 500.0, w, h, prev)
        mats_list.append(mats)
    return sc, cfg, mats_list, w, h


CASES = {"cornell_plain_32": cornell_case, "spheres_realtime_48x32": spheres_case}


SCENE_FIELDS = ("positions", "normals", "indices", "tri_material", "meshes", "materials", "sun")


def save_case(name, sc, cfg, mats_list, w, h, images):
    arrays = {f"scene_{k}": getattr(sc, k) for k in SCENE_FIELDS}
    if sc.env is not None:
        arrays["scene_env"] = sc.env
    np.savez_compressed(os.path.join(HERE, name + ".npz"), images=images, mats=np.stack(mats_list),
                        size=np.array([w, h]), cfg_keys=np.array(sorted(cfg)),
                        cfg_vals=np.array([float(cfg[k]) for k in sorted(cfg)]), **arrays)


def load_case(name):
    """Returns (scene, cfg, mats (F,4,16), w, h, images) exactly as frozen."""
    z = np.load(os.path.join(HERE, name + ".npz"))
    env = z["scene_env"] if "scene_env" in z.files else None
    sc = scenes.Scene(*(z[f"scene_{k}"] for k in SCENE_FIELDS[:-1]), env, z["scene_sun"])
    cfg = {}
    for k, v in zip(z["cfg_keys"], z["cfg_vals"]):
        cfg[str(k)] = float(v) if str(k) in ("di_temporal_m_factor", "gi_temporal_m_cap",
                                              "taa_history_influence") else int(v)
    w, h = (int(x) for x in z["size"])
    return sc, cfg, z["mats"], w, h, z["images"]


def render_frozen(sc, cfg, mats, w, h):
    fr = OracleFrame(OracleScene(sc), w, h, cfg, threads=os.cpu_count())
    return np.stack([fr.render(m) for m in mats])


def main():
    for name, make in CASES.items():
        sc, cfg, mats_list, w, h = make()
        imgs = render_frozen(sc, cfg, np.stack(mats_list), w, h)
        save_case(name, sc, cfg, mats_list, w, h, imgs)
        print(name, imgs.shape, float(imgs.mean()))


if __name__ == "__main__":
    main()
