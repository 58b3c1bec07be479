"""Builds libappearance_cuda.so in-tree for sm_100a with nvcc.

Flags that are part of the numerical contract: -fmad=false (no contraction of
separate multiplies and adds) and the default IEEE division / square root
(no --use_fast_math); host code is compiled with -ffp-contract=off.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libappearance_cuda.so")
SOURCES = ["frame.cu", "api.cu", "noalloc.cu", "serve.cu", "mlp.cu", "spectral.cu", "bvh_build.cpp", "spectral_fit.cpp",
           "world.cpp"]
HEADERS = ["detmath.h", "dev_common.cuh", "dev_shade.cuh", "traverse.cuh", "frame.cuh", "scene_layout.h",
           "bvh_build.h", "spectral.h", "spectral.cuh", "spectral_fit.h", "persistent.cuh", "device_scope.h",
           "spectral_tables.h", "spectral_data.h", "world.h", "traverse2.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-v"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "appearance_cuda.h"), __file__]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    def compile_one(s):
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = ["nvcc", *NVCC_FLAGS, "-c", s, "-o", o]
        if s.endswith(".cpp"):
            cmd = ["nvcc", "-x", "cu", *NVCC_FLAGS, "-c", s, "-o", o]
        return o, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as pool:
        results = list(pool.map(compile_one, srcs))
    objs, logs = [], []
    for s, (o, r) in zip(srcs, results):
        logs.append(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {s}")
        objs.append(o)
    tmp = LIB + ".tmp"
    r = subprocess.run(["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp,
                        "-lcudart"], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    with open(os.path.join(objdir, "ptxas.log"), "w") as f:
        f.write("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
