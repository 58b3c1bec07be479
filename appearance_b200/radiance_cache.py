"""Host side of the radiance cache (ap_rc_* in include/appearance_cuda.h).

A small MLP (144 encoded inputs, 4 hidden layers of 64 with ReLU, 3 outputs
with exp; FP16 weights and activations, FP32 accumulation and master weights)
that predicts the outgoing radiance of a path vertex.  Inference runs on the
tensor cores (tcgen05); training computes the relative L2 loss, its gradients
and an Adam step on the GPU.  A query is 16 floats: position (3), roughness,
outgoing direction (3), 0, diffuse albedo (3), specular albedo (3), 0, 0.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .renderer import RendererError

NUM_PARAMS = 21696
QUERY_FLOATS = 16


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RadianceCache:
    def __init__(self, scene_lo, scene_hi, seed: int = 0, device: int = 0):
        self._lib = _native.load()
        lo = np.ascontiguousarray(scene_lo, np.float32)
        hi = np.ascontiguousarray(scene_hi, np.float32)
        err = ctypes.c_int(0)
        self._c = self._lib.ap_rc_create(device, _p(lo), _p(hi), seed, ctypes.byref(err))
        if not self._c:
            raise RendererError(err.value, "ap_rc_create failed")

    def _check(self, rc):
        if rc != _native.AP_OK:
            raise RendererError(rc, self._lib.ap_rc_last_error(self._c).decode())

    def close(self):
        if getattr(self, "_c", None):
            self._lib.ap_rc_destroy(self._c)
            self._c = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        out = np.zeros(NUM_PARAMS, np.float32)
        self._check(self._lib.ap_rc_get_params(self._c, _p(out), NUM_PARAMS))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self._check(self._lib.ap_rc_set_params(self._c, _p(p), p.size))

    def infer(self, queries) -> np.ndarray:
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, QUERY_FLOATS)
        out = np.zeros((q.shape[0], 3), np.float32)
        self._check(self._lib.ap_rc_infer(self._c, _p(q), q.shape[0], _p(out)))
        return out

    def train(self, queries, targets, lr: float = 1e-3, update: bool = True, want_grad: bool = False):
        """One step; returns (loss, gradient or None)."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, QUERY_FLOATS)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        loss = ctypes.c_float(0.0)
        g = np.zeros(NUM_PARAMS, np.float32) if want_grad else None
        self._check(self._lib.ap_rc_train(self._c, _p(q), _p(t), q.shape[0], lr, 1 if update else 0,
                                          ctypes.byref(loss), None if g is None else _p(g)))
        return loss.value, g


def random_queries(n: int, seed: int, lo=(-1.0, -1.0, -1.0), hi=(11.0, 11.0, 11.0)) -> np.ndarray:
    """n seeded query records (16 floats each): positions uniform in the box,
    roughness in [0.05, 1], unit directions, albedos in [0, 1]."""
    rng = np.random.default_rng(seed)
    q = np.zeros((n, QUERY_FLOATS), np.float32)
    q[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    q[:, 3] = rng.uniform(0.05, 1.0, n)
    d = rng.normal(size=(n, 3))
    q[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 8:14] = rng.uniform(0.0, 1.0, (n, 6))
    return q


def _bench_cli(argv=None):
    """Runs inference over --infer queries (--infer-calls times) and --steps
    training steps of --train samples on seeded random queries: the fixed
    command that profiler captures of the cache's kernels run."""
    import argparse

    ap = argparse.ArgumentParser(prog="python -m appearance_b200.radiance_cache")
    ap.add_argument("--infer", type=int, default=1 << 19)
    ap.add_argument("--infer-calls", type=int, default=3)
    ap.add_argument("--train", type=int, default=1 << 16)
    ap.add_argument("--steps", type=int, default=4)
    a = ap.parse_args(argv)
    lo, hi = np.array([-1.0] * 3, np.float32), np.array([11.0] * 3, np.float32)
    rc = RadianceCache(lo, hi, seed=3)
    q = random_queries(a.infer, 77)
    for _ in range(a.infer_calls):
        rc.infer(q)
    qt = random_queries(a.train, 5)
    t = np.random.default_rng(8).uniform(0.0, 3.0, (a.train, 3)).astype(np.float32)
    for _ in range(a.steps):
        loss, _ = rc.train(qt, t, lr=1e-3)
        print(f"train loss {loss:.6f}", flush=True)
    rc.close()


if __name__ == "__main__":
    _bench_cli()
