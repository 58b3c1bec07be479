"""Radiance cache on the GPU against the numpy oracle (oracle/mlp_oracle.py):
tensor-core inference, training gradients and the Adam step; and that training
fits a smooth radiance field."""
import ctypes

import numpy as np
import pytest

from appearance_b200.radiance_cache import NUM_PARAMS, RadianceCache
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu
LO, HI = np.array([-1.0, -1.0, -1.0], np.float32), np.array([11.0, 11.0, 11.0], np.float32)


def rand_queries(n, seed):
    rng = np.random.default_rng(seed)
    q = np.zeros((n, 16), np.float32)
    q[:, 0:3] = rng.uniform(-1.0, 11.0, (n, 3))
    q[:, 3] = rng.uniform(0.05, 1.0, n)
    d = rng.normal(size=(n, 3))
    q[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 8:14] = rng.uniform(0.0, 1.0, (n, 6))
    return q


def rand_params(seed, scale=0.12):
    return (np.random.default_rng(seed).normal(size=NUM_PARAMS) * scale).astype(np.float32)


def test_tensor_core_inference_matches_oracle():
    rc = RadianceCache(LO, HI, seed=3)
    p = rand_params(4)
    rc.set_params(p)
    for n in (1000, 128, 1):  # partial, exact and single-query tiles
        q = rand_queries(n, 5 + n)
        got = rc.infer(q)
        ref = mo.predict(p, mo.encode(q, LO, HI))
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-3)
        # FP16 activations, FP32 accumulation in a different order: rare roundings
        # of an activation to the neighbouring FP16 value
        assert np.median(rel) < 1e-3, np.median(rel)
        assert np.max(rel) < 2e-2, np.max(rel)
    rc.close()


def test_gradients_match_oracle():
    rc = RadianceCache(LO, HI, seed=3)
    p = rand_params(6)
    rc.set_params(p)
    q = rand_queries(3000, 7)
    t = np.random.default_rng(8).uniform(0.0, 3.0, (3000, 3)).astype(np.float32)
    loss, g = rc.train(q, t, update=False, want_grad=True)
    ref_loss, ref_g = mo.loss_and_grad(p, mo.encode(q, LO, HI), t)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    assert np.linalg.norm(g - ref_g) / np.linalg.norm(ref_g) < 1e-3
    for lo_, hi_ in zip(mo.OFFS[:-1], mo.OFFS[1:]):  # every layer
        assert np.linalg.norm(g[lo_:hi_] - ref_g[lo_:hi_]) <= 2e-3 * np.linalg.norm(ref_g[lo_:hi_]) + 1e-9
    assert np.array_equal(rc.params(), p)  # no update requested
    rc.close()


def test_adam_step_matches_oracle():
    rc = RadianceCache(LO, HI, seed=3)
    p = rand_params(9)
    rc.set_params(p)
    q = rand_queries(2048, 10)
    t = np.random.default_rng(11).uniform(0.0, 3.0, (2048, 3)).astype(np.float32)
    _, g = rc.train(q, t, update=False, want_grad=True)
    rc.train(q, t, lr=1e-3, update=True)
    w_ref, _, _ = mo.adam(p.astype(np.float64), 0.0, 0.0, g.astype(np.float64), 1, 1e-3)
    np.testing.assert_allclose(rc.params(), w_ref, rtol=0, atol=2e-6)
    rc.close()


def test_training_fits_a_smooth_radiance_field():
    def field(q):
        x = q[:, 0:3] / 10.0
        base = 0.6 + 0.4 * np.sin(3.0 * x[:, 0:1]) * np.cos(2.0 * x[:, 1:2]) + 0.3 * x[:, 2:3]
        return (base * np.array([1.0, 0.8, 0.6]) * (0.5 + q[:, 8:11])).astype(np.float32)

    rc = RadianceCache(LO, HI, seed=12)
    held = rand_queries(4096, 999)
    before = np.mean(((rc.infer(held) - field(held)) / (field(held) + 0.1)) ** 2)
    losses = []
    for it in range(300):
        q = rand_queries(4096, 1000 + it)
        loss, _ = rc.train(q, field(q), lr=5e-3)
        losses.append(loss)
    after = np.mean(((rc.infer(held) - field(held)) / (field(held) + 0.1)) ** 2)
    assert np.mean(losses[-20:]) < 0.1 * np.mean(losses[:5])
    assert after < 0.05 * before
    rc.close()


def test_bounded_wait_reports_timeout():
    """The tensor-core completion wait gives up after its iteration limit and
    reports it (the path that turns a stalled wait into AP_E_TIMEOUT), without
    faulting or hanging the GPU: a barrier that nothing arrives on times out,
    one that has completed does not."""
    import numpy as np
    from appearance_b200 import _native
    lib = _native.load()
    out = np.full(2, 7, np.uint32)
    assert lib.ap_rc_wait_selftest(0, 1024, out.ctypes.data_as(ctypes.c_void_p)) == _native.AP_OK
    assert out.tolist() == [0, 1]
    assert lib.ap_rc_wait_selftest(0, 0, out.ctypes.data_as(ctypes.c_void_p)) == _native.AP_E_INVALID
