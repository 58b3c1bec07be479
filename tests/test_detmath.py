"""Accuracy of the deterministic elementary functions (detmath.h) that both the
CUDA kernels and the oracle use, against float64 references."""
import numpy as np
import pytest

from oracle import oracle


def ulp_err(got, ref):
    got = got.astype(np.float64)
    ref32 = ref.astype(np.float32)
    ulp = np.spacing(np.abs(ref32)).astype(np.float64)
    return np.abs(got - ref) / np.maximum(ulp, np.spacing(np.float32(1e-30)))


@pytest.mark.parametrize("fn,lo,hi,tol", [("sin", -20, 20, 4), ("cos", -20, 20, 4), ("exp", -80, 80, 4),
                                          ("acos", -1, 1, 4)])
def test_unary_ulp(fn, lo, hi, tol):
    x = np.linspace(lo, hi, 200001).astype(np.float32)
    got = oracle.detmath(fn, x)
    ref = getattr(np, {"acos": "arccos"}.get(fn, fn))(x.astype(np.float64))
    err = ulp_err(got, ref)
    if fn in ("sin", "cos"):  # near the zeros compare absolutely (absolute error <= 2^-23)
        small = np.abs(ref) < 1e-3
        assert np.abs(got[small] - ref[small]).max() < 2.0 ** -23
        err = err[~small]
    assert err.max() <= tol, (fn, err.max())


def test_log_ulp():
    x = np.exp(np.linspace(np.log(1e-37), np.log(1e37), 200001)).astype(np.float32)
    err = ulp_err(oracle.detmath("log", x), np.log(x.astype(np.float64)))
    assert err.max() <= 4


def test_atan2_ulp():
    t = np.linspace(-np.pi, np.pi, 100001)
    y, x = np.sin(t).astype(np.float32), np.cos(t).astype(np.float32)
    err = ulp_err(oracle.detmath("atan2", y, x), np.arctan2(y.astype(np.float64), x.astype(np.float64)))
    assert err.max() <= 4


def test_pow_relative():
    rng = np.random.default_rng(0)
    x = rng.uniform(1e-3, 1.0, 100000).astype(np.float32)
    y = rng.choice([0.5, 2.0, 5.0, 128.0], 100000).astype(np.float32)
    ref = np.power(x.astype(np.float64), y.astype(np.float64))
    got = oracle.detmath("pow", x, y).astype(np.float64)
    keep = ref > 1e-30
    rel = np.abs(got[keep] - ref[keep]) / ref[keep]
    assert rel.max() < 3e-5


def test_special_values():
    nan = np.float32(np.nan)
    assert np.isnan(oracle.detmath("log", np.array([-1.0]))[0])
    assert oracle.detmath("log", np.array([0.0]))[0] == -np.inf
    assert oracle.detmath("exp", np.array([-200.0]))[0] == 0.0
    assert oracle.detmath("exp", np.array([200.0]))[0] == np.inf
    assert oracle.detmath("pow", np.array([0.0]), np.array([0.5]))[0] == 0.0
    assert oracle.detmath("pow", np.array([0.3]), np.array([0.0]))[0] == 1.0
    assert np.isnan(oracle.detmath("sin", np.array([nan]))[0])
