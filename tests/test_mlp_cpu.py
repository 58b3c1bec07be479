"""The radiance-cache oracle itself (CPU): its analytic gradients against
finite differences of its loss, the encoding's value ranges, and the Adam rule."""
import numpy as np

from oracle import mlp_oracle as mo


def rand_queries(n, rng):
    q = np.zeros((n, 16), np.float32)
    q[:, 0:3] = rng.uniform(-1.0, 11.0, (n, 3))
    q[:, 3] = rng.uniform(0.05, 1.0, n)
    d = rng.normal(size=(n, 3))
    q[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 8:14] = rng.uniform(0.0, 1.0, (n, 6))
    return q


def test_encoding_ranges():
    rng = np.random.default_rng(0)
    f = mo.encode(rand_queries(500, rng), [-1, -1, -1], [11, 11, 11])
    assert f.shape == (500, 144) and f.dtype == np.float32
    # octaves by the double-angle recurrence: within 1e-2 of sin/cos(2^o pi x)
    qq = rand_queries(500, np.random.default_rng(0))
    x = (qq[:, 0:3].astype(np.float64) + 1.0) / 12.0
    for a in range(3):
        for o in range(12):
            assert np.abs(f[:, a * 24 + 2 * o] - np.sin(2 ** o * np.pi * x[:, a])).max() < 1e-2
            assert np.abs(f[:, a * 24 + 2 * o + 1] - np.cos(2 ** o * np.pi * x[:, a])).max() < 1e-2
    assert np.all((f[:, 72:136] >= 0.0) & (f[:, 72:136] <= 1.0))
    # each one-blob peaks at the bin nearest the angle
    assert np.all(f[:, 72:104].max(1) > 0.88) and np.all(f[:, 104:136].max(1) > 0.88)
    assert np.all(f[:, 143] == 0.0)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    feats = mo.encode(rand_queries(64, rng), [-1, -1, -1], [11, 11, 11]).astype(np.float64)
    params = rng.normal(size=mo.NUM_PARAMS) * 0.15
    targets = rng.uniform(0.0, 2.0, (64, 3))
    _, g = mo.loss_and_grad(params, feats, targets, fp16=False)
    for idx in list(rng.choice(mo.NUM_PARAMS, 40, replace=False)) + [mo.OFFS[4] + 5, mo.OFFS[0] + 7]:
        e = 1e-6
        pp, pm = params.copy(), params.copy()
        pp[idx] += e
        pm[idx] -= e
        # the loss's denominator is held constant: differentiate the numerator form
        def num_loss(p):
            h, y = mo.forward(p, feats, fp16=False)
            _, y0 = mo.forward(params, feats, fp16=False)
            den = np.exp(y0) ** 2 + 0.01
            return np.sum((np.exp(y) - targets) ** 2 / den) / (3 * feats.shape[0])
        fd = (num_loss(pp) - num_loss(pm)) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])


def test_adam_first_step_moves_by_lr():
    master = np.ones(5)
    grad = np.array([1.0, -2.0, 0.5, 1e-3, -1e-3])
    w, m1, m2 = mo.adam(master, np.zeros(5), np.zeros(5), grad, 1, 1e-3)
    assert np.allclose(master - w, 1e-3 * np.sign(grad), rtol=1e-4)
