"""Oracle (test infrastructure only): numpy restatement of the radiance-cache
MLP of appearance_b200/csrc/mlp.cu -- input encoding (float32 arithmetic in
the device's order, elementary functions from the oracle's detmath, so the
features match bit for bit), forward pass with FP16-rounded weights and
activations, relative L2 loss, its gradients, and the Adam update -- in
float64 unless stated."""
from __future__ import annotations

import numpy as np

from .oracle import detmath

IN, HID, OUT = 144, 64, 3
SIZES = [(HID, IN), (HID, HID), (HID, HID), (HID, HID), (OUT, HID)]
OFFS = np.cumsum([0] + [a * b for a, b in SIZES])
NUM_PARAMS = int(OFFS[-1])
f32 = np.float32


def split(params):
    return [np.asarray(params[OFFS[i]:OFFS[i + 1]], np.float64).reshape(SIZES[i]) for i in range(5)]


def h16(x):
    return np.asarray(x, np.float64).astype(np.float16).astype(np.float64)


def encode(q, lo, hi):
    """(n, 16) float32 queries -> (n, 144) float32 features."""
    q = np.asarray(q, f32)
    n = q.shape[0]
    lo = np.asarray(lo, f32)
    ext = np.asarray(hi, f32) - lo
    inv = np.where(ext > 0, f32(1.0) / np.where(ext > 0, ext, f32(1.0)), f32(0.0)).astype(f32)
    f = np.zeros((n, IN), f32)
    pi = f32(3.14159265358979323846)
    for a in range(3):
        x = ((q[:, a] - lo[a]) * inv[a]).astype(f32)
        ang = (x * pi).astype(f32)
        s, c = detmath("sin", ang), detmath("cos", ang)
        for o in range(12):  # double-angle recurrence, float32 in the device's order
            f[:, a * 24 + 2 * o] = s
            f[:, a * 24 + 2 * o + 1] = c
            s, c = ((f32(2.0) * s) * c).astype(f32), (f32(1.0) - (f32(2.0) * s) * s).astype(f32)
    z = np.clip(q[:, 6], f32(-1.0), f32(1.0)).astype(f32)
    th = (detmath("acos", z) * f32(1.0 / np.float32(pi))).astype(f32)
    ph = (detmath("atan2", q[:, 5], q[:, 4]) * f32(f32(0.5) / pi) + f32(0.5)).astype(f32)
    # the device evaluates the 13 bins around each peak; the rest are far below
    # the FP16 subnormal range and round to 0 with the features
    for j, v in enumerate((th, ph)):
        b0 = np.clip(np.floor(v * f32(32.0)).astype(np.int64), 0, 31)
        for i in range(32):
            c = f32((f32(i) + f32(0.5)) * f32(1.0 / 32.0))
            ci = ((v - c) * f32(32.0)).astype(f32)
            val = detmath("exp", ((f32(-0.5) * ci) * ci).astype(f32))
            f[:, 72 + 32 * j + i] = np.where(np.abs(i - b0) <= 6, val, f32(0.0))
    f[:, 136] = q[:, 3]
    f[:, 137:140] = q[:, 8:11]
    f[:, 140:143] = q[:, 11:14]
    return f


def forward(params, feats, fp16=True):
    """Hidden activations h0..h4 (FP16-rounded unless fp16=False) and the
    pre-exp outputs y."""
    r = h16 if fp16 else (lambda x: np.asarray(x, np.float64))
    W = [r(w) for w in split(params)]
    h = [r(feats)]
    for l in range(4):
        h.append(r(np.maximum(h[-1] @ W[l].T, 0.0)))
    return h, h[-1] @ W[4].T


def predict(params, feats):
    return np.exp(forward(params, feats)[1])


def loss_and_grad(params, feats, targets, fp16=True):
    """Relative L2 loss mean((exp(y) - t)^2 / (exp(y)^2 + 0.01)) (denominator held
    constant) and its gradient with respect to the (FP16-rounded) weights."""
    W = [(h16(w) if fp16 else w) for w in split(params)]
    h, y = forward(params, feats, fp16)
    t = np.asarray(targets, np.float64)
    n = y.shape[0]
    p = np.exp(y)
    den = p * p + 0.01
    loss = np.sum((p - t) ** 2 / den) / (3 * n)
    d = [None] * 5
    d[4] = 2.0 * (p - t) / den * p / (3 * n)
    for l in range(3, -1, -1):
        d[l] = (d[l + 1] @ W[l + 1]) * (h[l + 1] > 0)
    grads = [d[l].T @ h[l] for l in range(5)]
    return loss, np.concatenate([g.reshape(-1) for g in grads])


def adam(master, m1, m2, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * grad
    m2 = b2 * m2 + (1 - b2) * grad * grad
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return master - lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps), m1, m2
