"""Fit the polynomial coefficients used by detmath.h.

Every elementary function of the frame (sin, cos, exp, log, atan, asin) is
evaluated with plain IEEE-754 binary32 multiplies and adds in a fixed order, so
the CUDA kernels and the CPU oracle produce the same bits.  The coefficients are
least-squares fits of the relative error on Chebyshev nodes of the reduced
argument range (the classic Cody-Waite reduction + polynomial method, as in
W. J. Cody and W. Waite, "Software Manual for the Elementary Functions", 1980).

Run:  python gen_detmath.py   (prints the constant block pasted into detmath.h)
"""
import math

import numpy as np


def cheb_nodes(a, b, n=4000):
    k = np.arange(n)
    x = np.cos((2 * k + 1) * np.pi / (2 * n))
    return 0.5 * (a + b) + 0.5 * (b - a) * x


def fit(x, target, basis_cols, weight):
    A = np.stack(basis_cols, axis=1) * weight[:, None]
    c, *_ = np.linalg.lstsq(A, target * weight, rcond=None)
    return c


def series(x, coef_fn, nterms=40):
    """Sum_{n>=0} coef_fn(n) * x**n, evaluated in float64 (no cancellation)."""
    acc = np.zeros_like(x)
    for n in reversed(range(nterms)):
        acc = acc * x + coef_fn(n)
    return acc


def split_const(v, bits):
    """Split v into hi (few significant bits, so k*hi is exact) + mid + lo (float32)."""
    e = np.floor(np.log2(abs(v)))
    q = 2.0 ** (e - bits + 1)
    hi = np.round(v / q) * q
    r = v - hi
    e2 = np.floor(np.log2(abs(r)))
    q2 = 2.0 ** (e2 - bits + 1)
    mid = np.round(r / q2) * q2
    lo = np.float32(r - mid)
    return np.float32(hi), np.float32(mid), lo


def main():
    out = []
    # sin / cos on |r| <= pi/4:  sin r = r + r^3 (s1 + s2 r^2 + s3 r^4 + s4 r^6)
    r = cheb_nodes(1e-4, np.pi / 4)
    z = r * r
    s = fit(r, series(z, lambda n: (-1) ** (n + 1) / math.factorial(2 * n + 3)), [z**0, z, z**2, z**3], np.ones_like(r))
    # cos r = 1 - r^2/2 + r^4 (c1 + c2 r^2 + c3 r^4 + c4 r^6)
    c = fit(r, series(z, lambda n: (-1) ** n / math.factorial(2 * n + 4)), [z**0, z, z**2, z**3], np.ones_like(r))
    p1, p2, p3 = split_const(np.pi / 2, 11)
    out.append(("SIN_C", s)); out.append(("COS_C", c))
    out.append(("PIO2_PARTS", [p1, p2, p3]))
    # exp on |r| <= ln2/2: exp r = 1 + r + r^2 (e0 + e1 r + ... + e5 r^5)
    r = cheb_nodes(-np.log(2) / 2, np.log(2) / 2)
    e = fit(r, series(r, lambda n: 1.0 / math.factorial(n + 2)), [r**i for i in range(6)], np.exp(-r))
    l1, l2, _ = split_const(np.log(2), 11)
    l2 = np.float32(np.log(2) - np.float64(l1))
    out.append(("EXP_C", e)); out.append(("LN2_PARTS", [l1, l2]))
    # log via s=(m-1)/(m+1), |s| <= 0.1716: log m = 2s + s^3 (g0 + g1 s^2 + g2 s^4 + g3 s^6)
    sv = cheb_nodes(1e-4, 0.1716)
    zz = sv * sv
    g = fit(sv, series(zz, lambda n: 2.0 / (2 * n + 3)), [zz**i for i in range(4)], np.ones_like(sv))
    out.append(("LOG_C", g))
    # atan on |u| <= tan(pi/8): atan u = u + u^3 (a0 + a1 u^2 + ... + a5 u^10)
    u = cheb_nodes(1e-4, np.tan(np.pi / 8))
    zu = u * u
    a = fit(u, series(zu, lambda n: (-1) ** (n + 1) / (2 * n + 3)), [zu**i for i in range(6)], np.ones_like(u))
    out.append(("ATAN_C", a))
    # asin on |t| <= 0.5: asin t = t + t^3 (b0 + b1 t^2 + ... + b5 t^10)
    t = cheb_nodes(1e-4, 0.5)
    zt = t * t
    b = fit(t, series(zt, lambda n: math.comb(2 * n + 2, n + 1) / (4 ** (n + 1) * (2 * n + 3))), [zt**i for i in range(6)], np.ones_like(t))
    out.append(("ASIN_C", b))
    for name, vals in out:
        vals = [np.float32(v) for v in vals]
        body = ", ".join(f"{float(v):.9e}f" for v in vals)
        print(f"// {name}: {len(vals)} coefficients\n{name} = {{ {body} }};")


if __name__ == "__main__":
    main()
