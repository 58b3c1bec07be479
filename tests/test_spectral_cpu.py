"""Spectral-mode building blocks on the CPU (the oracle's restatement of the
reference's CPU tracer, oracle_spectral.cpp): matching functions, wavelength
sampling, RGB upsampling, the ZSobol sampler and its hash, and the CPU render's
basic properties."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

SRGB_FROM_XYZ = np.array([[3.2404542, -1.5371385, -0.4985314],
                          [-0.9692660, 1.8760108, 0.0415560],
                          [0.0556434, -0.2040259, 1.0572252]])


def test_cie_y_normaliser_is_the_integral_of_y():
    lam = np.arange(360.0, 830.0 + 1e-9, 0.5)
    y = np.array([oracle.spectral_cmf(float(l))[1] for l in lam], np.float64)
    integral = float(np.sum(0.5 * (y[1:] + y[:-1]) * 0.5))
    assert integral == pytest.approx(106.922074, rel=2e-6)


@pytest.mark.parametrize("lam,k,val", [(555.0, 1, 1.0), (600.0, 0, 1.0622), (450.0, 2, 1.7721), (530.0, 1, 0.862)])
def test_matching_functions_near_the_cie_1931_values(lam, k, val):
    # the multi-lobe fit of Wyman, Sloan and Shirley is within a few percent of
    # the tabulated CIE 1931 2-degree observer near the lobe peaks
    assert oracle.spectral_cmf(lam)[k] == pytest.approx(val, rel=0.05)


def test_illuminant_is_planck_at_6504k_normalised_at_560nm():
    c2 = 1.4387769e7
    for lam in (400.0, 500.0, 560.0, 700.0):
        ref = (560.0 / lam) ** 5 * (math.exp(c2 / (560.0 * 6504.0)) - 1.0) / (math.exp(c2 / (lam * 6504.0)) - 1.0)
        assert oracle.spectral_cmf(lam)[3] == pytest.approx(ref, rel=1e-5)


def test_visible_wavelength_sampling_inverts_its_cdf():
    lam = np.linspace(360.0, 830.0, 94001)
    pdf = np.array([0.0039398042 / math.cosh(0.0072 * (l - 538.0)) ** 2 for l in lam])
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (pdf[1:] + pdf[:-1]) * (lam[1] - lam[0]))])
    assert cdf[-1] == pytest.approx(1.0, abs=2e-4)
    for u in (0.0, 0.1, 0.37, 0.5, 0.81, 0.999):
        l, p = oracle.spectral_wavelength(u)
        assert 360.0 - 1e-3 <= l <= 830.0 + 1e-3
        assert np.interp(l, lam, cdf) == pytest.approx(u, abs=2e-3)
        assert p == pytest.approx(np.interp(l, lam, pdf), rel=1e-4)


def _rgb_of(coef):
    """Linear sRGB of a sigmoid reflectance under the 6504 K illuminant (5 nm midpoint rule)."""
    xyz = np.zeros(3)
    norm = 0.0
    for i in range(94):
        lam = 362.5 + 5.0 * i
        x, y, z, e = (float(v) for v in oracle.spectral_cmf(lam))
        s = oracle.spectral_sigmoid(coef, lam)
        xyz += s * e * np.array([x, y, z])
        norm += e * y
    return SRGB_FROM_XYZ @ (xyz / norm)


def test_albedo_fit_reproduces_colours():
    rng = np.random.default_rng(3)
    cols = list(rng.uniform(0.05, 0.95, size=(12, 3))) + [np.array([0.63, 0.065, 0.05]),
                                                           np.array([0.14, 0.45, 0.091]),
                                                           np.array([0.725, 0.71, 0.68])]
    for rgb in cols:
        c = oracle.spectral_fit(rgb)
        assert np.all(np.isfinite(c))
        back = _rgb_of(c)
        assert np.max(np.abs(back - rgb)) < 0.02, (rgb, back)


def test_fitted_reflectance_is_a_reflectance():
    for rgb in ([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [2.0, -1.0, 0.5]):
        c = oracle.spectral_fit(rgb)
        for lam in (360.0, 450.0, 550.0, 650.0, 830.0):
            s = oracle.spectral_sigmoid(c, lam)
            assert 0.0 <= s <= 1.0


def _small_scene():
    from appearance_b200 import scenes
    sc = scenes.icosphere_field(seed=2, num_spheres=24, num_emissive=4, subdiv=1, box=8.0, env_size=(64, 32))
    sc.materials[:6, 8] = 1.0  # a few dielectrics (transmission > 0, metallic 0)
    sc.materials[:6, 3] = 0.0
    return sc


def test_illuminant_normaliser_is_near_one():
    assert 0.9 < oracle.spectral_illuminant_norm() < 1.1


def test_murmur3_x64_128_matches_its_published_verification_value():
    """MurmurHash3 x64_128, which the ZSobol sampler hashes (dimension, seed)
    with (the murmurhash3 crate): SMHasher's verification test hashes the keys
    [0..i) with seed 256 - i for i = 0..255, hashes the concatenated results
    with seed 0 and reads the first four bytes little-endian."""
    hashes = b""
    for i in range(256):
        h1, h2 = oracle.murmur3_x64_128(bytes(range(i)), 256 - i)
        hashes += h1.to_bytes(8, "little") + h2.to_bytes(8, "little")
    h1, _ = oracle.murmur3_x64_128(hashes, 0)
    assert h1 & 0xFFFFFFFF == 0x6384BA69
    assert oracle.murmur3_x64_128(b"", 0) == (0, 0)


def _block_draws(x0, y0, n, seed, kinds, res=(64, 64)):
    return np.array([oracle.zsobol(res, 1, seed, (x0 + x, y0 + y), 0, kinds) for y in range(n) for x in range(n)])


@pytest.mark.parametrize("seed", [0, 7])
def test_zsobol_pixels_of_an_aligned_block_stratify_every_draw(seed):
    """At one sample per pixel the 4^k pixels of an aligned 2^k x 2^k block
    take 4^k consecutive (permuted) Sobol indices, so each draw over the block
    is a stratified set: every 1-D draw puts one value in each of 256 equal
    intervals, every 2-D draw one point in each cell of a 16 x 16 grid."""
    kinds = [1, 2, 1, 2, 1]  # wavelength, light sample, light pick, BSDF, roulette order
    d = _block_draws(16, 32, 16, seed, kinds)
    assert d.shape == (256, 7) and np.all((d >= 0.0) & (d <= 1.0))
    for col in (0, 3, 6):
        assert sorted(np.floor(d[:, col] * 256).astype(int).tolist()) == list(range(256))
    for cx, cy in ((1, 2), (4, 5)):
        cells = np.floor(d[:, cx] * 16).astype(int) * 16 + np.floor(d[:, cy] * 16).astype(int)
        assert sorted(cells.tolist()) == list(range(256))


def test_zsobol_streams_depend_on_pixel_seed_and_dimension():
    a = oracle.zsobol((64, 64), 1, 0, (3, 5), 0, [1, 1, 1, 1])
    assert len(set(a.tolist())) == 4                      # successive dimensions differ
    assert not np.array_equal(a, oracle.zsobol((64, 64), 1, 1, (3, 5), 0, [1, 1, 1, 1]))  # frame seed
    assert not np.array_equal(a, oracle.zsobol((64, 64), 1, 0, (4, 5), 0, [1, 1, 1, 1]))  # pixel
    np.testing.assert_array_equal(a, oracle.zsobol((64, 64), 1, 0, (3, 5), 0, [1, 1, 1, 1]))


def test_spectral_render_is_deterministic_and_threads_agree():
    from appearance_b200 import scenes
    sc = _small_scene()
    os_ = oracle.OracleScene(sc)
    spec = oracle.OracleSpectral(os_, sun_scale=5.0, scene_radius=50.0)
    w, h = 24, 16
    mats, _ = scenes.camera_matrices((4.0, 5.0, -12.0), (4.0, 3.0, 4.0), 60.0, 0.01, 1000.0, w, h, None)
    a = spec.render(mats, w, h, spp=2, max_depth=6, seed=7, threads=1)
    b = spec.render(mats, w, h, spp=2, max_depth=6, seed=7, threads=4)
    np.testing.assert_array_equal(a, b)
    assert np.all(np.isfinite(a)) and a.mean() > 0.0
    c = spec.render(mats, w, h, spp=2, max_depth=6, seed=7, row0=5, row1=11, threads=2)
    np.testing.assert_array_equal(c, a[5:11])
    d = spec.render(mats, w, h, spp=2, max_depth=6, seed=8, threads=4)
    assert not np.array_equal(a, d)
