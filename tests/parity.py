"""Comparison rules of the GPU parity tests.

Bit-exact (every 32-bit word equal): traversal results (triangle id, t,
barycentrics), packed formats, and every per-pixel state buffer of the path
tracing stages (rays, payload, G-buffer, DI/GI reservoirs, light-sample
context), and frames that skip the SVGF a-trous passes and TAA.  The CUDA path
evaluates those stages with the oracle's arithmetic (no contraction, IEEE
division and square root, the same elementary functions, the same order).

Within a stated tolerance: frames (and the remodulated radiance buffer) that
went through the SVGF a-trous passes or TAA.  There the CUDA kernels use the
hardware exponential, reciprocals and fused multiply-adds, while the oracle
keeps the reference's literal expressions (svgf_atrous.wgsl:90-99,
taa.wgsl:67-171).  The weights then differ in their last bits; every pass
re-packs its output to RGB9E5 (9-bit mantissas with a shared exponent), which
hides most of that, and flips a rounding step elsewhere.  The tolerance,
per pixel p with channels c, relative to the pixel's brightest channel:

    e_p = max_c |gpu - oracle| / max(max_c |oracle|, 1e-4)

  * every pixel:            e_p <= POST_MAX_REL
  * mean over the pixels:   mean(e_p) <= POST_MEAN_REL
  * bit-identical pixels:   at least POST_MIN_EXACT of them
"""
import numpy as np

POST_MAX_REL = 2.0 ** -4      # a few RGB9E5 rounding steps, compounded over passes and frames
POST_MEAN_REL = 1e-3
POST_MIN_EXACT = 0.90


def uses_post_tolerance(cfg) -> bool:
    """Frames of this configuration pass the fast-math denoise kernels."""
    return bool(cfg.get("taa")) or (bool(cfg.get("svgf")) and cfg.get("svgf_atrous_passes", 5) > 0)


def assert_bits(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    same = a.view(np.uint32) == b.view(np.uint32)
    assert same.all(), f"{what}: {(~same).sum()} of {same.size} words differ"


def post_stats(gpu, ref):
    g = np.asarray(gpu, np.float64).reshape(-1, 3)
    o = np.asarray(ref, np.float64).reshape(-1, 3)
    err = np.abs(g - o).max(1) / np.maximum(np.abs(o).max(1), 1e-4)
    exact = (np.asarray(gpu, np.float32).reshape(-1, 3).view(np.uint32) ==
             np.asarray(ref, np.float32).reshape(-1, 3).view(np.uint32)).all(1)
    return float(err.max()), float(err.mean()), float(exact.mean())


def assert_post_close(gpu, ref, what):
    g, o = np.asarray(gpu, np.float32), np.asarray(ref, np.float32)
    assert g.shape == o.shape, what
    assert np.isfinite(g).all(), f"{what}: non-finite values"
    mx, mean, exact = post_stats(g, o)
    print(f"{what}: max rel {mx:.3g}, mean rel {mean:.3g}, bit-identical pixels {exact:.4f}")
    assert mx <= POST_MAX_REL, f"{what}: max relative error {mx:.3g} > {POST_MAX_REL}"
    assert mean <= POST_MEAN_REL, f"{what}: mean relative error {mean:.3g} > {POST_MEAN_REL}"
    assert exact >= POST_MIN_EXACT, f"{what}: only {exact:.4f} of the pixels bit-identical"


def assert_frame(gpu, ref, cfg, what):
    if uses_post_tolerance(cfg):
        assert_post_close(gpu, ref, what)
    else:
        assert_bits(gpu, ref, what)


# The spectral mode: the GPU runs the library's restatement of the reference's
# spectral integrator (spectral.h), the oracle its own (oracle_spectral.cpp),
# from the same ZSobol draws and bit-identical closest hits, but each with its
# platform's elementary functions (CUDA's and the C library's expf, logf,
# atan2f, acosf, sincosf, hypotf, within an ulp or two of each other).  A
# difference in the last bit moves a pixel by as much, unless it flips one of
# the path's decisions (Russian roulette, the dielectric's reflect-or-refract
# choice), after which that path differs entirely.  So: most pixels agree to
# SPECTRAL_PIXEL_REL (relative to the pixel's brightest channel, floor
# SPECTRAL_FLOOR x the image mean), at least SPECTRAL_MIN_CLOSE of them, and
# the per-channel image means agree to SPECTRAL_MEAN_REL.
SPECTRAL_PIXEL_REL = 1e-4
SPECTRAL_FLOOR = 1e-3
SPECTRAL_MIN_CLOSE = 0.97
SPECTRAL_MEAN_REL = 0.03


def spectral_stats(gpu, ref):
    g = np.asarray(gpu, np.float64).reshape(-1, 3)
    o = np.asarray(ref, np.float64).reshape(-1, 3)
    floor = SPECTRAL_FLOOR * max(float(np.abs(o).mean()), 1e-12)
    err = np.abs(g - o).max(1) / np.maximum(np.abs(o).max(1), floor)
    mean_rel = float(np.max(np.abs(g.mean(0) - o.mean(0)) / np.maximum(np.abs(o.mean(0)), 1e-12)))
    return float((err <= SPECTRAL_PIXEL_REL).mean()), mean_rel, float(np.median(err))


def assert_spectral_close(gpu, ref, what):
    g, o = np.asarray(gpu, np.float32), np.asarray(ref, np.float32)
    assert g.shape == o.shape, what
    assert np.isfinite(g).all(), f"{what}: non-finite values"
    close, mean_rel, med = spectral_stats(g, o)
    print(f"{what}: pixels within {SPECTRAL_PIXEL_REL:g}: {close:.4f}, image-mean difference {mean_rel:.3g}, "
          f"median pixel error {med:.3g}")
    assert close >= SPECTRAL_MIN_CLOSE, f"{what}: only {close:.4f} of the pixels within {SPECTRAL_PIXEL_REL}"
    assert mean_rel <= SPECTRAL_MEAN_REL, f"{what}: image means differ by {mean_rel:.3g}"


def rgb9e5_to_rgb(words):
    """RGB9E5 words (packing.wgsl:12-44) as float RGB, for tolerance checks."""
    w = np.asarray(words, np.uint32).reshape(-1)
    e = (w >> 27).astype(np.int32) - 15 - 9
    scale = np.ldexp(1.0, e)
    return np.stack([(w & 511) * scale, ((w >> 9) & 511) * scale, ((w >> 18) & 511) * scale], 1).astype(np.float32)
