"""The library's ZSobol sampler (spectral.h, the code the CUDA spectral
kernels run) against the oracle's own restatement of ZSobolSampler
(zsobol_sampler.rs:43-152): the same draws, bit for bit, for pixels, frame
seeds and draw sequences of the path integrator.  spectral.h compiles as plain
C++ on the host, so this runs without a GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = r'''
#include <stdint.h>
#include "spectral.h"
extern "C" void lib_zsobol(uint32_t W, uint32_t H, uint64_t seed, uint32_t x, uint32_t y, const uint8_t* kinds,
                           uint32_t n, float* out) {
  uint32_t px, py;
  spec::sampler_pixel(x, y, W, H, &px, &py);
  spec::ZSobol z{spec::morton2(px, py), spec::zsobol_digits(W, H), seed, 0u};
  uint32_t o = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (kinds[i] == 1) {
      out[o++] = z.get1d();
    } else {
      z.get2d(&out[o], &out[o + 1]);
      o += 2;
    }
  }
}
extern "C" void lib_pixel(uint32_t W, uint32_t H, uint32_t x, uint32_t y, uint32_t* p) {
  spec::sampler_pixel(x, y, W, H, &p[0], &p[1]);
}
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("zsobol")
    src, so = d / "shim.cpp", d / "shim.so"
    src.write_text(SHIM)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                    "-I", os.path.join(ROOT, "appearance_b200", "csrc"), str(src), "-o", str(so)], check=True)
    L = ctypes.CDLL(str(so))
    L.lib_zsobol.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                             ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
    L.lib_pixel.argtypes = [ctypes.c_uint32] * 4 + [ctypes.c_void_p]
    return L


def _lib_draws(L, W, H, seed, x, y, kinds):
    k = np.asarray(kinds, np.uint8)
    out = np.zeros(int(k.astype(np.int64).sum()), np.float32)
    L.lib_zsobol(W, H, seed, x, y, k.ctypes.data, len(k), out.ctypes.data)
    return out


@pytest.mark.parametrize("W,H", [(64, 48), (96, 96), (4096, 4096), (1920, 1080), (17, 9)])
def test_library_sampler_equals_the_oracle_sampler(lib, W, H):
    # wavelength; per vertex: light sample (2d), light pick, BSDF (1d, 2d), roulette
    kinds = [1] + [2, 1, 1, 2, 1] * 6
    rng = np.random.default_rng(W * 31 + H)
    for _ in range(12):
        x, y = int(rng.integers(0, W)), int(rng.integers(0, H))
        seed = int(rng.integers(0, 1 << 40))
        p = np.zeros(2, np.uint32)
        lib.lib_pixel(W, H, x, y, p.ctypes.data)
        got = _lib_draws(lib, W, H, seed, x, y, kinds)
        ref = oracle.zsobol((W, H), 1, seed, (int(p[0]), int(p[1])), 0, kinds)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (x, y, seed)


def test_sampler_pixel_flips_rows(lib):
    p = np.zeros(2, np.uint32)
    lib.lib_pixel(64, 48, 5, 0, p.ctypes.data)
    assert tuple(p) == (5, 47)
    lib.lib_pixel(64, 48, 63, 47, p.ctypes.data)
    assert tuple(p) == (63, 0)
