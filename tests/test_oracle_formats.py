"""The oracle's packing formats and RNG against independent statements of their
published definitions: shared-exponent RGB9E5 (EXT_texture_shared_exponent:
value = mantissa * 2^(exponent - 24)), the 2x15-bit octahedral direction code,
and the PCG hash / xorshift / hash_combine streams of random.wgsl."""
import numpy as np

from oracle import oracle

M = 0xFFFFFFFF


def pcg_hash_py(x):
    state = (x * 747796405 + 2891336453) & M
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M
    return (word >> 22) ^ word


def xor_shift_py(s):
    s = (s ^ (s << 13)) & M
    s ^= s >> 17
    s = (s ^ (s << 5)) & M
    return s


def hash_combine_py(x, y):
    seed = (((x * 1664525) + y + 1013904223) * 1664525) & M
    seed ^= seed >> 11
    seed ^= (seed << 7) & 0x9D2C5680
    seed ^= (seed << 15) & 0xEFC60000
    seed ^= seed >> 18
    return seed & M


def test_rng_streams():
    L = oracle.lib()
    rng = np.random.default_rng(1)
    for x in list(range(16)) + list(rng.integers(0, 2 ** 32, 2000)):
        x = int(x)
        assert L.orc_pcg_hash(x) == pcg_hash_py(x)
        assert L.orc_xor_shift(x) == xor_shift_py(x)
        assert L.orc_hash_combine(x, x ^ 0x5bd1e995) == hash_combine_py(x, x ^ 0x5bd1e995)


def decode_rgb9e5(d):
    e = (d >> 27) & 31
    return np.array([(d >> s) & 0x1FF for s in (0, 9, 18)], np.float64) * 2.0 ** (e - 24)


def test_rgb9e5_decode_matches_format():
    rng = np.random.default_rng(2)
    for d in list(rng.integers(0, 2 ** 32, 5000)) + [0, 0xFFFFFFFF, 0x80000000]:
        assert np.array_equal(oracle.rgb9e5_unpack(int(d)).astype(np.float64), decode_rgb9e5(int(d)))


def test_rgb9e5_encode_error_bound_and_edges():
    rng = np.random.default_rng(3)
    v = np.exp(rng.uniform(np.log(1e-6), np.log(6e4), (20000, 3))).astype(np.float32)
    for x in v:
        d = oracle.rgb9e5_pack(x)
        y = decode_rgb9e5(d)
        e = (d >> 27) & 31
        step = 2.0 ** (e - 24)
        # every channel is the nearest multiple of the shared step (half a step at most)
        assert np.all(np.abs(y - x.astype(np.float64)) <= 0.5 * step + 1e-30)
    assert oracle.rgb9e5_pack([0, 0, 0]) & 0x07FFFFFF == 0
    assert np.array_equal(oracle.rgb9e5_unpack(oracle.rgb9e5_pack([np.nan, 1.0, np.nan])), [0.0, 1.0, 0.0])
    mx = np.float32(np.frombuffer(np.uint32(0x477F8000).tobytes(), np.float32)[0])  # 65408
    assert np.array_equal(oracle.rgb9e5_unpack(oracle.rgb9e5_pack([1e9, 1e9, -5.0])), [mx, mx, 0.0])
    # exactly representable values round-trip
    for m, e in [(1, 0), (511, 31), (256, 10), (3, 24)]:
        x = np.float32(m * 2.0 ** (e - 24))
        assert oracle.rgb9e5_unpack(oracle.rgb9e5_pack([x, 0, 0]))[0] == x


def test_oct30_roundtrip_accuracy():
    rng = np.random.default_rng(4)
    d = rng.normal(size=(20000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    worst = 0.0
    for v in d.astype(np.float32):
        u = oracle.oct30_unpack(oracle.oct30_pack(v))
        assert abs(np.linalg.norm(u) - 1.0) < 1e-6
        worst = max(worst, float(np.linalg.norm(u.astype(np.float64) - v.astype(np.float64))))
    assert worst < 2e-4  # 15-bit octahedral grid: spacing 2/32767, stretched up to ~2x near the diagonals
    for axis in np.eye(3).tolist() + (-np.eye(3)).tolist():
        # the 15-bit code has no exact centre (0.5 * 32767 is not an integer): ~3e-5
        assert np.allclose(oracle.oct30_unpack(oracle.oct30_pack(axis)), axis, atol=1e-4)
    # zero vector (an unset clearcoat basis in the reference) encodes to 0 -> (0,0,-1)
    assert oracle.oct30_pack([0.0, 0.0, 0.0]) == 0
    assert np.allclose(oracle.oct30_unpack(0), [0, 0, -1])
