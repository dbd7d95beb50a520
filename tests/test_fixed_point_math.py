"""The bit-level arithmetic the mixed pair passes rely on, restated in numpy
and checked on the host (moldy_b200/csrc/common.cuh: fix32, fix_to_float,
floor_small):

* fix32(x) = round-to-nearest-even(x * 2^32) mod 2^32 through one fused
  multiply-add against the bias 1.5 * 2^52;
* fix_to_float(d): the upper 20 and lower 12 bits of an int32 made exact
  floats by power-of-two biases and joined by one fused multiply-add equal
  float(d) rounded once to nearest;
* floor_small(x): one round-down addition of 2^23 gives floor(x) for
  0 <= x < 2^23;
* the 32-bit difference of two fixed-point coordinates is the minimum image."""
import numpy as np

RNG = np.random.default_rng(7)


def bits_f32(u):
    return np.asarray(u, dtype=np.uint32).view(np.float32)


def fix_to_float(d):
    d = np.asarray(d, dtype=np.int32)
    hi = (d >> 12).astype(np.int64)
    lo = (d & 0xFFF).astype(np.int64)
    fhi = bits_f32((0x4B400000 + hi).astype(np.uint32)).astype(np.float64) - 12582912.0
    flo = bits_f32((0x4B000000 + lo).astype(np.uint32)).astype(np.float64) - 8388608.0
    # fhi*4096 + flo is exact in float64; the fused multiply-add rounds it once to float32
    return (fhi * 4096.0 + flo).astype(np.float32)


def fix32(x):
    y = np.asarray(x, dtype=np.float64) * 4294967296.0 + 6755399441055744.0   # exact product, one rounding
    return (y.view(np.uint64) & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)


def test_fix_to_float_is_one_rounding():
    d = np.concatenate([RNG.integers(-2**31, 2**31, size=2_000_000, dtype=np.int64),
                        [-2**31, 2**31 - 1, 0, 1, -1, 4095, 4096, -4096, 2**24 + 1, -(2**24 + 1)]]).astype(np.int32)
    assert np.array_equal(fix_to_float(d), d.astype(np.float32))


def test_fix32_rounds_to_nearest_mod_2_32():
    x = np.concatenate([RNG.uniform(-5.0, 5.0, size=1_000_000), [0.0, 0.5, -0.5, 1.0 - 2**-40, 2**-33, -2**-33]])
    want = (np.rint(x * 2.0**32).astype(np.int64) % 2**32).astype(np.uint32).view(np.int32)
    assert np.array_equal(fix32(x), want)


def test_fixed_point_difference_is_minimum_image():
    xa = RNG.uniform(-3.0, 3.0, size=200_000)
    dx = RNG.uniform(-0.45, 0.45, size=200_000)
    xb = xa - dx + RNG.integers(-2, 3, size=200_000)        # the partner, some box lengths away
    d = (fix32(xa).astype(np.int64) - fix32(xb).astype(np.int64)).astype(np.int64)
    d = ((d + 2**31) % 2**32 - 2**31).astype(np.int32)        # 32-bit wrap-around
    ref = (xa - xb) - np.round(xa - xb)
    assert np.max(np.abs(d.astype(np.float64) * 2.0**-32 - ref)) <= 2.0**-32 + 1e-15


def test_floor_small():
    x = np.concatenate([RNG.uniform(0.0, 8.0e6, size=1_000_000).astype(np.float32),
                        np.array([0.0, 0.999999, 1.0, 4095.9995, 8388606.5], dtype=np.float32)])
    # round-down addition of 2^23 in float32: exact floor for x < 2^23
    b = np.floor(x.astype(np.float64) + 8388608.0).astype(np.float32)   # the sum is exact in float64
    idx = b.view(np.uint32).astype(np.int64) - 0x4B000000
    assert np.array_equal(idx, np.floor(x.astype(np.float64)).astype(np.int64))
