"""The bit-level arithmetic the mixed pair passes rely on, restated in numpy
and checked on the host (moldy_b200/csrc/common.cuh: fix32, floor_small;
moldy_b200/csrc/pairs.cu: the wrap test of the virial corrections):

* fix32(x) = round-to-nearest-even(x * 2^32) mod 2^32 through one fused
  multiply-add against the bias 1.5 * 2^52;
* floor_small(x): one round-down addition of 2^23 gives floor(x) for
  0 <= x < 2^23;
* the 32-bit difference of two fixed-point coordinates is the minimum image;
* ((qa ^ qj) & (qa ^ e)) < 0, e the wrapped 32-bit difference qa - qj, flags
  exactly the differences that wrapped, the image being m = +1 for qa >= 0 and
  -1 otherwise (qa - qj = e + m 2^32), and no pair within M of an atom wraps
  when |qa| <= 2^31 - 1 - M."""
import numpy as np

RNG = np.random.default_rng(7)


def bits_f32(u):
    return np.asarray(u, dtype=np.uint32).view(np.float32)


def fix32(x):
    y = np.asarray(x, dtype=np.float64) * 4294967296.0 + 6755399441055744.0   # exact product, one rounding
    return (y.view(np.uint64) & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)


def test_wrap_flag_and_image():
    qa = RNG.integers(-2**31, 2**31, size=2_000_000, dtype=np.int64)
    qj = RNG.integers(-2**31, 2**31, size=2_000_000, dtype=np.int64)
    exact = qa - qj
    e = ((exact + 2**31) % 2**32 - 2**31)                     # the 32-bit difference
    a32, j32, e32 = (v.astype(np.int32) for v in (qa, qj, e))
    flag = ((a32 ^ j32) & (a32 ^ e32)) < 0
    assert np.array_equal(flag, exact != e)
    m = np.where(qa >= 0, 1, -1)
    assert np.array_equal((exact - e)[flag], (m * 2**32)[flag])


def test_no_wrap_away_from_the_faces():
    M = 56_000_000                                            # a pair's span, fixed-point units
    lim = 2**31 - 1 - M
    qa = RNG.integers(-lim, lim + 1, size=1_000_000, dtype=np.int64)
    d = RNG.integers(-M, M + 1, size=1_000_000, dtype=np.int64)
    qj = qa - d                                               # the partner's true image
    assert np.all((qj >= -2**31) & (qj < 2**31))              # stored without wrapping: qa - qj = d


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
