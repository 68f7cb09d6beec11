"""Arithmetic facts the IRT kernels' f32 prefilters rely on (csrc/dmath.cuh,
csrc/irt.cu), checked on the CPU by emulating the f32 operations exactly.

* u01f32(a) = fmaf(__uint2float_rz(a), 2^-32, 2^-33): the f32 uniform the
  bounds use. Its upward error against (a + 1/2) / 2^32 must not exceed that
  of a correctly rounded f32 (half an ulp): an upward error shrinks
  -2 ln u and with it the Box-Muller radius bound.
* the draw-free displacement factor 11.8 exceeds the largest Box-Muller radius
  of 32-bit draws, sqrt(3 * 2 ln 2^33) = 11.72 (u01d32 >= 2^-33).
"""
import math

import numpy as np


def _uint2float_rz(a):
    """CUDA __uint2float_rz: a rounded toward zero to 24 significant bits."""
    a = np.asarray(a, dtype=np.uint64)
    bits = np.where(a > 0, np.floor(np.log2(np.maximum(a, 1).astype(np.float64))).astype(np.int64) + 1, 0)
    sh = np.maximum(bits - 24, 0).astype(np.uint64)
    return ((a >> sh) << sh).astype(np.float32)


def _u01f32(a):
    # the fma's exact sum trunc(a) * 2^-32 + 2^-33 fits an f64, so one f32 rounding of it is fmaf
    t = _uint2float_rz(a).astype(np.float64)
    return (t * 2.0 ** -32 + 2.0 ** -33).astype(np.float32)


def test_u01f32_upward_error_at_most_half_ulp():
    rng = np.random.default_rng(7)
    edge = [0, 1, 2, 3, (1 << 23) - 1, 1 << 23, (1 << 23) + 1, (1 << 24) - 1, 1 << 24, (1 << 24) + 1,
            (1 << 24) + 3, (1 << 31) - 1, 1 << 31, (1 << 32) - 129, (1 << 32) - 128, (1 << 32) - 1]
    for k in range(25, 33):                                  # just below and above every power of two
        edge += [(1 << k) - 1, (1 << k) - 2 ** (k - 24), (1 << k) - 2 ** (k - 25)]
    a = np.concatenate([np.array([x for x in edge if x < 2 ** 32], np.uint64),
                        rng.integers(0, 2 ** 32, 400_000, dtype=np.uint64)])
    exact = (a.astype(np.float64) + 0.5) * 2.0 ** -32        # exact in f64 (34 significant bits)
    got = _u01f32(a).astype(np.float64)
    half_ulp = np.spacing(exact.astype(np.float32)).astype(np.float64) / 2
    assert np.all(got - exact <= half_ulp)
    # and below by at most 1.5 ulp (truncation of up to one ulp, then the rounding)
    assert np.all(exact - got <= 3 * half_ulp)
    assert np.all(got > 0) and np.all(got <= 1.0)


def test_draw_free_displacement_factor():
    b_max = math.sqrt(3 * 2 * 33 * math.log(2))
    assert 11.71 < b_max < 11.72 and b_max < 11.8
