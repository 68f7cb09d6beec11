"""Error bounds of the elementary functions the CUDA path defines for itself.

The kernels (csrc/dmath.cuh) and the oracle (oracle/om.h) carry the same
log / exp / sin / cos / pow so that the GPU reproduces the oracle bit for bit
(the reference's WGSL builtins and JS Math.* are implementation defined).
GPU = oracle equality is shown by the transport and IRT parity tests; this file
bounds the shared arithmetic against 40-digit references (mpmath) in ulps of
the result, over the argument ranges the path uses, and checks how the split
constants of the argument reductions are derived:

  f32 ln2 = 0x3f317200 + 0x35bfbe8e     ln2 rounded to 15 bits + the rest (the
                                        split of fdlibm's e_expf.c, Sun 1993)
  f64 ln2 = 0x1.62e42fefa3800p-1 + 0x1.ef35793c76730p-45
                                        ln2 rounded to 42 bits + the rest (the
                                        split of ARM optimized-routines log_data.c)
  f32 pi/2 = 1.5703125 + 4.837513e-4 + 7.54979e-8
                                        twice Cephes sinf.c's DP1..DP3 (Moshier)
  f64 pi/2 = pio2_1 + pio2_1t parts of fdlibm's e_rem_pio2.c (33 bits each)
"""
import ctypes as C

import mpmath
import numpy as np
import pytest

import oracle

mpmath.mp.dps = 40
N = 1500


def _ev(fn, x):
    L = oracle.lib()
    L.orc_elem.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint64]
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(x)
    assert L.orc_elem(fn, x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
                      x.size) == 0
    return y


def _ulps(x, y, ref, f32):
    worst = 0.0
    for xi, yi in zip(x, y):
        r = ref(mpmath.mpf(float(xi)))
        u = float(np.spacing(np.float32(abs(float(r))))) if f32 else float(np.spacing(abs(float(r))))
        worst = max(worst, abs(float(mpmath.mpf(float(yi)) - r)) / u)
    return worst


RNG = np.random.default_rng(2024)
P13 = mpmath.mpf(float(np.float32(1.3)))
CASES = [
    # fn, name, reference, arguments (the ranges the kernels use), bound in ulps, f32
    (0, "logf", mpmath.log, np.exp(RNG.uniform(np.log(1e-30), np.log(3e4), N)).astype(np.float32), 1.0, True),
    (1, "expf", mpmath.exp, RNG.uniform(-87.0, 0.7, N).astype(np.float32), 1.0, True),
    (2, "sinf", mpmath.sin, RNG.uniform(-6000.0, 6000.0, N).astype(np.float32), 2.0, True),
    (3, "cosf", mpmath.cos, RNG.uniform(-6000.0, 6000.0, N).astype(np.float32), 2.0, True),
    # pow = exp(y ln x): the log's error is amplified by |y ln x| <= 13.4 here
    (4, "powf", lambda x: mpmath.power(x, P13), np.exp(RNG.uniform(np.log(7.5), np.log(3e4), N)).astype(np.float32),
     24.0, True),
    (5, "log", mpmath.log, np.exp(RNG.uniform(np.log(1e-300), np.log(1e300), N)), 1.0, False),
    (6, "exp", mpmath.exp, RNG.uniform(-700.0, 700.0, N), 1.0, False),
    # exp(x) - 1 beyond |x| = ln2/2 keeps exp's absolute error
    (7, "expm1", mpmath.expm1, RNG.uniform(-3.0, 3.0, N), 4.0, False),
    (8, "cos", mpmath.cos, RNG.uniform(-100.0, 100.0, N), 2.0, False),
]


@pytest.mark.parametrize("fn,name,ref,x,bound,f32", CASES, ids=[c[1] for c in CASES])
def test_ulp_bound(fn, name, ref, x, bound, f32):
    y = _ev(fn, x.astype(np.float64))
    if f32:
        assert np.array_equal(y, y.astype(np.float32).astype(np.float64)), "f32 result expected"
    assert _ulps(x, y, ref, f32) <= bound


def test_split_constants():
    ln2, pio2 = mpmath.log(2), mpmath.pi / 2
    # f32 ln2: a 15-bit head (k * hi exact for |k| < 2^9) and the rest rounded to f32
    hi, lo = np.float32(0.693145752), np.float32(1.42860677e-06)
    assert int(hi.view(np.uint32)) == 0x3F317200 and int(lo.view(np.uint32)) == 0x35BFBE8E
    assert np.float32(float(ln2 - mpmath.mpf(float(hi)))) == lo
    # f64 ln2: a 42-bit head (low 11 mantissa bits zero) and the rest rounded to f64
    hi64, lo64 = 6.93147180559890330187e-01, 5.49792301870837115524e-14
    assert float.hex(hi64) == "0x1.62e42fefa3800p-1" and float.hex(lo64) == "0x1.ef35793c76730p-45"
    assert float(ln2 - mpmath.mpf(hi64)) == lo64
    # f32 pi/2 in three parts: 8 + 11 significant bits, then the rest
    p1, p2, p3 = np.float32(1.5703125), np.float32(4.83751297e-04), np.float32(7.54979013e-08)
    assert int(p1.view(np.uint32)) & 0xFFFF == 0 and int(p2.view(np.uint32)) & 0x1FFF == 0
    assert np.float32(float(pio2 - mpmath.mpf(float(p1)) - mpmath.mpf(float(p2)))) == p3
    # f64 pi/2: two 33-bit heads and the rest
    q1, q2, q3 = 1.57079632673412561417e+00, 6.07710050630396597660e-11, 2.02226624879595063154e-21
    assert float.hex(q1).endswith("400000p+0") and float(pio2 - mpmath.mpf(q1) - mpmath.mpf(q2)) == q3
