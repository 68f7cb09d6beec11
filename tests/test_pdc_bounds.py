"""Error bounds that the f32 prefilter of SamplePDC (public/irt-worker.js:91-113)
relies on, checked against 60-digit arithmetic.

The IRT kernels decide most PDC trials in f32 and keep the f64 evaluation for
trials whose bracket straddles the draw.  For z >= 6 the bracket uses
1 - Q = beta + (1 - beta) h s, h = 1/(2 z^2), with s the truncated asymptotic
series of erfcx; the f64 value it must enclose is computed with the continued
fraction of erfcx_pos.  Both error figures written beside that code are
pinned here."""
import numpy as np
import pytest

mp = pytest.importorskip("mpmath")


def erfcx_cf(x):
    """erfcx_pos for x >= 6: the 30-term continued fraction (irt-worker.js:53-88)."""
    f = 0.0
    for n in range(30, 0, -1):
        f = (0.5 * n) / (x + f)
    return 0.5641895835477563 / (x + f)


def hs_f32(z):
    """h s of the kernel, in f32 with correctly rounded 1/z."""
    f32 = np.float32
    zf = f32(z)
    iz = f32(1) / zf
    h = f32(0.5) * iz * iz
    s = f32(1) - f32(13) * h
    for c in (11, 9, 7, 5, 3):
        s = f32(1) - f32(c) * h * s
    return zf, h * s


ZS = np.concatenate([np.linspace(6, 30, 600), np.logspace(np.log10(30), 15, 600)])


def test_continued_fraction_within_2p2e_16():
    with mp.workdps(50):
        worst = 0.0
        for z in ZS:
            zm = mp.mpf(float(z))
            ex = mp.erfc(zm) * mp.exp(zm * zm)
            worst = max(worst, abs(float((mp.mpf(erfcx_cf(float(z))) - ex) / ex)))
    assert worst <= 2.2e-16


def test_asymptotic_series_f32_within_2p2e_7():
    with mp.workdps(60):
        worst = 0.0
        for z in ZS:
            zf, hs = hs_f32(z)
            zm = mp.mpf(float(zf))
            g = 1 - mp.sqrt(mp.pi) * zm * mp.erfc(zm) * mp.exp(zm * zm)   # = h s exactly
            worst = max(worst, abs(float((mp.mpf(float(hs)) - g) / g)))
    assert worst <= 2.3e-7
