"""Surrogate chemistry: the MLP's forward and backward tensor-core kernels
against the CPU reference (oracle/surrogate_ref.py), whose gradient formulas
are checked by finite differences; per-track IRT curves against the oracle;
and a trained network against the IRT it replaces."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import surrogate_ref as ref
import wgdna
from wgdna import _lib


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = ref.init(3).astype(np.float64)
    p[ref.OFFS[0][1]:ref.OFFS[0][1] + 128] = rng.normal(0, 0.1, 128)      # nonzero biases
    X = rng.normal(size=(7, ref.IN))
    T = rng.normal(size=(7, ref.OUT))
    loss, g = ref.loss_and_grad(p, X, T, exact=True)
    idx = rng.choice(ref.NPARAM, 60, replace=False)
    h = 1e-6
    for i in idx:
        q = p.copy(); q[i] += h
        lp, _ = ref.loss_and_grad(q, X, T, exact=True)
        q[i] -= 2 * h
        lm, _ = ref.loss_and_grad(q, X, T, exact=True)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125 + 2 ** -9, -3.14159], np.float32)
    got = ref.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1.0); 1.005859375 rounds up
    np.testing.assert_array_equal(got[:3], np.array([1.0, 1.0, 1.0078125], np.float32))
    assert got[4] == np.float32(-3.140625)


def _ctx_model(ctx, seed=5):
    L = _lib.lib()
    _lib.check("init", L.wgdna_surrogate_init(ctx.h, seed))
    p = np.zeros(ref.NPARAM, np.float32)
    _lib.check("params", L.wgdna_surrogate_params(ctx.h, _lib.ptr(p), None))
    return L, p


@pytest.mark.gpu
def test_forward_matches_reference(ctx):
    L, p = _ctx_model(ctx)
    rng = np.random.default_rng(2)
    # nonzero biases so the bias path is exercised
    p[ref.OFFS[1][1]:ref.OFFS[1][1] + 128] = rng.normal(0, 0.2, 128).astype(np.float32)
    p[ref.OFFS[3][1]:ref.OFFS[3][1] + 80] = rng.normal(0, 0.2, 80).astype(np.float32)
    _lib.check("params", L.wgdna_surrogate_params(ctx.h, None, _lib.ptr(p)))
    n = 300                                                     # two full tiles and a partial one
    X = rng.normal(size=(n, ref.IN)).astype(np.float32)
    G = np.zeros((n, ref.OUT), np.float32)
    _lib.check("predict", L.wgdna_surrogate_predict(ctx.h, _lib.ptr(X), n, _lib.ptr(G)))
    Y, _ = ref.forward(p, X)
    err = np.abs(G - Y).max() / np.abs(Y).max()
    assert err < 1e-2, err


@pytest.mark.gpu
def test_gradient_matches_reference(ctx):
    L, p = _ctx_model(ctx, seed=9)
    rng = np.random.default_rng(4)
    n = 256
    X = rng.normal(size=(n, ref.IN)).astype(np.float32)
    T = rng.normal(size=(n, ref.OUT)).astype(np.float32)
    _lib.check("load", L.wgdna_surrogate_load(ctx.h, _lib.ptr(X), _lib.ptr(T), n))
    g = np.zeros(ref.NPARAM, np.float32)
    loss = C.c_double()
    _lib.check("grad", L.wgdna_surrogate_grad(ctx.h, n, _lib.ptr(g), C.byref(loss)))
    lr, gr = ref.loss_and_grad(p, X, T)
    assert abs(loss.value - lr) <= 1e-4 * lr
    for (w0, b0), (n_out, n_in) in zip(ref.OFFS, ref.SHAPES):
        for a, b in ((w0, w0 + n_out * n_in), (b0, b0 + n_out)):
            d = np.linalg.norm(g[a:b] - gr[a:b]) / np.linalg.norm(gr[a:b])
            assert d < 2e-2, (a, d)


@pytest.mark.gpu
def test_irt_curves_bit_exact(ctx):
    o = oracle.transport(32, 10000.0, seed=17, rng_mode=0, want_dose=False)
    rad = np.ascontiguousarray(o["rad"])
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    ref_ = oracle.irt(rad, nth, 10000.0, seed=2, curves=True)
    L = _lib.lib()
    _lib.check("rec", L.wgdna_irt_record_curves(ctx.h, 1))
    r = _lib.IrtResult()
    _lib.check("irt", L.wgdna_run_irt(ctx.h, _lib.ptr(rad), rad.shape[0], nth, 10000.0, 2, C.byref(r)))
    n = C.c_uint64()
    _lib.check("curves", L.wgdna_irt_curves(ctx.h, None, 0, C.byref(n)))
    cv = np.zeros((n.value, 16, 5), np.float32)
    _lib.check("curves", L.wgdna_irt_curves(ctx.h, _lib.ptr(cv), n.value, C.byref(n)))
    _lib.check("rec", L.wgdna_irt_record_curves(ctx.h, 0))
    np.testing.assert_array_equal(cv, ref_["curves"][:n.value])
    # the curve at 1 us is the 7th checkpoint summed over tracks
    np.testing.assert_array_equal(cv[:, 15, :].sum(axis=0), ref_["tl"][6])


@pytest.mark.gpu
def test_trained_surrogate_against_irt(ctx):
    """Trained by the library's kernels with the recipe the benchmark uses
    (~2e5 IRT tracks at 1, 3 and 10 keV), then three held-out 4096-track batches
    at each energy: the batch G(t) within 2 % of the IRT's on the same 12,288
    tracks at every curve time and species (where G > 0.05), and the surrogate
    chemistry at least 20 times faster than the batched IRT on the same tracks
    (what the network gains over the method alone)."""
    from wgdna import surrogate as S
    info = S.train_on_irt(ctx)
    assert info["loss_last"] < info["loss_first"]
    for E in S.TRAIN_ENERGIES:
        gis, gcs = [], []
        for b in range(3):                                     # 12,288 held-out tracks
            gi, gc, irt_ms, sg_ms, Xh = S.held_out(ctx, E, 424242 + int(E) + 17 * b)
            assert irt_ms >= 20.0 * sg_ms, (E, irt_ms, sg_ms)
            gis.append(gi)
            gcs.append(gc)
        e1, eall = S.g_errors(np.mean(gis, axis=0), np.mean(gcs, axis=0))
        assert eall <= 0.02, (E, e1, eall)
        if E == 10000.0 and Xh.shape[0] == 4096:               # every track holds species
            # the whole-batch device path matches the host-side prediction
            gp = S.batch_G(S.predict(ctx, Xh), np.full(4096, E))
            np.testing.assert_allclose(gc, gp, rtol=2e-3, atol=1e-4)


@pytest.mark.gpu
def test_out_of_range_batch_falls_back_to_the_irt(ctx):
    """A network fitted at 10 keV only: a 10 keV batch stays in its range and
    runs the surrogate; a 300 eV batch leaves it and runs the IRT, whose G at the
    curve times that are also checkpoints (1 ps, 100 ps, 10 ns, 1 us) equals
    a direct wgdna_irt call's."""
    from wgdna import surrogate as S
    X, G, _, _ = S.track_data(ctx, np.full(4096, 10000.0, np.float32), 9001)
    S.fit(ctx, X, G, schedule=((3, 2e-3),), seed=2)
    L = _lib.lib()
    for E, expect_sg in ((10000.0, True), (300.0, False)):
        p = wgdna.transport_params(1024, E, 15000.0, 7.5, seed=77, dna_enable=0)
        st = _lib.TransportStats()
        _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
        Gc, used = S.chemistry(ctx, st.n_therm, E, seed=1)
        assert used == expect_sg, E
        if not used:
            ir = _lib.IrtResult()
            _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, E, 1, C.byref(ir)))
            np.testing.assert_allclose(Gc[[0, 5, 10, 15]], np.array(ir.G)[[0, 2, 4, 6]], rtol=1e-12, atol=0)
