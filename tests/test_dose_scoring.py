"""Dose-grid scoring (src/scoring/ssb-dsb.ts:227-334) and dose reductions
(src/scoring/dose.ts:13-85).

CPU: the oracle against a transcription of the JavaScript loops with JS
number semantics (f64 arithmetic, f32 stores into Float32Arrays).  GPU: the
CUDA kernels against the oracle -- per-site values bit for bit; sums over
sites, which the GPU adds in another order (a tree instead of the
reference's 7.8-million-term running sum), to a relative 1e-9."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from wgdna import _lib

VC = 128


def js_voxel_ssb(d, dose, box_nm):
    vox_nm = (2 * box_nm) / VC
    vox_vol = vox_nm * vox_nm * vox_nm
    half, inv_vox = box_nm, 1 / vox_nm
    r = 0.29
    K = (((4.0 / 3) * math.pi * r * r * r / vox_vol) * 0.15) / 22
    n = d.n_bp
    lam = np.zeros(2 * n, np.float32)
    direct = 0.0
    for fi in range(d.n_fibers):
        fy, fz = float(d.fy[fi]), float(d.fz[fi])
        base = fi * d.n_bp_per
        for b in range(d.n_bp_per):
            bx = d.x0 + b * d.rise
            vx = math.floor((bx + half) * inv_vox)
            if vx < 0 or vx >= VC:
                continue
            y0, z0 = fy + float(d.rbb0[2 * b]), fz + float(d.rbb0[2 * b + 1])
            y1, z1 = fy + float(d.rbb1[2 * b]), fz + float(d.rbb1[2 * b + 1])
            vy0, vz0 = math.floor((y0 + half) * inv_vox), math.floor((z0 + half) * inv_vox)
            vy1, vz1 = math.floor((y1 + half) * inv_vox), math.floor((z1 + half) * inv_vox)
            if 0 <= vy0 < VC and 0 <= vz0 < VC:
                l = int(dose[(vz0 * VC + vy0) * VC + vx]) / 100.0 * K
                lam[base + b] = l
                direct += l
            if 0 <= vy1 < VC and 0 <= vz1 < VC:
                l = int(dose[(vz1 * VC + vy1) * VC + vx]) / 10.0 * K
                lam[n + base + b] = l
                direct += l
    return direct, lam


def js_expected_dsb(d, lam, hits):
    W, n, n_per = 10, d.n_bp, d.n_bp_per
    e = 0.0
    for fi in range(d.n_fibers):
        base = fi * n_per
        s0 = np.zeros(n_per, np.float32)
        s1 = np.zeros(n_per, np.float32)
        a = b_ = 0.0
        for b in range(n_per):
            v0 = float(lam[base + b]) + (1 if hits is not None and hits[base + b] == 1 else 0)
            v1 = float(lam[n + base + b]) + (1 if hits is not None and hits[n + base + b] == 1 else 0)
            s0[b], s1[b] = v0, v1
            a += v0
            b_ += v1
        if a == 0 or b_ == 0:
            continue
        win = 0.0
        for b in range(min(W, n_per - 1) + 1):
            win += float(s1[b])
        for b in range(n_per):
            e += float(s0[b]) * win
            if b + 1 + W < n_per:
                win += float(s1[b + 1 + W])
            if b - W >= 0:
                win -= float(s1[b - W])
    return e


def small_target():
    return oracle.DnaTarget(L_nm=300.0, grid_N=3, spacing_nm=30.0)


def dense_dose(seed, box_nm):
    """A dose grid dense around the small target (the grid spans +-box_nm)."""
    rng = np.random.default_rng(seed)
    g = np.zeros(VC ** 3, np.uint32)
    idx = rng.integers(0, VC ** 3, 400_000)
    g[idx] = rng.integers(1, 50_000, idx.size, dtype=np.uint32)
    return g


def test_voxel_ssb_oracle_equals_js_transcription():
    d = small_target()
    box = 200.0
    dose = dense_dose(1, box)
    e, lam = oracle.voxel_ssb(d, dose, box_nm=box)
    ej, lj = js_voxel_ssb(d, dose, box)
    np.testing.assert_array_equal(lam.view(np.uint32), lj.view(np.uint32))
    assert e == ej and e > 0


def test_expected_dsb_local_oracle_equals_js_transcription():
    d = small_target()
    _, lam = oracle.voxel_ssb(d, dense_dose(2, 200.0), box_nm=200.0)
    hits = (np.random.default_rng(3).random(2 * d.n_bp) < 0.01).astype(np.uint8)
    for h in (None, hits):
        assert oracle.expected_dsb_local(d, lam, h) == js_expected_dsb(d, lam, h)


def test_dose_reductions_oracle():
    g = dense_dose(4, 100.0)
    assert oracle.dose_sum_ev(g) == int(g.astype(np.uint64).sum()) / 100.0
    p = oracle.dose_projection(g, 0)
    np.testing.assert_array_equal(p, g.reshape(VC, VC, VC).astype(np.float64).sum(axis=0).astype(np.float32))
    p = oracle.dose_projection(g, 1)
    np.testing.assert_array_equal(p, g.reshape(VC, VC, VC).astype(np.float64).sum(axis=2).astype(np.float32))


@pytest.mark.gpu
def test_dose_scoring_gpu_equals_oracle(ctx):
    L = _lib.lib()
    o = oracle.transport(96, 10000.0, seed=23, rng_mode=0)
    dose = np.ascontiguousarray(o["dose"])
    d = oracle.DnaTarget()
    box = 15000.0
    e_ref, lam_ref = oracle.voxel_ssb(d, dose, box_nm=box)
    lam = np.zeros(2 * d.n_bp, np.float32)
    e = C.c_double()
    _lib.check("voxel", L.wgdna_score_voxel_ssb(ctx.h, _lib.ptr(dose), box, _lib.ptr(lam), C.byref(e)))
    np.testing.assert_array_equal(lam.view(np.uint32), lam_ref.view(np.uint32))
    assert e.value == pytest.approx(e_ref, rel=1e-9)
    hits = (np.random.default_rng(5).random(2 * d.n_bp) < 0.001).astype(np.uint8)
    for h in (None, hits):
        x = C.c_double()
        _lib.check("dsb", L.wgdna_expected_dsb_local(ctx.h, None, _lib.ptr(h) if h is not None else None,
                                                     C.byref(x)))
        assert x.value == pytest.approx(oracle.expected_dsb_local(d, lam_ref, h), rel=1e-9)
    s = C.c_double()
    _lib.check("sum", L.wgdna_dose_sum(ctx.h, _lib.ptr(dose), C.byref(s)))
    assert s.value == oracle.dose_sum_ev(dose)
    for axis in (0, 1):
        p = np.zeros(VC * VC, np.float32)
        _lib.check("proj", L.wgdna_dose_projection(ctx.h, _lib.ptr(dose), axis, _lib.ptr(p)))
        np.testing.assert_array_equal(p.reshape(VC, VC), oracle.dose_projection(dose, axis))


def test_rad_dump_round_trip(tmp_path):
    from wgdna import dumps
    o = oracle.transport(8, 1000.0, seed=2, rng_mode=0, want_dose=False)
    p = dumps.write_rad_dump(str(tmp_path), 1000, 8, o["rad"])
    assert p.endswith("rad_E1000_N8.bin")
    rad, E, n = dumps.read_rad_dump(p)
    assert (E, n) == (1000, 8)
    np.testing.assert_array_equal(rad.view(np.uint32), o["rad"].view(np.uint32))
    assert dumps.thermalised_primaries(rad) <= 8
    # a dump read back gives the same IRT as the list it was written from
    a = oracle.irt(rad, 8, 1000.0, seed=4)
    b = oracle.irt(o["rad"], 8, 1000.0, seed=4)
    np.testing.assert_array_equal(a["tl"], b["tl"])


def test_results_table_classes():
    from wgdna import app
    assert app.classify(1.05) == "ok" and app.classify(0.6) == "meh" and app.classify(3.0) == "bad"
