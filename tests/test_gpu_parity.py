"""CUDA path vs CPU oracle: bit-exact parity on the same seeds (GPU tests).

Transport (Phase A+B), IRT and scoring are compared through the C ABI with
the oracle under oracle/.  Tolerances: integer / byte / index outputs and the
f32 physics outputs must match bit for bit; only the f64 sum of all deposits
(accumulated in a different order) is compared with rtol 1e-12.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import wgdna
from wgdna import _lib

pytestmark = pytest.mark.gpu


def gpu_transport(ctx, np_, E, seed, dna_enable, box=15000.0, ce=7.5):
    p = wgdna.transport_params(np_, E, box, ce, seed=seed, dna_enable=dna_enable,
                               dna=wgdna.build_dna_target())
    st = _lib.TransportStats()
    L = _lib.lib()
    _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    res = np.zeros(np_ * 8, np.float32)
    dose = np.zeros(ctx.vc ** 3, np.uint32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), _lib.ptr(dose), _lib.ptr(rad),
                                                       st.rad_n_stored, C.byref(n)))
    return st, res, dose, rad


def assert_transport_equal(st, res, dose, rad, o):
    assert st.device_error == 0
    np.testing.assert_array_equal(res.view(np.uint32), o["results"].view(np.uint32))
    np.testing.assert_array_equal(np.array(st.counters[:]), o["counters"])
    np.testing.assert_array_equal(np.array(st.sec_stats[:]), o["sec_stats"])
    np.testing.assert_array_equal(np.array(st.dbg[:6]), o["dbg"][:6])
    assert st.rad_dropped == 0 and st.sec_dropped == 0
    assert rad.shape == o["rad"].shape
    np.testing.assert_array_equal(rad.view(np.uint32), o["rad"].view(np.uint32))
    np.testing.assert_array_equal(dose, o["dose"])
    assert st.dep_units == o["dep_units"]
    assert st.steps == o["steps"]
    np.testing.assert_allclose(st.dep_eV_f64, o["dep_eV_f64"], rtol=1e-12)


@pytest.mark.parametrize("E,np_,seed,dna", [(10000.0, 48, 7, 1), (1000.0, 256, 3, 0), (100.0, 512, 11, 0),
                                           (30000.0, 8, 5, 0), (7.0, 16, 1, 0)])
def test_transport_bit_exact(ctx, E, np_, seed, dna):
    st, res, dose, rad = gpu_transport(ctx, np_, E, seed, dna)
    o = oracle.transport(np_, E, seed=seed, rng_mode=0, dna_enable=dna)
    assert_transport_equal(st, res, dose, rad, o)


def test_transport_bit_exact_small_box(ctx):
    """Escapes and the bounds termination of secondaries (box 50 nm)."""
    st, res, dose, rad = gpu_transport(ctx, 64, 5000.0, 9, 0, box=50.0)
    o = oracle.transport(64, 5000.0, seed=9, rng_mode=0, dna_enable=0, box_nm=50.0)
    assert res.view(np.uint32).reshape(-1, 8)[:, 5].sum() > 0      # some primaries escaped
    assert o["sec_stats"][2] > 0
    assert_transport_equal(st, res, dose, rad, o)


def test_irt_bit_exact(ctx):
    o = oracle.transport(48, 10000.0, seed=21, rng_mode=0, want_dose=False)
    rad = np.ascontiguousarray(o["rad"])
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    ref = oracle.irt(rad, nth, 10000.0, seed=5)
    r = _lib.IrtResult()
    _lib.check("wgdna_run_irt", _lib.lib().wgdna_run_irt(ctx.h, _lib.ptr(rad), rad.shape[0], nth, 10000.0, 5,
                                                         C.byref(r)))
    assert r.device_error == 0
    np.testing.assert_array_equal(np.array(r.counts), ref["tl"])
    np.testing.assert_array_equal(np.array(r.rxn_counts[:]), ref["rxn_counts"])
    assert r.n_reacted == ref["n_reacted"] and r.n_pairs == ref["n_pairs"] and r.n_events == ref["n_events"]
    np.testing.assert_array_equal(np.array(r.G), ref["G"])


def test_irt_device_resident_matches_host_input(ctx):
    st, res, dose, rad = gpu_transport(ctx, 32, 10000.0, 13, 1)
    nth = st.n_therm
    r1 = _lib.IrtResult()
    _lib.check("wgdna_irt", _lib.lib().wgdna_irt(ctx.h, nth, 10000.0, 2, C.byref(r1)))
    r2 = _lib.IrtResult()
    rad = np.ascontiguousarray(rad)
    _lib.check("wgdna_run_irt", _lib.lib().wgdna_run_irt(ctx.h, _lib.ptr(rad), rad.shape[0], nth, 10000.0, 2,
                                                         C.byref(r2)))
    np.testing.assert_array_equal(np.array(r1.counts), np.array(r2.counts))
    np.testing.assert_array_equal(np.array(r1.rxn_counts[:]), np.array(r2.rxn_counts[:]))
    ref = oracle.irt(rad, nth, 10000.0, seed=2)
    np.testing.assert_array_equal(np.array(r1.counts), ref["tl"])


def synthetic_sites(dna, n, seed, frac_near=0.3, dup=0.4):
    """rad_buf entries: a fraction placed within 0.4 nm of a backbone atom,
    the rest spread over the grid; some consecutive duplicates."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 4), np.float32)
    i = 0
    while i < n:
        if rng.random() < frac_near:
            f = rng.integers(dna.n_fibers)
            b = rng.integers(dna.n_bp_per)
            s = rng.integers(2)
            off = (dna.rbb0 if s == 0 else dna.rbb1)[2 * b: 2 * b + 2]
            x = dna.x0 + b * dna.rise + rng.normal(0, 0.15)
            y = dna.fy[f] + off[0] + rng.normal(0, 0.15)
            z = dna.fz[f] + off[1] + rng.normal(0, 0.15)
        else:
            x, y, z = rng.uniform(-1600, 1600, 3)
        k = 3 if rng.random() < dup * 0.3 else (2 if rng.random() < dup else 1)
        for _ in range(k):
            if i < n:
                out[i] = (x, y, z, float(rng.integers(0, 7)))
                i += 1
    return out


@pytest.mark.parametrize("n,seed", [(1, 1), (5000, 2), (200_000, 3)])
def test_score_direct_bit_exact(ctx, n, seed):
    dna = wgdna.build_dna_target()
    od = oracle.DnaTarget()
    rad = synthetic_sites(dna, n, seed)
    rng = wgdna.make_ssb_rng()
    got = wgdna.score_direct_ssb_events(ctx, dna, rad, n, rng)
    ref = oracle.score_direct(od, rad, 0x12345678)
    assert got["ssb_count"] == ref["ssb"]
    assert got["candidates"] == ref["candidates"] and got["in_reach"] == ref["in_reach"]
    assert rng.state == ref["lcg_state"]
    np.testing.assert_array_equal(got["hits"], ref["hits"])
    cd = wgdna.cluster_dsb(ctx, dna, got["hits"])
    rc = oracle.cluster_dsb(od, ref["hits"])
    assert (cd["dsb"], cd["ssb0"], cd["ssb1"]) == (rc["dsb"], rc["ssb0"], rc["ssb1"])
    np.testing.assert_allclose(cd["dsb_expected"], rc["dsb_expected"], rtol=1e-12, atol=0)


def test_score_indirect_bit_exact(ctx):
    dna = wgdna.build_dna_target()
    od = oracle.DnaTarget()
    n = 100_000
    pos = synthetic_sites(dna, n, 4, frac_near=0.5, dup=0.0)
    pos[:, 3] = np.random.default_rng(5).integers(0, 3, n)          # species codes 0..2
    alive = (np.random.default_rng(6).random(n) < 0.8).astype(np.uint32)
    rng = wgdna.make_ssb_rng(0xABCDEF)
    got = wgdna.score_indirect_ssb(ctx, dna, pos, alive, n, rng)
    ref = oracle.score_indirect(od, pos, alive, 0xABCDEF)
    assert (got["ssb0"], got["ssb1"]) == (ref["ssb0"], ref["ssb1"])
    assert got["in_reach"] == ref["in_reach"] and got["candidates"] == ref["candidates"]
    assert rng.state == ref["lcg_state"]
    np.testing.assert_array_equal(got["hits"], ref["hits"])


def test_cluster_dense_hits(ctx):
    """Many hits per fibre: greedy pairing order matters."""
    dna = wgdna.build_dna_target()
    od = oracle.DnaTarget()
    hits = (np.random.default_rng(8).random(2 * dna.n_bp) < 0.01).astype(np.uint8)
    cd = wgdna.cluster_dsb(ctx, dna, hits)
    rc = oracle.cluster_dsb(od, hits)
    assert (cd["dsb"], cd["ssb0"], cd["ssb1"]) == (rc["dsb"], rc["ssb0"], rc["ssb1"])
    np.testing.assert_allclose(cd["dsb_expected"], rc["dsb_expected"], rtol=1e-12)


def test_irt_graph_replay_takes_each_seed(ctx):
    """The IRT launch sequence is captured once as a CUDA graph and replayed;
    the seed is read from device memory, so replays with other seeds on the
    same tracks give the oracle's result for each seed."""
    st, res, dose, rad = gpu_transport(ctx, 24, 10000.0, 31, 0)
    rad = np.ascontiguousarray(rad)
    for seed in (7, 8, 7):
        r = _lib.IrtResult()
        _lib.check("wgdna_irt", _lib.lib().wgdna_irt(ctx.h, st.n_therm, 10000.0, seed, C.byref(r)))
        ref = oracle.irt(rad, st.n_therm, 10000.0, seed=seed)
        np.testing.assert_array_equal(np.array(r.counts), ref["tl"])
        assert r.n_pairs == ref["n_pairs"] and r.n_events == ref["n_events"]
        assert r.ms > 0 and r.ms_events > 0
