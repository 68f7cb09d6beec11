"""Pins of the CPU oracle against the reference's published 10 keV outputs
(validation/webgpu-results.json:6-30; 4096 primaries, box +-15 um, cutoff
7.4 eV) and against the reference's own IRT smoke test
(tools/test_worker_codes.cjs:26-93).

The oracle in reference RNG mode uses the reference's xoshiro generator and
seeding (helpers.wgsl:188-190, buffers.ts:91-104) with floor(E) as the seed,
like runAtEnergy.  Statistical pins use 3-sigma bands: the published numbers
are themselves means over 4096 primaries, so sigma combines both samples.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle

_W = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                 "reference_outputs.json")))["webgpu_10keV"]
PUBLISHED = {"csda": _W["tracking"]["csdaNm"], "ions": _W["tracking"]["ionsPerPriPrimaryOnly"],
             "sec_per_pri": _W["tracking"]["secPerPri"], "G_OH": _W["pre_chemistry"]["G_OH_init"],
             "G_eaq": _W["pre_chemistry"]["G_eaq_init"], "G_H": _W["pre_chemistry"]["G_H_init"],
             "G1us": tuple(_W["chemistry_1us"][k] for k in ("G_OH", "G_eaq", "G_H", "G_H2O2", "G_H2"))}


@pytest.fixture(scope="module")
def ref_mode_run():
    return oracle.transport(1024, 10000.0, seed=10000, rng_mode=1, ce_eV=7.4)


def per_primary(o):
    r = o["results"].reshape(-1, 8)
    ru = r.view(np.uint32)
    th = ru[:, 5] == 0
    return r[th, 0].astype(np.float64), ru[th, 3].astype(np.float64), int(th.sum())


def band(x, ref, s, n, n_ref=4096, k=3.0):
    sig = s * math.sqrt(1.0 / n + 1.0 / n_ref)
    return abs(x - ref) < k * sig, sig


def test_transport_matches_published_10keV(ref_mode_run):
    o = ref_mode_run
    path, ions, n = per_primary(o)
    ok, sig = band(path.mean(), PUBLISHED["csda"], path.std(), n)
    assert ok, (path.mean(), sig)
    ok, sig = band(ions.mean(), PUBLISHED["ions"], ions.std(), n)
    assert ok, (ions.mean(), sig)
    assert abs(o["sec_n"] / 1024 - PUBLISHED["sec_per_pri"]) / PUBLISHED["sec_per_pri"] < 0.03
    dep = o["dose"].astype(np.float64).sum() / 100.0
    per100 = dep / 100.0
    c = o["counters"]
    for k, name in ((0, "G_OH"), (1, "G_eaq"), (2, "G_H")):
        assert abs(c[k] / per100 - PUBLISHED[name]) / PUBLISHED[name] < 0.03, name
    # energy conservation: the reference reports 100.0 % (u32 x100 truncation loses ~0.05 %)
    assert 0.998 < dep / (n * 10000.0) <= 1.0
    # the in-grid integer sum equals the dose-grid sum
    assert o["dep_units"] == int(o["dose"].astype(np.uint64).sum())


def test_build_rng_statistics_match_reference_rng(ref_mode_run):
    """The build's Philox streams give the reference's physics statistics."""
    a = ref_mode_run
    b = oracle.transport(1024, 10000.0, seed=0, rng_mode=0, ce_eV=7.4)
    pa, ia, na = per_primary(a)
    pb, ib, nb = per_primary(b)
    s = math.sqrt(pa.var() / na + pb.var() / nb)
    assert abs(pa.mean() - pb.mean()) < 3 * s
    s = math.sqrt(ia.var() / na + ib.var() / nb)
    assert abs(ia.mean() - ib.mean()) < 3 * s


def test_irt_matches_published_G_1us(ref_mode_run):
    o = ref_mode_run
    _, _, n = per_primary(o)
    # first 320 tracks (the rad_buf is in pid order)
    pid = np.floor(o["rad"][:, 3].astype(np.float64) / 8 + 1e-9).astype(np.int64)
    sel = pid < 320
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:320, 5] == 0).sum())
    r = oracle.irt(o["rad"][sel], nth, 10000.0, seed=1)
    g = r["G"][6]
    for got, ref in zip(g, PUBLISHED["G1us"]):
        assert abs(got - ref) / ref < 0.06, (g, PUBLISHED["G1us"])
    # G decreases for the radicals and grows for the molecular products
    assert (np.diff(r["G"][:, 0]) <= 1e-12).all() and (np.diff(r["G"][:, 4]) >= -1e-12).all()


def rec(pid, s, x, y, z):
    return [x, y, z, pid * 8 + s]


def test_worker_codes_smoke_known_answer():
    """tools/test_worker_codes.cjs:26-93: 4 primaries exercising codes 0..7.
    Two H2 markers (pids 1 and 2) and no H2-producing reaction is possible, so
    G(H2) = 2 / (4 * 10000 / 100) = 0.005 at every checkpoint; OH- (pid 1) and
    H3O+ (pid 0) are in different tracks, so reaction 8 cannot fire."""
    buf = np.array([rec(0, 0, 0, 0, 0), rec(0, 1, 2, 0, 0), rec(0, 3, 0, 0, 0),
                    rec(1, 0, 10, 0, 0), rec(1, 6, 10, 0, 0), rec(1, 7, 10, 0, 0),
                    rec(2, 0, 20, 0, 0), rec(2, 0, 20, 0, 0), rec(2, 7, 20, 0, 0),
                    rec(3, 0, 30, 0, 0), rec(3, 2, 30, 0, 0)], dtype=np.float32)
    for seed in (1, 2, 3):
        r = oracle.irt(buf, 4, 10000.0, seed=seed)
        np.testing.assert_array_equal(r["G"][:, 4], np.full(7, 0.005))
        assert r["rxn_counts"][8] == 0 and r["n_tracks"] == 4


def test_irt_contact_pair_known_answer():
    """Two pre-thermalised eaq (code 5, no displacement) at one point: r0 = 0 <=
    sigma, so eaq+eaq -> 2 OH- + H2 fires at t = 0 (irt-worker.js:118)."""
    buf = np.array([rec(0, 5, 1, 2, 3), rec(0, 5, 1, 2, 3)], dtype=np.float32)
    r = oracle.irt(buf, 1, 10000.0, seed=4)
    assert r["rxn_counts"][3] == 1 and r["n_reacted"] == 1
    per100 = 10000.0 / 100
    np.testing.assert_array_equal(r["G"][:, 1], np.zeros(7))
    np.testing.assert_array_equal(r["G"][:, 4], np.full(7, 1 / per100))


def test_irt_beyond_cutoff_known_answer():
    """Species farther apart than R_CUT = 1.45 + 2 sqrt(8 * 9.46 * 1000) nm
    never pair (irt-worker.js:364, 553): the counts stay at their initial values."""
    buf = np.array([rec(0, 5, 0, 0, 0), rec(0, 5, 2000, 0, 0), rec(0, 6, 0, 2000, 0)], dtype=np.float32)
    r = oracle.irt(buf, 1, 10000.0, seed=5)
    assert r["n_reacted"] == 0 and r["n_pairs"] == 0
    np.testing.assert_array_equal(r["tl"][:, 1], np.full(7, 2.0))


def test_irt_h2_markers_only_track_is_dropped():
    """A primary whose only entries are H2 markers never enters the worker's
    priMap (irt-worker.js:387-393), so its markers are not counted."""
    buf = np.array([rec(0, 7, 0, 0, 0), rec(1, 0, 5, 5, 5)], dtype=np.float32)
    r = oracle.irt(buf, 2, 10000.0, seed=6)
    assert r["n_tracks"] == 1
    np.testing.assert_array_equal(r["tl"][:, 4], np.zeros(7))
