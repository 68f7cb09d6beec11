"""Pins of the CPU oracle against the reference's published 10 keV outputs
(validation/webgpu-results.json:6-30; 4096 primaries, box +-15 um, cutoff
7.4 eV) and against the reference's own IRT smoke test
(tools/test_worker_codes.cjs:26-93).

The oracle in reference RNG mode uses the reference's xoshiro generator and
seeding (helpers.wgsl:188-190, buffers.ts:91-104) with floor(E) as the seed,
like runAtEnergy, on the same 4096 primaries.  Statistical pins use 2-sigma
bands: sigma is the per-track standard deviation of the quantity (path, ions,
species counts per 100 eV, IRT counts at 1 us per 100 eV) times
sqrt(1/n + 1/4096), since the published numbers are themselves means over 4096
primaries.  The DNA-damage counts (SSB_dir, DSB, kernel hits) are Poisson
counts: the band is 2 sqrt(published + ours).
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
             "G1us": tuple(_W["chemistry_1us"][k] for k in ("G_OH", "G_eaq", "G_H", "G_H2O2", "G_H2")),
             "damage": _W["dna_damage"]}
N = 4096
K = 2.0


@pytest.fixture(scope="module")
def ref_mode_run():
    return oracle.transport(N, 10000.0, seed=10000, rng_mode=1, ce_eV=7.4)


@pytest.fixture(scope="module")
def ref_mode_irt(ref_mode_run):
    _, _, n = per_primary(ref_mode_run)
    return oracle.irt(ref_mode_run["rad"], n, 10000.0, seed=1, curves=True)


def per_primary(o):
    r = o["results"].reshape(-1, 8)
    ru = r.view(np.uint32)
    th = ru[:, 5] == 0
    return r[th, 0].astype(np.float64), ru[th, 3].astype(np.float64), int(th.sum())


def band(x, ref, s, n, n_ref=N, k=K):
    sig = s * math.sqrt(1.0 / n + 1.0 / n_ref)
    return abs(x - ref) < k * sig, sig


def test_transport_matches_published_10keV(ref_mode_run):
    o = ref_mode_run
    path, ions, n = per_primary(o)
    assert n == N                                       # nothing escapes the 30 um box
    ok, sig = band(path.mean(), PUBLISHED["csda"], path.std(), n)
    assert ok, (path.mean(), sig)
    ok, sig = band(ions.mean(), PUBLISHED["ions"], ions.std(), n)
    assert ok, (ions.mean(), sig)
    assert abs(o["sec_n"] / N - PUBLISHED["sec_per_pri"]) / PUBLISHED["sec_per_pri"] < 0.01
    dep = o["dose"].astype(np.float64).sum() / 100.0
    per100 = dep / 100.0
    c = o["counters"]
    # per-primary species counts from the rad_buf codes (OH 0, e-aq 1 and 5, H 2)
    w = np.rint(o["rad"][:, 3]).astype(np.int64)
    pid, code = w >> 3, w & 7
    for k, name, codes in ((0, "G_OH", [0]), (1, "G_eaq", [1, 5]), (2, "G_H", [2])):
        cnt = np.bincount(pid[np.isin(code, codes)], minlength=N).astype(np.float64)
        assert cnt.sum() == c[k], name
        ok, sig = band(c[k] / per100, PUBLISHED[name], cnt.std() / 100.0, N)
        assert ok, (name, c[k] / per100, sig)
    # energy conservation: the reference reports 100.0 % (u32 x100 truncation loses ~0.05 %)
    assert 0.998 < dep / (n * 10000.0) <= 1.0
    # the in-grid integer sum equals the dose-grid sum
    assert o["dep_units"] == int(o["dose"].astype(np.uint64).sum())


def test_dna_damage_matches_published_10keV(ref_mode_run):
    """SSB_dir 24, DSB 2, kernel hits 117 (webgpu-results.json:24-30): direct
    SSB scoring with the reference's LCG seed, greedy +-10 bp DSB clustering."""
    o = ref_mode_run
    dna = oracle.DnaTarget()
    sc = oracle.score_direct(dna, o["rad"], 0x12345678)
    cl = oracle.cluster_dsb(dna, sc["hits"])
    pub = PUBLISHED["damage"]
    for got, ref in ((sc["ssb"], pub["SSB_dir"]), (cl["dsb"], pub["DSB"]), (int(o["counters"][4]), pub["kernelHits"])):
        assert abs(got - ref) <= K * math.sqrt(got + ref), (got, ref)


def test_build_rng_statistics_match_reference_rng(ref_mode_run):
    """The build's Philox streams give the reference's physics statistics."""
    a = ref_mode_run
    b = oracle.transport(N, 10000.0, seed=0, rng_mode=0, ce_eV=7.4)
    pa, ia, na = per_primary(a)
    pb, ib, nb = per_primary(b)
    s = math.sqrt(pa.var() / na + pb.var() / nb)
    assert abs(pa.mean() - pb.mean()) < K * s
    s = math.sqrt(ia.var() / na + ib.var() / nb)
    assert abs(ia.mean() - ib.mean()) < K * s


def test_irt_matches_published_G_1us(ref_mode_run, ref_mode_irt):
    _, _, n = per_primary(ref_mode_run)
    r = ref_mode_irt
    g = r["G"][6]
    # per-track G at 1 us: the curve's last time (10^3 ns) is the 1 us checkpoint
    per_track = r["curves"][:N, 15, :].astype(np.float64) / 100.0
    np.testing.assert_allclose(per_track.sum(axis=0) / n, g, rtol=1e-12)
    for j, (got, ref) in enumerate(zip(g, PUBLISHED["G1us"])):
        ok, sig = band(got, ref, per_track[:, j].std(), n)
        assert ok, (j, got, ref, sig)
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
