"""The benchmark's own workload through the C ABI against the oracle, bit for
bit, and its physics against the reference's published 10 keV run (GPU tests).

Workload (bench.py's default step): 4096 primaries at 10 keV, box +-15 um,
cutoff 7.5 eV, Philox seed 0, DNA on; IRT to 1 us with seed 1; direct SSB with
the LCG seed 0x12345678 and DSB clustering on the 21 x 21 fibre grid.

Bit-exact: results, counters, canonical rad_buf, dose grid, step count, IRT
checkpoint counts / reactions / pairs / events / per-track curves, SSB counts,
LCG state, hit bytes and DSB.  The f64 sum of all deposits is accumulated in
another order: rtol 1e-12.  Physics against validation/webgpu-results.json:6-30
(4096 primaries, cutoff 7.4 eV, the reference's own generator): CSDA, ions per
primary, initial G and G(1 us) within 2 sigma, sigma = the per-track standard
deviation times sqrt(1/4096 + 1/4096); SSB_dir and DSB within 2 sqrt(sum) (Poisson); kernel
hits within 2 sigma with sigma from the spread of eight further seeds (hits
come in clusters along a track, so they spread more than a Poisson count).
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

import oracle
import wgdna
from wgdna import _lib

pytestmark = pytest.mark.gpu

NP, E, BOX, CE, SEED, IRT_SEED, LCG = 4096, 10000.0, 15000.0, 7.5, 0, 1, 0x12345678
PUB = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                  "reference_outputs.json")))["webgpu_10keV"]


def _transport(ctx, seed):
    p = wgdna.transport_params(NP, E, BOX, CE, seed=seed, dna_enable=1, dna=wgdna.build_dna_target())
    st = _lib.TransportStats()
    _lib.check("wgdna_transport", _lib.lib().wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    return st


@pytest.fixture(scope="module")
def run(ctx):
    L = _lib.lib()
    st = _transport(ctx, SEED)
    res = np.zeros(NP * 8, np.float32)
    dose = np.zeros(ctx.vc ** 3, np.uint32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), _lib.ptr(dose), _lib.ptr(rad),
                                                       st.rad_n_stored, C.byref(n)))
    ir = _lib.IrtResult()
    _lib.check("wgdna_irt_record_curves", L.wgdna_irt_record_curves(ctx.h, 1))
    try:
        _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, E, IRT_SEED, C.byref(ir)))
        curves = np.zeros((NP, 16, 5), np.float32)
        _lib.check("wgdna_irt_curves", L.wgdna_irt_curves(ctx.h, _lib.ptr(curves), NP, C.byref(n)))
    finally:
        L.wgdna_irt_record_curves(ctx.h, 0)
    ssb, dsb = _lib.SsbResult(), _lib.DsbResult()
    _lib.check("wgdna_score", L.wgdna_score(ctx.h, LCG, C.byref(ssb), C.byref(dsb)))
    o = oracle.transport(NP, E, seed=SEED, rng_mode=0, dna_enable=1, box_nm=BOX, ce_eV=CE)
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    oi = oracle.irt(o["rad"], nth, E, seed=IRT_SEED, curves=True)
    od = oracle.DnaTarget()
    osc = oracle.score_direct(od, o["rad"], LCG)
    ocl = oracle.cluster_dsb(od, osc["hits"])
    return dict(st=st, res=res, dose=dose, rad=rad, ir=ir, curves=curves, ssb=ssb, dsb=dsb,
                o=o, nth=nth, oi=oi, osc=osc, ocl=ocl)


def test_bench_transport_bit_exact(run):
    from test_gpu_parity import assert_transport_equal
    assert_transport_equal(run["st"], run["res"], run["dose"], run["rad"], run["o"])
    assert run["st"].n_therm == run["nth"] == NP


def test_bench_irt_bit_exact(run):
    ir, oi = run["ir"], run["oi"]
    assert ir.device_error == 0
    np.testing.assert_array_equal(np.array(ir.counts), oi["tl"])
    np.testing.assert_array_equal(np.array(ir.G), oi["G"])
    np.testing.assert_array_equal(np.array(ir.rxn_counts[:]), oi["rxn_counts"])
    assert (ir.n_reacted, ir.n_pairs, ir.n_events) == (oi["n_reacted"], oi["n_pairs"], oi["n_events"])
    np.testing.assert_array_equal(run["curves"], oi["curves"][:NP])


def test_bench_scoring_bit_exact(ctx, run):
    ssb, dsb, osc, ocl = run["ssb"], run["dsb"], run["osc"], run["ocl"]
    assert (ssb.ssb, ssb.ssb0, ssb.ssb1) == (osc["ssb"], osc["ssb0"], osc["ssb1"])
    assert (ssb.candidates, ssb.in_reach, ssb.lcg_state) == (osc["candidates"], osc["in_reach"], osc["lcg_state"])
    assert (dsb.dsb, dsb.ssb0, dsb.ssb1) == (ocl["dsb"], ocl["ssb0"], ocl["ssb1"])
    np.testing.assert_allclose(dsb.dsb_expected, ocl["dsb_expected"], rtol=1e-12)
    # the hit bytes, through the host-buffer entry point on the same rad_buf
    dna = wgdna.build_dna_target()
    rng = wgdna.make_ssb_rng(LCG)
    got = wgdna.score_direct_ssb_events(ctx, dna, run["rad"], run["rad"].shape[0], rng)
    np.testing.assert_array_equal(got["hits"], osc["hits"])


def _within(x, ref, sig, k=2.0):
    return abs(x - ref) < k * sig


def test_bench_physics_within_2_sigma_of_published(ctx, run):
    r = run["res"].reshape(-1, 8)
    ru = r.view(np.uint32)
    th = ru[:, 5] == 0
    f = math.sqrt(1.0 / th.sum() + 1.0 / 4096)
    path, ions = r[th, 0].astype(np.float64), ru[th, 3].astype(np.float64)
    assert _within(path.mean(), PUB["tracking"]["csdaNm"], path.std() * f), path.mean()
    assert _within(ions.mean(), PUB["tracking"]["ionsPerPriPrimaryOnly"], ions.std() * f), ions.mean()
    st = run["st"]
    per100 = st.dep_units / 100.0 / 100.0
    w = np.rint(run["rad"][:, 3]).astype(np.int64)
    pid, code = w >> 3, w & 7
    for k, name, codes in ((0, "G_OH_init", [0]), (1, "G_eaq_init", [1, 5]), (2, "G_H_init", [2])):
        cnt = np.bincount(pid[np.isin(code, codes)], minlength=NP).astype(np.float64)
        assert cnt.sum() == st.counters[k]
        assert _within(st.counters[k] / per100, PUB["pre_chemistry"][name], cnt.std() / 100.0 * f), name
    per_track = run["curves"][:, 15, :].astype(np.float64) / 100.0
    for j, sp in enumerate(("G_OH", "G_eaq", "G_H", "G_H2O2", "G_H2")):
        g = run["ir"].G[6][j]
        assert _within(g, PUB["chemistry_1us"][sp], per_track[:, j].std() * f), (sp, g)
    d = PUB["dna_damage"]
    for got, ref in ((run["ssb"].ssb, d["SSB_dir"]), (run["dsb"].dsb, d["DSB"])):
        assert abs(got - ref) <= 2.0 * math.sqrt(got + ref), (got, ref)
    hits = [int(_transport(ctx, s).counters[4]) for s in range(1, 9)]
    sig = float(np.std(hits, ddof=1)) * math.sqrt(2.0)
    assert _within(int(st.counters[4]), d["kernelHits"], sig), (st.counters[4], hits)
