"""The oracle against the reference's own IRT outputs at 1, 3 and 5 keV
(experiments/results/2026-05-07/level-4/E10-irt-vs-karamitros.json,
summary.perEnergyHeadline: tools/run_irt.cjs on 4096-primary rad_buf dumps of
the WebGPU transport), read from the committed fixture
tests/golden/reference_outputs.json (made by tests/golden/make_golden.py).

The oracle runs in reference RNG mode (xoshiro + seedPrimaryRNG with floor(E),
cutoff 7.4 eV, as runAtEnergy does) and its IRT restatement to 1 us.  The
reference values are one sample of 4096 tracks; with 1024-4096 tracks here the
combined statistical spread of G(1 us) is about 1 %, so the band is 3 %."""
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_outputs.json")))
SPECIES = ("OH", "eaq", "H", "H2O2", "H2")


def e10_row(E):
    return next(r for r in GOLD["e10_irt_G_1us"] if r["E_eV"] == E)


@pytest.mark.parametrize("E,npri", [(1000, 4096), (3000, 1024), (5000, 1024)])
def test_oracle_G_1us_matches_reference_irt(E, npri):
    o = oracle.transport(npri, float(E), seed=E, rng_mode=1, ce_eV=7.4)
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    r = oracle.irt(o["rad"], nth, float(E), seed=3)
    ref = e10_row(E)["G"]
    for got, sp in zip(r["G"][6], SPECIES):
        assert abs(got - ref[sp]) / ref[sp] < 0.03, (E, sp, got, ref[sp])


def test_fixture_is_the_published_10keV_run():
    w = GOLD["webgpu_10keV"]
    assert w["n_primaries"] == 4096 and w["E_eV"] == 10000
    assert w["tracking"]["csdaNm"] == 2714.4
    assert e10_row(10000)["G"]["OH"] == pytest.approx(w["chemistry_1us"]["G_OH"], abs=5e-4)

