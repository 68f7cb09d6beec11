"""The oracle against the reference's own IRT outputs at 1, 3 and 5 keV
(experiments/results/2026-05-07/level-4/E10-irt-vs-karamitros.json,
summary.perEnergyHeadline: tools/run_irt.cjs on 4096-primary rad_buf dumps of
the WebGPU transport), read from the committed fixture
tests/golden/reference_outputs.json (made by tests/golden/make_golden.py).

The oracle runs in reference RNG mode (xoshiro + seedPrimaryRNG with floor(E),
cutoff 7.4 eV, as runAtEnergy does) on 4096 primaries and its IRT restatement
to 1 us.  The reference values are one sample of 4096 tracks, so each G(1 us)
must lie within 2 sigma, sigma = the per-track standard deviation of the
species count per 100 eV times sqrt(1/n + 1/4096)."""
import json
import math
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_outputs.json")))
SPECIES = ("OH", "eaq", "H", "H2O2", "H2")


def e10_row(E):
    return next(r for r in GOLD["e10_irt_G_1us"] if r["E_eV"] == E)


@pytest.mark.parametrize("E", [1000, 3000, 5000])
def test_oracle_G_1us_matches_reference_irt(E):
    n_pri = 4096
    o = oracle.transport(n_pri, float(E), seed=E, rng_mode=1, ce_eV=7.4)
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    r = oracle.irt(o["rad"], nth, float(E), seed=3, curves=True)
    per_track = r["curves"][:n_pri, 15, :].astype(np.float64) / (E / 100.0)
    ref = e10_row(E)["G"]
    for j, (got, sp) in enumerate(zip(r["G"][6], SPECIES)):
        sig = per_track[:, j].std() * math.sqrt(1.0 / nth + 1.0 / 4096)
        assert abs(got - ref[sp]) < 2.0 * sig, (E, sp, got, ref[sp], sig)


def test_fixture_is_the_published_10keV_run():
    w = GOLD["webgpu_10keV"]
    assert w["n_primaries"] == 4096 and w["E_eV"] == 10000
    assert w["tracking"]["csdaNm"] == 2714.4
    assert e10_row(10000)["G"]["OH"] == pytest.approx(w["chemistry_1us"]["G_OH"], abs=5e-4)

