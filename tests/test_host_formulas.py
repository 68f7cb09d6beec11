"""Host arithmetic of runAtEnergy and scoreDamageAt10keV against direct
transcriptions of the reference's TypeScript.

The transcriptions below follow the JS statement by statement with Python
floats, which are the same IEEE doubles as JS numbers:
  * src/gpu/dispatch.ts:178-226 -- deposited energy from the u32 dose grid,
    initial G per 100 eV, per-primary means over non-escaped primaries,
    conservation ratio, rad_buf drops;
  * src/app.ts:190-194 -- box dose in Gy, DSB per Gy per Gbp, DSB / SSB
    (Math.pow is the C library's pow here, as in the product code);
  * src/ui/table.ts:21-25 -- classify.
The inputs are oracle transport runs (CPU), including a small box with
escaped primaries and a cap below the rad_buf size.
"""
import math

import numpy as np
import pytest

import oracle
from wgdna import app
from wgdna.dispatch import energy_summary


def js_run_at_energy_tail(rs_f32, dose_arr, counters_b, E_eV, np_, sec_n, MAX_RAD):
    """dispatch.ts:178-226 with JS number arithmetic."""
    rs_u32 = rs_f32.view(np.uint32)
    dose_sum = 0
    for i in range(len(dose_arr)):
        dose_sum += int(dose_arr[i])
    total_deposited_eV = dose_sum / 100.0
    rad_OH, rad_eaq, rad_H = int(counters_b[0]), int(counters_b[1]), int(counters_b[2])
    kernel_dna_hits = int(counters_b[4])
    rad_n_raw = int(counters_b[7])
    rad_n_stored = min(rad_n_raw, MAX_RAD)
    rad_dropped = max(0, rad_n_raw - MAX_RAD)
    per100 = total_deposited_eV / 100.0
    G_OH = rad_OH / per100 if per100 > 0 else 0
    G_eaq = rad_eaq / per100 if per100 > 0 else 0
    G_H = rad_H / per100 if per100 > 0 else 0
    total_sum = prod_sum = sp_sum = ions_sum = 0.0
    n_therm = n_esc = 0
    for i in range(np_):
        path = float(rs_f32[i * 8 + 0])
        prod = float(rs_f32[i * 8 + 1])
        finalE = float(rs_f32[i * 8 + 2])
        ni = int(rs_u32[i * 8 + 3])
        esc = int(rs_u32[i * 8 + 5])
        if esc == 1:
            n_esc += 1
            continue
        n_therm += 1
        total_sum += path
        prod_sum += prod
        if path > 0:
            sp_sum += (E_eV - finalE) / path
        ions_sum += ni
    mean_total = total_sum / n_therm if n_therm > 0 else 0
    mean_prod = prod_sum / n_therm if n_therm > 0 else 0
    mean_sp = sp_sum / n_therm if n_therm > 0 else 0
    mean_ions = ions_sum / n_therm if n_therm > 0 else 0
    expected_deposited_eV = n_therm * E_eV
    cons_ratio = total_deposited_eV / expected_deposited_eV if expected_deposited_eV > 0 else 0
    return {"n_therm": n_therm, "n_esc": n_esc, "mean_total": mean_total, "mean_prod": mean_prod,
            "mean_sp": mean_sp, "mean_ions": mean_ions, "total_deposited_eV": total_deposited_eV,
            "expected_deposited_eV": expected_deposited_eV, "cons_ratio": cons_ratio, "G_OH": G_OH,
            "G_eaq": G_eaq, "G_H": G_H, "rad_OH": rad_OH, "rad_eaq": rad_eaq, "rad_H": rad_H,
            "kernel_dna_hits": kernel_dna_hits, "rad_n_raw": rad_n_raw, "rad_n_stored": rad_n_stored,
            "rad_dropped": rad_dropped, "sec_per_pri": sec_n / np_}


def js_damage(totalDepositedEV, boxNm, n_bp, ssb_dir, ssb_ind, dsb):
    """app.ts:190-194."""
    dose_box_Gy = (totalDepositedEV * 1.602e-19) / (math.pow(2 * boxNm * 1e-9, 3) * 1000)
    target_Gbp = n_bp * 1e-9
    dsb_per_gy_gbp = dsb / (dose_box_Gy * target_Gbp) if dose_box_Gy > 0 else 0
    ssbTot = ssb_dir + ssb_ind
    dsbFrac = dsb / ssbTot if ssbTot > 0 else 0
    return dose_box_Gy, dsb_per_gy_gbp, dsbFrac


def js_classify(ratio):
    """table.ts:21-25."""
    if ratio >= 0.9 and ratio <= 1.1:
        return "ok"
    if ratio >= 0.5 and ratio <= 2.0:
        return "meh"
    return "bad"


CASES = [
    # np, E, box half-width nm, cutoff, DNA, rad_buf cap (MAX_RAD)
    (48, 10000.0, 15000.0, 7.5, 1, 16_000_000),
    (64, 1000.0, 40.0, 7.4, 0, 16_000_000),       # small box: escaped primaries
    (32, 3000.0, 15000.0, 7.5, 0, 5_000),         # cap below the rad_buf size: drops counted
]


@pytest.mark.parametrize("np_,E,box,ce,dna,cap", CASES)
def test_energy_summary_matches_dispatch_ts(np_, E, box, ce, dna, cap):
    o = oracle.transport(np_, E, seed=11, box_nm=box, ce_eV=ce, dna_enable=dna, nthreads=4)
    res = o["results"]
    counters = np.array(o["counters"], np.uint32)
    rad_n_raw = int(o["rad"].shape[0])
    counters[7] = rad_n_raw
    js = js_run_at_energy_tail(res, o["dose"], counters, E, np_, o["sec_n"], cap)
    dose_units = int(o["dose"].astype(np.uint64).sum())
    py = energy_summary(E, np_, res, dose_units, counters, o["sec_n"], rad_n_raw, cap)
    for k, v in js.items():
        assert py[k] == v, k
    if box < 100:
        assert js["n_esc"] > 0
    if cap < rad_n_raw:
        assert js["rad_dropped"] == rad_n_raw - cap > 0


def test_damage_numbers_match_app_ts():
    n_bp = 441 * 8823
    for dep, box, s_dir, s_ind, dsb in [(3.9e7, 15000.0, 24, 0, 2), (4.1e7, 15000.0, 30, 0, 4), (0.0, 15000.0, 0, 0, 0),
                                        (1.2345e6, 2500.0, 7, 3, 1), (9.99e8, 50000.0, 101, 0, 0)]:
        assert app.damage_numbers(dep, box, n_bp, s_dir, s_ind, dsb) == js_damage(dep, box, n_bp, s_dir, s_ind, dsb)
    # the published 10 keV row: ~4096 x 10 keV deposited in the 30 um box is ~0.243 Gy
    gy, _, _ = app.damage_numbers(4096 * 10000.0 * 0.9997, 15000.0, n_bp, 24, 0, 2)
    assert abs(gy - 0.243) < 0.001


def test_classify_matches_table_ts():
    for r in [0.0, 0.49, 0.5, 0.8999, 0.9, 1.0, 1.1, 1.1001, 2.0, 2.0001, float("inf")]:
        assert app.classify(r) == js_classify(r)


def test_oracle_secondary_cap_counting():
    """dispatch.ts:124-126 with the emission rule of primary.wgsl:363-364:
    sec_n = min(emitted, MAX_SEC), sec_dropped = emitted - sec_n, and dropped
    secondaries leave their energy undeposited."""
    full = oracle.transport(16, 10000.0, seed=3, nthreads=1, want_dose=False)
    cap = oracle.transport(16, 10000.0, seed=3, nthreads=1, want_dose=False, max_sec=300)
    assert not full["capped"] and full["sec_n"] == full["counters"][6]
    assert cap["capped"] and cap["sec_n"] == 300 and cap["counters"][6] > 300
    assert cap["dep_eV_f64"] < full["dep_eV_f64"]
    # primaries run one after another here: the first primaries keep every secondary
    r0, r1 = full["results"].reshape(-1, 8), cap["results"].reshape(-1, 8)
    assert np.array_equal(r0[0].view(np.uint32), r1[0].view(np.uint32))
