"""runValidation orchestrator (src/app.ts:42-240) on the CUDA path."""
from .chemistry import run_chemistry_worker
from .constants import (DEFAULT_CHEM_BACKEND, DNA_GRID_N, DNA_LENGTH_NM, DNA_SPACING_NM, KARAMITROS_2011)
from .dispatch import run_at_energy
from .estar import ESTAR
from .geometry import build_dna_target
from .scoring import cluster_dsb, combine_hits, make_ssb_rng, score_direct_ssb_events, score_indirect_ssb
from . import _lib

_cache = None


def _nolog(msg, cls=""):
    pass


def ensure_pipelines(np_, log=_nolog):
    """ensurePipelines (app.ts:65-84): one context cached on np."""
    global _cache
    if _cache is not None and _cache.max_primaries >= np_:
        return _cache
    if _cache is not None:
        _cache.close()
    _cache = _lib.Context(max_primaries=max(np_, 4096))
    log(f"Shaders compiled, buffers allocated (np={np_})", "data")
    return _cache


def damage_numbers(total_deposited_eV, box_nm, n_bp, ssb_dir, ssb_ind, dsb):
    """The arithmetic of scoreDamageAt10keV (app.ts:190-194): box dose in Gy
    over the full edge 2 * box_nm (box_nm is the half-width), DSB per Gy per
    Gbp of target, DSB / SSB."""
    dose_box_Gy = (total_deposited_eV * 1.602e-19) / (((2 * box_nm * 1e-9) ** 3) * 1000)
    target_Gbp = n_bp * 1e-9
    dsb_per_gy_gbp = dsb / (dose_box_Gy * target_Gbp) if dose_box_Gy > 0 else 0.0
    ssb_tot = ssb_dir + ssb_ind
    frac = dsb / ssb_tot if ssb_tot > 0 else 0.0
    return dose_box_Gy, dsb_per_gy_gbp, frac


def score_damage_at_10kev(ctx, dna, chem, rad_buf, rad_n, total_deposited_eV, box_nm, rng, log, kernel_dna_hits):
    """scoreDamageAt10keV (app.ts:167-207)."""
    if chem.get("chem_pos_final") is not None and chem.get("chem_alive_final") is not None:
        indirect = score_indirect_ssb(ctx, dna, chem["chem_pos_final"], chem["chem_alive_final"], chem["chem_n"], rng)
    else:
        indirect = {"hits": None, "ssb0": 0, "ssb1": 0, "candidates": 0, "in_reach": 0}
    direct = score_direct_ssb_events(ctx, dna, rad_buf, rad_n, rng)
    hits = direct["hits"] if indirect["hits"] is None else combine_hits(direct["hits"], indirect["hits"])
    clust = cluster_dsb(ctx, dna, hits)
    ssb_dir = direct["ssb_count"]
    ssb_ind = indirect["ssb0"] + indirect["ssb1"]
    dsb = clust["dsb"]
    dose_box_Gy, dsb_per_gy_gbp, frac = damage_numbers(total_deposited_eV, box_nm, dna.n_bp, ssb_dir, ssb_ind, dsb)
    log(f"    DAMAGE: SSB_dir={ssb_dir}  SSB_ind={ssb_ind}  DSB={dsb}  (DSB/SSB={frac:.3f})  "
        f"box_dose={dose_box_Gy:.3f} Gy  target={dna.n_bp / 1e6:.1f} Mbp  reach_dir={direct['in_reach']} "
        f"reach_ind={indirect['in_reach']}  kernel_hits={kernel_dna_hits or 0}", "data")
    return {"ssb_dir": ssb_dir, "ssb_ind": ssb_ind, "dsb": dsb, "dsb_per_gy_gbp": dsb_per_gy_gbp,
            "dsb_expected": clust["dsb_expected"], "dose_box_Gy": dose_box_Gy}


def log_chemistry_timeline(cr, log):
    log(f"    chemistry IRT: N={cr['chem_n']} radicals, {cr['t_wall']:.0f}ms total", "data")
    log(f"    {'t':<8} {'G(OH)':>7} {'G(eaq)':>7} {'G(H)':>7} {'G(H2O2)':>8} {'G(H2)':>7}", "data")
    for cp in cr["timeline"]:
        log(f"    {cp['label']:<8} {cp['G_OH']:7.3f} {cp['G_eaq']:7.3f} {cp['G_H']:7.3f} {cp['G_H2O2']:8.3f} "
            f"{cp['G_H2']:7.3f}", "data")
    k = KARAMITROS_2011
    log(f"    Karamitros 2011 reference (1 μs): G(OH)={k['G_OH']} G(eaq)={k['G_eaq']} G(H)={k['G_H']} "
        f"G(H2O2)={k['G_H2O2']} G(H2)={k['G_H2']}", "data")


def run_validation(np=4096, boxNm=15000.0, ceEV=7.4, log=_nolog, chemBackend=DEFAULT_CHEM_BACKEND,
                   energies=None, device_chemistry=True):
    """runValidation (app.ts:91-161): the ESTAR sweep, chemistry + damage at 10 keV.

    Returns one row per energy (the reference paints them into a table).
    chemBackend 'worker' runs the CUDA IRT; 'gpu' the grid-hash diffusion-reaction
    backend (its radical positions feed the indirect SSB scoring); 'none'
    skips chemistry (src/chemistry/backend.ts:16-18)."""
    if chemBackend not in ("worker", "gpu", "none"):
        raise ValueError(f"chemBackend {chemBackend!r}: expected 'worker', 'gpu' or 'none'")
    ctx = ensure_pipelines(np, log)
    log(f"Running {np} primaries at {len(ESTAR)} energies, box={boxNm}nm, cutoff={ceEV}eV", "data")
    dna = build_dna_target(DNA_LENGTH_NM, DNA_GRID_N, DNA_SPACING_NM)
    log(f"DNA target: {dna.n_fibers} fibers × {dna.n_bp_per} bp = {dna.n_bp / 1e6:.2f} Mbp "
        f"({DNA_LENGTH_NM} nm, {DNA_GRID_N}² grid, {DNA_SPACING_NM} nm spacing)", "data")
    rng = make_ssb_rng()
    if chemBackend == "none":
        chem = None
    elif chemBackend == "gpu":
        from .chemistry import run_chemistry_grid
        chem = lambda rb, rn, nt, e: run_chemistry_grid(ctx, nt, e, rad_n=rn)    # device rad_buf
    elif device_chemistry:
        chem = "device"
    else:
        chem = lambda rb, rn, nt, e: run_chemistry_worker(ctx, rb, rn, nt, e, log)
    rows = []
    for ref in ESTAR:
        if energies is not None and ref["E"] not in energies:
            continue
        r = run_at_energy(ctx, ref["E"], np, boxNm, ceEV, dna, chem)
        csda_ratio = r["mean_total"] / ref["csda"]
        damage = None
        if r["chem_result"] is not None and r["rad_buf_final"] is not None and ref["E"] == 10000:
            damage = score_damage_at_10kev(ctx, dna, r["chem_result"], r["rad_buf_final"], r["rad_n_stored"],
                                           r["total_deposited_eV"], boxNm, rng, log, r["kernel_dna_hits"])
        drop = f" ⚠{r['rad_dropped']}dropped" if r["rad_dropped"] > 0 else ""
        log(f"  E={r['E']} eV: CSDA={r['mean_total']:.1f}nm ({csda_ratio:.2f}×) ions/pri={r['mean_ions']:.1f} "
            f"sec/pri={r['sec_per_pri']:.1f} G_init(OH/eaq/H)={r['G_OH']:.2f}/{r['G_eaq']:.2f}/{r['G_H']:.2f} "
            f"rad_n={r['rad_n_stored']}{drop} E_cons={r['cons_ratio'] * 100:.1f}%", "data")
        if r["chem_result"] is not None:
            log_chemistry_timeline(r["chem_result"], log)
        rows.append({"ref": ref, "result": r, "damage": damage, "csda_ratio": csda_ratio})
    log("Validation run complete.", "ok")
    return rows


def results_json(rows, n_primaries):
    """The shape of validation/webgpu-results.json for the 10 keV row."""
    for row in rows:
        if row["ref"]["E"] != 10000:
            continue
        r, d = row["result"], row["damage"] or {}
        tl = (r["chem_result"] or {}).get("timeline") or [{}] * 7
        last = tl[-1]
        return {
            "harnessVersion": "wgdna-b200",
            "primaryEnergyEv": 10000,
            "nPrimaries": n_primaries,
            "tracking": {"csdaNm": r["mean_total"], "ionsPerPriPrimaryOnly": r["mean_ions"],
                         "secPerPri": r["sec_per_pri"], "eConservationPct": r["cons_ratio"] * 100},
            "preChemistry": {"G_OH_init": r["G_OH"], "G_eaq_init": r["G_eaq"], "G_H_init": r["G_H"]},
            "chemistry1Us": {k: last.get(k) for k in ("G_OH", "G_eaq", "G_H", "G_H2O2", "G_H2")},
            "dnaDamage": {"SSB_dir": d.get("ssb_dir"), "SSB_ind": d.get("ssb_ind"), "DSB": d.get("dsb"),
                          "kernelHits": r["kernel_dna_hits"]},
        }
    return None


def classify(ratio):
    """classify (src/ui/table.ts:21-25): 'ok' within 10 %, 'meh' within 2x, else 'bad'."""
    if 0.9 <= ratio <= 1.1:
        return "ok"
    if 0.5 <= ratio <= 2.0:
        return "meh"
    return "bad"


def results_table(rows):
    """The cells of the results table, one dict per energy, in the order of
    appendResultRow (src/ui/table.ts:38-73)."""
    out = []
    for row in rows:
        r, est = row["result"], row["ref"]
        d = row["damage"] or {"ssb_dir": 0, "ssb_ind": 0, "dsb": 0, "dsb_per_gy_gbp": 0}
        csda_ratio = r["mean_total"] / est["csda"]
        sp_ratio = r["mean_sp"] / est["sp"]
        out.append({
            "E_eV": r["E"], "n_therm": r["n_therm"], "n_esc": r["n_esc"],
            "csda_nm": r["mean_total"], "estar_csda_nm": est["csda"], "csda_ratio": csda_ratio,
            "csda_class": classify(csda_ratio),
            "prod_path_nm": r["mean_prod"], "sp_eV_per_nm": r["mean_sp"], "estar_sp": est["sp"],
            "sp_ratio": sp_ratio, "sp_class": classify(sp_ratio),
            "ions_per_primary": r["mean_ions"], "sec_per_primary": r["sec_per_pri"], "sec_dropped": r["sec_dropped"],
            "e_conservation": r["cons_ratio"], "e_conservation_class": classify(r["cons_ratio"]),
            "G_OH_init": r["G_OH"], "G_eaq_init": r["G_eaq"], "G_H_init": r["G_H"],
            "SSB_dir": d["ssb_dir"], "SSB_ind": d["ssb_ind"], "DSB": d["dsb"], "DSB_per_Gy_Gbp": d["dsb_per_gy_gbp"],
            "dt_ms": r["dt"],
        })
    return out


def write_results(rows, n_primaries, path):
    """The sweep's results as JSON: every energy's table row plus the
    validation/webgpu-results.json shape of the 10 keV row."""
    import json
    doc = {"rows": results_table(rows), "tenKeV": results_json(rows, n_primaries)}
    with open(path, "w") as f:
        json.dump(doc, f, indent=1, default=float)
    return doc


runValidation = run_validation
ensurePipelines = ensure_pipelines
