"""Phase A -> Phase B -> readback (src/gpu/dispatch.ts:85-285)."""
import ctypes as C
import math
import time

import numpy as np

from . import _lib
from .constants import MAX_PRIMARY_STEPS, MAX_SEC_STEPS


def transport_params(np_, E_eV, box_nm, ce_eV, dna=None, seed=None, dna_enable=None):
    """The uniform structs P / SP (dispatch.ts:13-70).  The Philox key defaults
    to floor(E), the seed seedPrimaryRNG receives (dispatch.ts:98)."""
    p = _lib.TransportParams()
    p.np = int(np_)
    p.E_eV = float(E_eV)
    p.box_nm = float(box_nm)
    p.ce_eV = float(ce_eV)
    p.max_steps = MAX_PRIMARY_STEPS
    p.sec_steps = MAX_SEC_STEPS
    p.start_half = 0.0
    if dna_enable is None:
        dna_enable = 1 if (dna is not None and E_eV == 10000) else 0
    p.dna_enable = int(dna_enable)
    p.dna_grid_n = dna.grid_N if dna is not None else 21
    p.dna_rise = dna.rise if dna is not None else 0.34
    p.dna_spacing = dna.spacing_nm if dna is not None else 150.0
    p.dna_x0 = dna.x0 if dna is not None else -1499.74
    p.dna_r_bb = dna.r_bb if dna is not None else 1.0
    p.seed = int(math.floor(E_eV)) if seed is None else int(seed)
    return p


def aggregate(results, E_eV):
    """Per-primary aggregation over non-escaped primaries (dispatch.ts:199-226),
    left-to-right f64 sums as the reference's JS loop."""
    r = np.asarray(results, dtype=np.float32).reshape(-1, 8)
    ru = r.view(np.uint32)
    esc = ru[:, 5] == 1
    th = ~esc
    path = r[th, 0].astype(np.float64)
    prod = r[th, 1].astype(np.float64)
    fE = r[th, 2].astype(np.float64)
    ni = ru[th, 3].astype(np.float64)

    def seqsum(a):
        return float(np.cumsum(a)[-1]) if a.size else 0.0

    n_therm = int(th.sum())
    pos = path > 0
    sp_terms = (float(E_eV) - fE[pos]) / path[pos]
    tot, pr, sp, ions = seqsum(path), seqsum(prod), seqsum(sp_terms), seqsum(ni)
    return {
        "n_therm": n_therm, "n_esc": int(esc.sum()),
        "mean_total": tot / n_therm if n_therm else 0.0,
        "mean_prod": pr / n_therm if n_therm else 0.0,
        "mean_sp": sp / n_therm if n_therm else 0.0,
        "mean_ions": ions / n_therm if n_therm else 0.0,
    }


def energy_summary(E_eV, np_, results, dose_units, counters, sec_n, rad_n_raw, max_rad):
    """The readback arithmetic of runAtEnergy (dispatch.ts:178-226): deposited
    energy from the u32 dose grid (x100 per eV), initial G per 100 eV of it,
    the per-primary means over non-escaped primaries and the conservation
    ratio against n_therm * E.  ``dose_units`` is the grid's integer sum."""
    total_deposited_eV = dose_units / 100.0
    per100 = total_deposited_eV / 100.0
    agg = aggregate(results, E_eV)
    expected = agg["n_therm"] * E_eV
    rad_n_stored = min(int(rad_n_raw), int(max_rad))
    return {
        **agg,
        "total_deposited_eV": total_deposited_eV, "expected_deposited_eV": expected,
        "cons_ratio": total_deposited_eV / expected if expected > 0 else 0.0,
        "rad_OH": int(counters[0]), "rad_eaq": int(counters[1]), "rad_H": int(counters[2]),
        "G_OH": counters[0] / per100 if per100 > 0 else 0.0,
        "G_eaq": counters[1] / per100 if per100 > 0 else 0.0,
        "G_H": counters[2] / per100 if per100 > 0 else 0.0,
        "kernel_dna_hits": int(counters[4]),
        "rad_n_raw": int(rad_n_raw), "rad_n_stored": rad_n_stored,
        "rad_dropped": max(0, int(rad_n_raw) - int(max_rad)),
        "sec_per_pri": sec_n / np_,
    }


def run_at_energy(ctx, E_eV, np_, box_nm, ce_eV, dna=None, run_chemistry=None, seed=None, keep_rad=True):
    """runAtEnergy: transport on the GPU, readbacks, optional chemistry callback
    (called only at 10 keV, dispatch.ts:244).  ``run_chemistry`` may be the
    string "device" to run the IRT on the device-resident rad_buf."""
    t0 = time.perf_counter()
    p = transport_params(np_, E_eV, box_nm, ce_eV, dna, seed)
    st = _lib.TransportStats()
    L = _lib.lib()
    _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    results = np.zeros(np_ * 8, np.float32)
    dose = np.zeros(ctx.vc ** 3, np.uint32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32) if keep_rad else None
    n = C.c_uint64()
    _lib.check("wgdna_transport_copy_out",
               L.wgdna_transport_copy_out(ctx.h, _lib.ptr(results), _lib.ptr(dose),
                                          _lib.ptr(rad) if keep_rad else None,
                                          st.rad_n_stored if keep_rad else 0, C.byref(n)))
    summ = energy_summary(E_eV, np_, results, st.dep_units, list(st.counters), st.sec_n, st.rad_n_raw, ctx.max_rad)
    agg = {k: summ[k] for k in ("n_therm", "n_esc", "mean_total", "mean_prod", "mean_sp", "mean_ions")}
    out = {
        "E": E_eV, **summ,
        "dt": 0.0, "t_prim": st.ms_transport, "t_sec": 0.0,
        "sec_n": int(st.sec_n), "sec_dropped": int(st.sec_dropped),
        "sec_terminated_cutoff": int(st.sec_stats[1]), "sec_terminated_bounds": int(st.sec_stats[2]),
        "sec_steps": int(st.sec_stats[3]), "sec_tertiary_ions": int(st.sec_stats[4]),
        "chem_result": None, "rad_buf_final": rad,
        "dose_arr": dose if E_eV == 10000 else None, "results": results, "stats": st,
        "dep_eV_f64": st.dep_eV_f64, "steps": int(st.steps),
    }
    if E_eV == 10000 and st.rad_n_stored > 0 and run_chemistry is not None:
        if run_chemistry == "device":
            from .chemistry import run_chemistry_device
            out["chem_result"] = run_chemistry_device(ctx, agg["n_therm"], E_eV)
        else:
            out["chem_result"] = run_chemistry(rad, int(st.rad_n_stored), agg["n_therm"], E_eV)
    out["dt"] = (time.perf_counter() - t0) * 1000.0
    return out


runAtEnergy = run_at_energy
