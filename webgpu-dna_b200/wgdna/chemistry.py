"""Phase C: Karamitros 9-reaction IRT (src/chemistry/worker.ts:32-87 +
public/irt-worker.js:370-699), run by the CUDA kernel through the C ABI."""
import ctypes as C
import time

import numpy as np

from . import _lib
from .constants import CHECKPOINT_LABELS, CHECKPOINTS_NS, IRT_WORKER_RXN_LABELS


def _chem_result(r, rad_n, log=None):
    timeline = []
    for c in range(7):
        g = r.G[c]
        timeline.append({"label": CHECKPOINT_LABELS[c], "t_ns": CHECKPOINTS_NS[c], "G_OH": g[0], "G_eaq": g[1],
                         "G_H": g[2], "G_H2O2": g[3], "G_H2": g[4]})
    tab = _lib.reaction_table()
    rxn_info = [{"label": IRT_WORKER_RXN_LABELS[k], "count": int(r.rxn_counts[k]),
                 "sigma": f"{tab[k, 0]:.4f}", "rc": f"{tab[k, 2]:.3f}"} for k in range(9)]
    res = {"chem_n": int(rad_n), "t_wall": float(r.ms), "timeline": timeline, "chem_pos_final": None,
           "chem_alive_final": None, "n_reacted": int(r.n_reacted), "rxn_info": rxn_info,
           "n_tracks": int(r.n_tracks), "n_pairs": int(r.n_pairs), "n_events": int(r.n_events),
           "counts": np.array(r.counts, dtype=np.float64)}
    if log:
        for cp in timeline:
            log(f"  {cp['label']} {cp['G_OH']:.3f} {cp['G_eaq']:.3f} {cp['G_H']:.3f} "
                f"{cp['G_H2O2']:.3f} {cp['G_H2']:.3f}", "data")
        log(f"  IRT kernel: {res['n_reacted']} reactions in {res['t_wall'] / 1000:.3f}s ({rad_n} radicals)", "data")
    return res


def run_chemistry_worker(ctx, rad_buf, rad_n, n_therm, E_eV, log=None, seed=1):
    """runChemistryWorker: IRT on a host rad_buf (vec4 f32, w = pid*8 + code).

    Like the reference worker, chem_pos_final / chem_alive_final are None, so
    indirect SSB scoring is skipped downstream (app.ts:178-180)."""
    rad = np.ascontiguousarray(np.asarray(rad_buf, dtype=np.float32).reshape(-1)[: 4 * int(rad_n)])
    r = _lib.IrtResult()
    _lib.check("wgdna_run_irt", _lib.lib().wgdna_run_irt(ctx.h, _lib.ptr(rad), int(rad_n), int(n_therm),
                                                         float(E_eV), int(seed), C.byref(r)))
    return _chem_result(r, rad_n, log)


def run_chemistry_device(ctx, n_therm, E_eV, log=None, seed=1):
    """The same IRT on the rad_buf the last transport left in device memory."""
    r = _lib.IrtResult()
    _lib.check("wgdna_irt", _lib.lib().wgdna_irt(ctx.h, int(n_therm), float(E_eV), int(seed), C.byref(r)))
    return _chem_result(r, r.chem_n, log)


GRID_LABELS = ("t=0", "1 ps", "10 ps", "100 ps", "1 ns", "10 ns", "100 ns", "1 μs")
GRID_T_NS = (0.0, 0.001, 0.01, 0.1, 1.0, 10.0, 100.0, 1000.0)


def run_chemistry_grid(ctx, n_therm, E_eV, rad_buf=None, rad_n=None, seed=1, log=None):
    """runChemistry of the 'gpu' backend (src/chemistry/schedule.ts:48-247): the
    grid-hash diffusion-reaction schedule on the device rad_buf of the last
    transport (or on a host rad_buf), with the final radical positions and
    alive flags that scoreIndirectSSB consumes."""
    L = _lib.lib()
    r = _lib.ChemGridResult()
    if rad_buf is not None:
        rad = np.ascontiguousarray(np.asarray(rad_buf, dtype=np.float32).reshape(-1, 4)[: int(rad_n)])
        n_all = rad.shape[0]
        src = _lib.ptr(rad)
    else:
        rad, n_all, src = None, 0, None
    cap = min(n_all if rad is not None else int(rad_n or 8_000_000), 8_000_000)
    # sizes are known after the call; ask for positions with a buffer of the cap
    k = C.c_uint64()
    pos = np.zeros((cap, 4), np.float32) if cap else np.zeros((1, 4), np.float32)
    alive = np.zeros(max(cap, 1), np.uint32)
    t0 = time.perf_counter()
    _lib.check("wgdna_chem_grid", L.wgdna_chem_grid(ctx.h, src, n_all, int(n_therm), float(E_eV), int(seed),
                                                    C.byref(r), _lib.ptr(pos), _lib.ptr(alive), pos.shape[0]))
    n = int(r.chem_n)
    timeline = []
    for kk in range(8):
        c = r.counts[kk]
        g = r.G[kk]
        timeline.append({"label": GRID_LABELS[kk], "t_ns": GRID_T_NS[kk],
                         "G_OH": g[0], "G_eaq": g[1], "G_H": g[2], "G_H2O2": g[3], "G_H2": g[4],
                         "alive_OH": c[0], "alive_eaq": c[1], "alive_H": c[2], "prod_H2O2": c[3], "prod_H2": c[4]})
    return {"chem_n": n, "t_wall": (time.perf_counter() - t0) * 1000.0, "timeline": timeline,
            "chem_pos_final": pos[:n].reshape(-1), "chem_alive_final": alive[:n], "deposited_eV": r.deposited_eV,
            "ms": r.ms}


runChemistryWorker = run_chemistry_worker
