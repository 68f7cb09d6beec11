"""Autotuner of the launch and scheduling shapes (wgdna_tuning) on the device.

    python -m wgdna.autotune [--np 4096] [--E 10000] [--reps 3] [--out PATH] [--dry-run]

Runs the benchmark's workload (np primaries at E, box +-15 um, cutoff 7.5 eV,
DNA on, Philox seed 0, then the IRT to 1 us) under candidate shapes and keeps,
group by group, the one with the smallest median device time of the kernels
it affects:
  transport  transport_ctas_per_sm x prim_take x (stash_keep, stash_spill) x
             queue_poll, scored by the transport kernel's time;
  IRT        irt_init_blocks_per_sm scored by the pairing kernel's time and
             irt_loop_blocks_per_sm by the event kernel's.
Every candidate must reproduce the first run's results, counters, rad_buf and
IRT counts bit for bit (the shapes move work between warps, never change it);
a candidate that does not is reported and the tuning aborts.  The table is
written to webgpu-dna_b200/data/tuning.txt, which wgdna_create reads.
"""
import argparse
import ctypes as C
import hashlib
import itertools
import json
import os
import statistics
import sys
import time

import numpy as np

from . import _lib
from .dispatch import transport_params
from .geometry import build_dna_target

TRANSPORT_CTAS = (1, 2)
PRIM_TAKE = (1, 2, 4)
STASH = ((16, 32), (8, 16), (4, 8), (0, 4), (0, 0), (24, 40))
QUEUE_POLL = (4, 8, 32)
IRT_INIT = (4, 5, 6, 7)
IRT_LOOP = (1, 2, 3, 4)
FIELDS = ("transport_ctas_per_sm", "prim_take", "stash_keep", "stash_spill", "queue_poll",
          "irt_init_blocks_per_sm", "irt_loop_blocks_per_sm")


def _digest(ctx, st, ir, npr):
    """SHA-256 of the transport's results, canonical rad_buf and counters, and
    (when the IRT ran) of its checkpoint and reaction counts."""
    L = _lib.lib()
    res = np.zeros(npr * 8, np.float32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), None, _lib.ptr(rad), st.rad_n_stored,
                                                       C.byref(n)))
    h = hashlib.sha256()
    parts = [res.view(np.uint32), rad.view(np.uint32), np.array(st.counters[:], np.uint32)]
    if ir is not None:
        parts += [np.array(ir.counts, np.float64), np.array(ir.rxn_counts[:], np.uint64)]
    for a in parts:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def measure(ctx, tune, p, npr, E, reps, want_irt=True):
    """Median kernel times (transport, pairing, events) over reps runs, and the digest of the last."""
    L = _lib.lib()
    ctx.set_tuning(tune)
    st, ir = _lib.TransportStats(), _lib.IrtResult()
    tt, ti, te = [], [], []
    for _ in range(reps):
        _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
        tt.append(st.ms_transport)
        if want_irt:
            _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, E, 1, C.byref(ir)))
            ti.append(ir.ms_pairing)
            te.append(ir.ms_events)
    dig = _digest(ctx, st, ir if want_irt else None, npr)
    med = statistics.median
    return {"transport": med(tt), "pairing": med(ti) if ti else None, "events": med(te) if te else None}, dig


def tune(npr=4096, E=10000.0, reps=3, log=print):
    ctx = _lib.Context(max_primaries=npr, max_rad=max(npr * 1600, 1_000_000), max_sec=max(npr * 250, 100_000))
    try:
        dna = build_dna_target()
        p = transport_params(npr, E, 15000.0, 7.5, dna=dna, seed=0, dna_enable=1)
        base = _lib.Tuning()
        _lib.lib().wgdna_default_tuning(C.byref(base))
        measure(ctx, base, p, npr, E, 1)                                    # warm-up
        t0, ref = measure(ctx, base, p, npr, E, reps)
        _, ref_tr = measure(ctx, base, p, npr, E, 1, want_irt=False)
        log(f"default {base.as_dict()}: {t0}")
        rows = []
        best, best_t = _lib.Tuning.from_buffer_copy(base), t0["transport"]
        for ctas, take, (keep, spill), poll in itertools.product(TRANSPORT_CTAS, PRIM_TAKE, STASH, QUEUE_POLL):
            cand = _lib.Tuning.from_buffer_copy(best)
            cand.transport_ctas_per_sm, cand.prim_take = ctas, take
            cand.stash_keep, cand.stash_spill, cand.queue_poll = keep, spill, poll
            t, dig = measure(ctx, cand, p, npr, E, reps, want_irt=False)
            rows.append({**cand.as_dict(), "transport_ms": round(t["transport"], 4)})
            if dig != ref_tr:
                raise RuntimeError(f"results changed under {cand.as_dict()}")
            if t["transport"] < best_t:
                best, best_t = cand, t["transport"]
        log(f"transport: best {best.as_dict()} {best_t:.3f} ms (default {t0['transport']:.3f} ms)")
        bi = {"pairing": t0["pairing"], "events": t0["events"]}
        for init in IRT_INIT:
            cand = _lib.Tuning.from_buffer_copy(best)
            cand.irt_init_blocks_per_sm = init
            t, dig = measure(ctx, cand, p, npr, E, reps)
            rows.append({**cand.as_dict(), "pairing_ms": round(t["pairing"], 4)})
            if dig != ref:
                raise RuntimeError(f"results changed under {cand.as_dict()}")
            if t["pairing"] < bi["pairing"]:
                best, bi["pairing"] = cand, t["pairing"]
        for loop in IRT_LOOP:
            cand = _lib.Tuning.from_buffer_copy(best)
            cand.irt_loop_blocks_per_sm = loop
            t, dig = measure(ctx, cand, p, npr, E, reps)
            rows.append({**cand.as_dict(), "events_ms": round(t["events"], 4)})
            if dig != ref:
                raise RuntimeError(f"results changed under {cand.as_dict()}")
            if t["events"] < bi["events"]:
                best, bi["events"] = cand, t["events"]
        t1, dig = measure(ctx, best, p, npr, E, reps)
        if dig != ref:
            raise RuntimeError(f"results changed under {best.as_dict()}")
        log(f"chosen {best.as_dict()}: {t1} (default {t0})")
        return best, {"default": t0, "chosen": t1, "rows": rows}
    finally:
        ctx.close()


def write_table(t, path, summary, device_name):
    with open(path, "w") as f:
        f.write(f"# wgdna_tuning for {device_name}, written by python -m wgdna.autotune\n")
        f.write(f"# workload: 4096 x 10 keV transport + IRT; kernel ms default {json.dumps(summary['default'])}\n")
        f.write(f"# chosen {json.dumps(summary['chosen'])}\n")
        for k in FIELDS:
            f.write(f"{k} {int(getattr(t, k))}\n")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--np", type=int, default=4096)
    ap.add_argument("--E", type=float, default=10000.0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(_lib.LIB_PATH), "data", "tuning.txt"))
    ap.add_argument("--rows", default=None, help="also write every candidate's times as JSON here")
    ap.add_argument("--dry-run", action="store_true", help="do not write the table")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    best, summary = tune(a.np, a.E, a.reps)
    try:
        import torch
        name = torch.cuda.get_device_name(0)
    except Exception:
        name = "the current device"
    if not a.dry_run:
        write_table(best, a.out, summary, name)
        print(f"wrote {a.out}")
    if a.rows:
        with open(a.rows, "w") as f:
            json.dump(summary, f, indent=1)
    print(f"tuned in {time.perf_counter() - t0:.1f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
