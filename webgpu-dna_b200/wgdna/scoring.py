"""SSB / DSB scoring (src/scoring/ssb-dsb.ts) on the GPU through the C ABI."""
import ctypes as C

import numpy as np

from . import _lib
from .constants import SPECIES


class SsbRng:
    """makeSsbRng (ssb-dsb.ts:421-427): LCG s = 1664525 s + 1013904223 mod 2^32,
    returning s / 2^32.  The GPU scoring passes advance ``state`` by the number
    of draws they made, exactly as the sequential reference loop would."""

    def __init__(self, seed=0x12345678):
        self.state = seed & 0xFFFFFFFF

    def __call__(self):
        self.state = (self.state * 1664525 + 1013904223) & 0xFFFFFFFF
        return self.state / 4294967296.0


def make_ssb_rng(seed=0x12345678):
    return SsbRng(seed)


def _use_target(ctx, dna):
    if getattr(ctx, "_dna_key", None) != dna.key:
        _lib.check("wgdna_set_dna_target",
                   _lib.lib().wgdna_set_dna_target(ctx.h, float(dna.L_nm), int(dna.grid_N), float(dna.spacing_nm)))
        ctx._dna_key = dna.key


def score_direct_ssb_events(ctx, dna, rad_buf, rad_n, rng):
    """scoreDirectSSB_events: direct SSBs from rad_buf sites (ssb-dsb.ts:135-217)."""
    _use_target(ctx, dna)
    rad = np.ascontiguousarray(np.asarray(rad_buf, dtype=np.float32).reshape(-1)[: 4 * rad_n])
    hits = np.zeros(2 * dna.n_bp, np.uint8)
    r = _lib.SsbResult()
    _lib.check("wgdna_score_direct", _lib.lib().wgdna_score_direct(ctx.h, _lib.ptr(rad), int(rad_n), rng.state,
                                                                  _lib.ptr(hits), C.byref(r)))
    rng.state = r.lcg_state
    return {"hits": hits, "ssb_count": r.ssb, "candidates": r.candidates, "in_reach": r.in_reach,
            "ms": r.ms}


def score_indirect_ssb(ctx, dna, chem_pos_final, chem_alive_final, chem_n, rng):
    """scoreIndirectSSB: OH alive at 1 us near a backbone (ssb-dsb.ts:43-121)."""
    _use_target(ctx, dna)
    pos = np.ascontiguousarray(np.asarray(chem_pos_final, dtype=np.float32).reshape(-1)[: 4 * chem_n])
    alive = np.ascontiguousarray(np.asarray(chem_alive_final, dtype=np.uint32)[:chem_n])
    hits = np.zeros(2 * dna.n_bp, np.uint8)
    r = _lib.SsbResult()
    _lib.check("wgdna_score_indirect",
               _lib.lib().wgdna_score_indirect(ctx.h, _lib.ptr(pos), _lib.ptr(alive), int(chem_n), rng.state,
                                               _lib.ptr(hits), C.byref(r)))
    rng.state = r.lcg_state
    return {"hits": hits, "ssb0": r.ssb0, "ssb1": r.ssb1, "candidates": r.candidates, "in_reach": r.in_reach}


def cluster_dsb(ctx, dna, hits):
    """clusterDSB: greedy +-10 bp pairing per fibre (ssb-dsb.ts:348-407)."""
    _use_target(ctx, dna)
    h = np.ascontiguousarray(np.asarray(hits, dtype=np.uint8))
    if h.size != 2 * dna.n_bp:
        raise ValueError(f"hits must have 2*n_bp = {2 * dna.n_bp} bytes")
    r = _lib.DsbResult()
    _lib.check("wgdna_cluster_dsb", _lib.lib().wgdna_cluster_dsb(ctx.h, _lib.ptr(h), C.byref(r)))
    return {"dsb": r.dsb, "dsb_expected": r.dsb_expected, "ssb0": r.ssb0, "ssb1": r.ssb1}


def combine_hits(a, b):
    """combineHits (ssb-dsb.ts:413-418)."""
    return ((np.asarray(a, np.uint8) | np.asarray(b, np.uint8)) != 0).astype(np.uint8)


makeSsbRng = make_ssb_rng
scoreDirectSSB_events = score_direct_ssb_events
scoreIndirectSSB = score_indirect_ssb
clusterDSB = cluster_dsb
combineHits = combine_hits
OH_CODE = SPECIES["OH"]
