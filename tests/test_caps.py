"""Capacity caps: overflows are counted, not errors (dispatch.ts:124-126,
190-192; primary.wgsl:253-364).  GPU tests against the oracle.

rad_buf cap (max_rad): storage only.  The physics is that of the uncapped run
(results, counters, dose grid, step count bit for bit with the oracle); the
first max_rad entries to reach the buffer are kept, rad_dropped counts the rest,
and the kept entries are a sub-multiset of the oracle's full list.  (Here each
entry is stored while a slot is free; the reference stores an event's 2-3
entries only when all of them fit, so its last one or two slots can stay
unwritten.)

Secondary cap (max_sec): every emission takes a sec_buf index; at or beyond
max_sec the secondary is dropped together with its angle draws and the
primary's momentum update, as in the reference.  Which emissions come last
depends on the order the primaries run in (all at once on the GPU, like the
reference's one thread per primary; primary by primary in the oracle), so the
counting is compared exactly and the rest as bounds.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import wgdna
from wgdna import _lib

pytestmark = pytest.mark.gpu


def _run(ctx, np_, E, seed):
    p = wgdna.transport_params(np_, E, 15000.0, 7.5, seed=seed, dna_enable=0)
    st = _lib.TransportStats()
    L = _lib.lib()
    _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    res = np.zeros(np_ * 8, np.float32)
    dose = np.zeros(ctx.vc ** 3, np.uint32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), _lib.ptr(dose), _lib.ptr(rad),
                                                       st.rad_n_stored, C.byref(n)))
    return st, res, dose, rad


def _rows(a):
    v = np.ascontiguousarray(a, np.float32).view(np.uint32).reshape(-1, 4)
    u, c = np.unique(v, axis=0, return_counts=True)
    return {tuple(r): k for r, k in zip(u.tolist(), c.tolist())}


def test_rad_buf_cap_counts_drops_and_keeps_the_physics():
    cap = 50_000
    ctx = wgdna.Context(max_primaries=64, max_rad=cap, max_sec=200_000)
    try:
        st, res, dose, rad = _run(ctx, 64, 10000.0, 17)
        o = oracle.transport(64, 10000.0, seed=17, rng_mode=0, dna_enable=0)
        raw = o["rad"].shape[0]
        assert raw > cap
        assert st.device_error == 0
        assert (st.rad_n_raw, st.rad_n_stored, st.rad_dropped) == (raw, cap, raw - cap)
        assert st.counters[7] == raw
        np.testing.assert_array_equal(res.view(np.uint32), o["results"].view(np.uint32))
        np.testing.assert_array_equal(np.array(st.counters[:7]), o["counters"][:7])
        np.testing.assert_array_equal(dose, o["dose"])
        assert st.steps == o["steps"] and st.sec_dropped == 0
        full, kept = _rows(o["rad"]), _rows(rad)
        assert sum(kept.values()) == cap
        assert all(full.get(r, 0) >= k for r, k in kept.items())
        # the stages after the transport run on the kept entries
        ir = _lib.IrtResult()
        _lib.check("wgdna_irt", _lib.lib().wgdna_irt(ctx.h, st.n_therm, 10000.0, 1, C.byref(ir)))
        assert ir.device_error == 0 and ir.n_particles > 0
    finally:
        ctx.close()


def test_secondary_cap_counts_drops_like_the_reference():
    cap = 500
    ctx = wgdna.Context(max_primaries=64, max_rad=2_000_000, max_sec=cap)
    try:
        st, res, dose, rad = _run(ctx, 64, 10000.0, 5)
        assert st.device_error == 0
        assert st.sec_n_raw == st.counters[6] > cap
        assert st.sec_n == cap and st.sec_dropped == st.sec_n_raw - cap
        # processed secondaries end at the cutoff, at the box or at the step cap
        assert st.sec_stats[1] + st.sec_stats[2] <= cap
        # dropped secondaries take their energy with them
        assert st.dep_eV_f64 < 0.9 * 64 * 10000.0
        o = oracle.transport(64, 10000.0, seed=5, rng_mode=0, dna_enable=0, max_sec=cap, nthreads=1)
        assert o["capped"] and o["sec_n"] == cap and o["counters"][6] > cap
        assert o["sec_stats"][1] + o["sec_stats"][2] <= cap
        # the same run without the cap keeps every secondary and is the oracle's bit for bit
        big = wgdna.Context(max_primaries=64, max_rad=2_000_000, max_sec=200_000)
        try:
            st2, res2, _, _ = _run(big, 64, 10000.0, 5)
            o2 = oracle.transport(64, 10000.0, seed=5, rng_mode=0, dna_enable=0)
            assert st2.sec_dropped == 0 and st2.sec_n == st2.sec_n_raw == o2["counters"][6]
            np.testing.assert_array_equal(res2.view(np.uint32), o2["results"].view(np.uint32))
        finally:
            big.close()
    finally:
        ctx.close()
