"""Launch and scheduling shapes (wgdna_tuning) move work between warps and
blocks but never change it: every particle, pair and track draws from its own
Philox stream.  The GPU test runs one workload under the default shapes and
under extreme ones and compares everything bit for bit."""
import ctypes as C

import numpy as np
import pytest

import wgdna
from wgdna import _lib


def test_default_tuning_values():
    t = _lib.Tuning()
    _lib.lib().wgdna_default_tuning(C.byref(t))
    assert t.as_dict() == {"transport_ctas_per_sm": 0, "prim_take": 2, "stash_keep": 16, "stash_spill": 32,
                           "queue_poll": 8, "irt_init_blocks_per_sm": 0, "irt_loop_blocks_per_sm": 0}


def _run(ctx):
    L = _lib.lib()
    p = wgdna.transport_params(512, 10000.0, 15000.0, 7.5, seed=21, dna_enable=1, dna=wgdna.build_dna_target())
    st = _lib.TransportStats()
    _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    res = np.zeros(512 * 8, np.float32)
    dose = np.zeros(ctx.vc ** 3, np.uint32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), _lib.ptr(dose), _lib.ptr(rad),
                                                       st.rad_n_stored, C.byref(n)))
    ir = _lib.IrtResult()
    _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, 10000.0, 3, C.byref(ir)))
    return st, res, dose, rad, ir


@pytest.mark.gpu
def test_results_do_not_depend_on_the_shapes(ctx):
    keep = ctx.tuning()
    try:
        a = _run(ctx)
        for fields in ({"transport_ctas_per_sm": 1, "prim_take": 32, "stash_keep": 0, "stash_spill": 0,
                        "queue_poll": 1, "irt_init_blocks_per_sm": 2, "irt_loop_blocks_per_sm": 1},
                       {"transport_ctas_per_sm": 2, "prim_take": 1, "stash_keep": 24, "stash_spill": 40,
                        "queue_poll": 32, "irt_init_blocks_per_sm": 3, "irt_loop_blocks_per_sm": 2}):
            ctx.set_tuning(**fields)
            assert ctx.tuning().as_dict() == {**keep.as_dict(), **fields}
            b = _run(ctx)
            np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
            np.testing.assert_array_equal(a[2], b[2])
            np.testing.assert_array_equal(a[3].view(np.uint32), b[3].view(np.uint32))
            assert list(a[0].counters) == list(b[0].counters) and a[0].steps == b[0].steps
            np.testing.assert_array_equal(np.array(a[4].counts), np.array(b[4].counts))
            assert (a[4].n_pairs, a[4].n_events) == (b[4].n_pairs, b[4].n_events)
        with pytest.raises(_lib.WgdnaError):
            ctx.set_tuning(stash_keep=40, stash_spill=32)
    finally:
        ctx.set_tuning(keep)
