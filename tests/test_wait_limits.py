"""Failure detection on the device without a GPU fault (GPU tests).

Every device-side wait of the path is bounded; a wait that runs out sets a bit
of the stage's error word, the entry point returns WGDNA_ERR_DEVICE, and the
context stays usable.  The bounds are shortened through
wgdna_set_wait_limits, and the waits are made to run out on flags that
nothing sets:
  * idle bound of a transport warp (bit 1): 1 us, while most warps of the grid
    have no primary to run;
  * queue wait of a transport lane (bit 0): 1 ms, with the secondaries
    published under an epoch that no consumer waits for;
  * tensor-core wait of a surrogate tile (SG_ERR_WAIT, bit 6): each tile gives
    up its first wait before polling, then waits for the tensor cores to finish
    before it reads or frees tensor memory.
After each, the same context runs a normal call whose results are the oracle's
(transport) or the earlier prediction's (surrogate), bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import wgdna
from wgdna import _lib

pytestmark = pytest.mark.gpu

DERR_QUEUE_WAIT, DERR_IDLE_WAIT, SG_ERR_WAIT = 1, 2, 1 << 6


def _transport(ctx, np_, seed):
    p = wgdna.transport_params(np_, 10000.0, 15000.0, 7.5, seed=seed, dna_enable=0)
    st = _lib.TransportStats()
    rc = _lib.lib().wgdna_transport(ctx.h, C.byref(p), C.byref(st))
    return rc, st


def _normal_run_is_exact(ctx):
    L = _lib.lib()
    _lib.check("wgdna_set_wait_limits", L.wgdna_set_wait_limits(ctx.h, 0, 0, 0, 0))
    rc, st = _transport(ctx, 32, 9)
    assert rc == _lib.WGDNA_OK and st.device_error == 0
    res = np.zeros(32 * 8, np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), None, None, 0, C.byref(n)))
    o = oracle.transport(32, 10000.0, seed=9, rng_mode=0, dna_enable=0, want_dose=False)
    np.testing.assert_array_equal(res.view(np.uint32), o["results"].view(np.uint32))


@pytest.fixture()
def wctx():
    c = wgdna.Context(max_primaries=1024, max_rad=4_000_000, max_sec=400_000)
    yield c
    c.close()


def test_transport_idle_bound_runs_out(wctx):
    L = _lib.lib()
    _lib.check("wgdna_set_wait_limits", L.wgdna_set_wait_limits(wctx.h, 0, 1000, 0, 0))
    rc, st = _transport(wctx, 64, 3)
    assert rc == _lib.WGDNA_ERR_DEVICE
    assert st.device_error & DERR_IDLE_WAIT
    assert b"device error" in L.wgdna_last_error()
    _normal_run_is_exact(wctx)


def test_transport_queue_wait_runs_out(wctx):
    L = _lib.lib()
    _lib.check("wgdna_set_wait_limits",
               L.wgdna_set_wait_limits(wctx.h, 1_000_000, 0, 0, _lib.WGDNA_TEST_UNPUBLISHED))
    rc, st = _transport(wctx, 512, 4)
    assert rc == _lib.WGDNA_ERR_DEVICE
    assert st.device_error & DERR_QUEUE_WAIT
    _normal_run_is_exact(wctx)


def test_surrogate_tensor_core_wait_runs_out(wctx):
    L = _lib.lib()
    _lib.check("wgdna_surrogate_init", L.wgdna_surrogate_init(wctx.h, 3))
    X = np.random.default_rng(1).normal(size=(300, _lib.SG_IN)).astype(np.float32)
    G0 = np.zeros((300, _lib.SG_OUT), np.float32)
    _lib.check("wgdna_surrogate_predict", L.wgdna_surrogate_predict(wctx.h, _lib.ptr(X), 300, _lib.ptr(G0)))
    _lib.check("wgdna_set_wait_limits", L.wgdna_set_wait_limits(wctx.h, 0, 0, 0, _lib.WGDNA_TEST_MMA_WAIT))
    G1 = np.zeros_like(G0)
    rc = L.wgdna_surrogate_predict(wctx.h, _lib.ptr(X), 300, _lib.ptr(G1))
    assert rc == _lib.WGDNA_ERR_DEVICE
    assert b"0x40" in L.wgdna_last_error()
    _lib.check("wgdna_set_wait_limits", L.wgdna_set_wait_limits(wctx.h, 0, 0, 0, 0))
    G2 = np.zeros_like(G0)
    _lib.check("wgdna_surrogate_predict", L.wgdna_surrogate_predict(wctx.h, _lib.ptr(X), 300, _lib.ptr(G2)))
    np.testing.assert_array_equal(G2, G0)
    _normal_run_is_exact(wctx)


def test_wait_limits_reject_unknown_test_flags(wctx):
    assert _lib.lib().wgdna_set_wait_limits(wctx.h, 0, 0, 0, 1 << 7) == _lib.WGDNA_ERR_ARG
