"""The device side of a sharded run (wgdna.sharded.device_step_exchange) on
one GPU with a one-rank NCCL group: the exchange path (views of the
library's buffers as torch tensors, the two scoring passes, the MAX-reduced
hits, clustering on the device) must reproduce the single-device step.  The
protocol itself is checked with two ranks on CPU in test_multirank.py."""
import ctypes as C
import datetime
import socket

import numpy as np
import pytest

import wgdna
from wgdna import _lib, sharded


@pytest.mark.gpu
def test_device_exchange_matches_single_device(ctx):
    import torch
    import torch.distributed as dist
    s = socket.socket(); s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]; s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dev = torch.device("cuda", 0)
        L = _lib.lib()
        p = wgdna.transport_params(256, 10000.0, 15000.0, 7.5, dna=wgdna.build_dna_target(), seed=4, dna_enable=1)
        st = _lib.TransportStats()
        _lib.check("t", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
        ssb, dsb = _lib.SsbResult(), _lib.DsbResult()
        _lib.check("score", L.wgdna_score(ctx.h, 0x12345678, C.byref(ssb), C.byref(dsb)))
        dose0 = np.zeros(ctx.vc ** 3, np.uint32)
        n = C.c_uint64()
        _lib.check("copy", L.wgdna_transport_copy_out(ctx.h, None, _lib.ptr(dose0), None, 0, C.byref(n)))
        got = sharded.device_step_exchange(ctx, dist, 0x12345678, dev, irt_counts=np.arange(5.0))
        assert got[0] == ssb.ssb and got[1] == dsb.dsb and got[2] == ssb.in_reach
        np.testing.assert_array_equal(got[3], np.arange(5.0))
        dose1 = np.zeros_like(dose0)
        _lib.check("copy", L.wgdna_transport_copy_out(ctx.h, None, _lib.ptr(dose1), None, 0, C.byref(n)))
        np.testing.assert_array_equal(dose0, dose1)
    finally:
        dist.destroy_process_group()
