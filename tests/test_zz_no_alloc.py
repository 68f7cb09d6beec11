"""wgdna_score_direct_noalloc: direct SSB scoring for callers that cannot
allocate device memory (GPU test, collected last).

The entry point gets every buffer from the caller and keeps its scratch in a
fixed device array.  It must give exactly what wgdna_score_direct gives (hit
bytes, SSB counts, candidates, in-reach count and the LCG state are integers
or bytes: compared for equality), on two calls in a row, so that the second
call is not disturbed by what the first left in the shared array.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sites(dna, n, seed):
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 4), np.float32)
    i = 0
    while i < n:
        if rng.random() < 0.3:
            f, b, s = rng.integers(dna.n_fibers), rng.integers(dna.n_bp_per), rng.integers(2)
            off = (dna.rbb0 if s == 0 else dna.rbb1)[2 * b: 2 * b + 2]
            x = dna.x0 + b * dna.rise + rng.normal(0, 0.15)
            y, z = dna.fy[f] + off[0] + rng.normal(0, 0.15), dna.fz[f] + off[1] + rng.normal(0, 0.15)
        else:
            x, y, z = rng.uniform(-1600, 1600, 3)
        for _ in range(2 if rng.random() < 0.4 else 1):
            if i < n:
                out[i] = (x, y, z, float(rng.integers(0, 7)))
                i += 1
    return out


def test_noalloc_matches_score_direct_twice():
    import torch

    import wgdna
    from wgdna import _lib

    L = _lib.lib()
    dna = wgdna.build_dna_target()
    info = _lib.DnaInfo()
    _lib.check("wgdna_build_dna_target",
               L.wgdna_build_dna_target(dna.L_nm, dna.grid_N, dna.spacing_nm, None, None, None, None, C.byref(info)))
    dev = torch.device("cuda", 0)
    d_fy, d_fz = torch.from_numpy(dna.fy).to(dev), torch.from_numpy(dna.fz).to(dev)
    d_r0, d_r1 = torch.from_numpy(dna.rbb0).to(dev), torch.from_numpy(dna.rbb1).to(dev)
    nh = 2 * dna.n_bp
    ctx = wgdna.Context(max_primaries=64, max_rad=1_000_000, max_sec=100_000)
    try:
        for n, seed, lcg in ((300_000, 31, 0x12345678), (170_001, 32, 0xDEADBEEF)):
            rad = _sites(dna, n, seed)
            # the existing entry point (host buffers, context-owned scratch)
            ref_hits = np.zeros(nh, np.uint8)
            ref = _lib.SsbResult()
            _lib.check("wgdna_score_direct", L.wgdna_score_direct(ctx.h, _lib.ptr(rad), n, lcg, _lib.ptr(ref_hits),
                                                                  C.byref(ref)))
            # the allocation-free one, on caller-owned device buffers
            d_rad = torch.from_numpy(rad).to(dev)
            d_hits = torch.zeros((nh + 3) // 4 * 4, dtype=torch.uint8, device=dev)
            got = _lib.SsbResult()
            stream = torch.cuda.current_stream(dev)
            _lib.check("wgdna_score_direct_noalloc",
                       L.wgdna_score_direct_noalloc(C.c_void_p(d_rad.data_ptr()), n, C.c_void_p(d_fy.data_ptr()),
                                                    C.c_void_p(d_fz.data_ptr()), C.c_void_p(d_r0.data_ptr()),
                                                    C.c_void_p(d_r1.data_ptr()), C.byref(info), lcg,
                                                    C.c_void_p(d_hits.data_ptr()), C.c_void_p(stream.cuda_stream),
                                                    C.byref(got)))
            hits = d_hits.cpu().numpy()[:nh]
            assert (got.ssb, got.ssb0, got.ssb1) == (ref.ssb, ref.ssb0, ref.ssb1)
            assert got.candidates == ref.candidates and got.in_reach == ref.in_reach
            assert got.lcg_state == ref.lcg_state
            np.testing.assert_array_equal(hits, ref_hits)
            assert ref.in_reach > 0 and ref.ssb > 0
    finally:
        ctx.close()


def test_noalloc_rejects_oversized_list():
    import wgdna
    from wgdna import _lib

    L = _lib.lib()
    info = _lib.DnaInfo()
    _lib.check("wgdna_build_dna_target", L.wgdna_build_dna_target(3000.0, 21, 150.0, None, None, None, None,
                                                                  C.byref(info)))
    got = _lib.SsbResult()
    dummy = C.c_void_p(256)          # never dereferenced: the size check comes first
    rc = L.wgdna_score_direct_noalloc(dummy, (1 << 22) + 1, dummy, dummy, dummy, dummy, C.byref(info), 1, dummy,
                                      None, C.byref(got))
    assert rc == -4
    assert b"4194304" in L.wgdna_last_error()
