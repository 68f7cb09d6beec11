"""The C ABI without a GPU: the library loads, exports every declared entry
point, and fails cleanly where a device is needed."""
import ctypes as C
import os
import re

import numpy as np

import oracle
from conftest import ROOT, has_gpu

import wgdna
from wgdna import _lib


def declared():
    text = open(os.path.join(ROOT, "include", "wgdna.h")).read()
    return sorted(set(re.findall(r"\b(wgdna_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTS) == names


def test_version_and_default_cfg():
    L = _lib.lib()
    assert L.wgdna_version() >= 10000
    cfg = _lib.Cfg()
    L.wgdna_default_cfg(C.byref(cfg))
    assert (cfg.max_primaries, cfg.max_sec, cfg.max_rad, cfg.vc) == (4096, 5_000_000, 16_000_000, 128)


def test_create_without_device_fails_cleanly():
    if has_gpu():
        return
    L = _lib.lib()
    h = C.c_void_p()
    rc = L.wgdna_create(None, C.byref(h))
    assert rc != 0 and not h.value
    assert L.wgdna_last_error()


def test_argument_errors():
    L = _lib.lib()
    info = _lib.DnaInfo()
    assert L.wgdna_build_dna_target(0.0, 21, 150.0, None, None, None, None, C.byref(info)) == -1
    assert b"invalid geometry" in L.wgdna_last_error()
    assert L.wgdna_create(None, None) == -1
    cfg = _lib.Cfg()
    L.wgdna_default_cfg(C.byref(cfg))
    cfg.max_primaries = 3_000_000
    h = C.c_void_p()
    assert L.wgdna_create(C.byref(cfg), C.byref(h)) == -1
    assert L.wgdna_reaction_table(None) == -1


def test_reaction_table_equals_oracle():
    np.testing.assert_array_equal(_lib.reaction_table(), oracle.irt_rxn_table())


def test_host_surface():
    from wgdna import constants as K
    assert len(wgdna.ESTAR) == 8 and wgdna.find_estar(10000)["csda"] == 2515
    rng = wgdna.make_ssb_rng()
    v = rng()
    assert 0 <= v < 1 and rng.state == (0x12345678 * 1664525 + 1013904223) % 2 ** 32
    a = np.array([0, 1, 0, 1], np.uint8)
    b = np.array([0, 0, 1, 1], np.uint8)
    np.testing.assert_array_equal(wgdna.combine_hits(a, b), [0, 1, 1, 1])
    assert K.MAX_SEC_STEPS == 2000 and K.VC == 128
    p = wgdna.transport_params(4096, 10000.0, 15000.0, 7.4, dna=wgdna.build_dna_target())
    assert p.dna_enable == 1 and p.seed == 10000 and p.max_steps == 65536
    p = wgdna.transport_params(4096, 3000.0, 15000.0, 7.4, dna=wgdna.build_dna_target())
    assert p.dna_enable == 0
