"""Cross-section tables: bit-identical to public/cross_sections.wgsl, plus the
assertions of the reference's tests/unit/cross-sections.test.ts:27-101."""
import hashlib
import json
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG

DATA = os.path.join(PKG, "data")


def load_blob():
    b = open(os.path.join(DATA, "cross_sections.bin"), "rb").read()
    assert b[:8] == b"WGDNAXS1"
    n, dbytes = struct.unpack("<II", b[8:16])
    hsz = (16 + 40 * n + 15) & ~15
    assert hsz + dbytes == len(b)
    out = {}
    for i in range(n):
        name, dtype, count, off, _ = struct.unpack("<24sIIII", b[16 + 40 * i: 56 + 40 * i])
        name = name.rstrip(b"\0").decode()
        dt = "<u4" if dtype else "<f4"
        out[name] = np.frombuffer(b, dtype=dt, count=count, offset=hsz + off)
    return out, b


T, BLOB = load_blob()
MAN = json.load(open(os.path.join(DATA, "cross_sections.json")))


def test_blob_matches_manifest():
    assert hashlib.sha256(BLOB).hexdigest() == MAN["blob_sha256"]
    assert set(T) == set(MAN["arrays"])
    for name, a in T.items():
        m = MAN["arrays"][name]
        assert a.size == m["count"]
        assert hashlib.sha256(a.tobytes()).hexdigest() == m["sha256"], name


def test_table_inventory():
    """31 f32 arrays (147,535 floats) and 12 scalar constants."""
    arrays = {k: v for k, v in T.items() if v.size > 1}
    assert len(arrays) == 31
    assert sum(v.size for v in arrays.values()) == 147_535
    assert int(T["XN"][0]) == 100 and int(T["N_WE"][0]) == 58 and int(T["N_WR"][0]) == 250
    assert int(T["N_AE"][0]) == 25 and int(T["N_AC"][0]) == 25 and int(T["N_VIB"][0]) == 38


def _wgsl_source():
    sys.path.insert(0, DATA)
    import gen_tables
    return gen_tables.DEFAULT_SRC


@pytest.mark.skipif(not (_wgsl_source() and os.path.exists(_wgsl_source())),
                    reason="reference checkout not given (WGDNA_REFERENCE)")
def test_blob_regenerates_bit_identical(tmp_path):
    """Re-parse the reference's WGSL and compare every array bit for bit."""
    import gen_tables
    text = open(_wgsl_source()).read()
    arrays = gen_tables.parse_wgsl(text)
    assert gen_tables.build_blob(arrays) == BLOB
    for name, a in arrays:
        np.testing.assert_array_equal(a.view(np.uint32), T[name].view(np.uint32))


def interp(E):
    """cross-sections.test.ts:27-33 (log grid from XE itself, f64)."""
    XE, XN = T["XE"].astype(np.float64), 100
    L0 = np.log(XE[0])
    step = (np.log(XE[XN - 1]) - L0) / (XN - 1)
    t = (np.log(E) - L0) / step
    i = int(min(max(np.floor(t), 0), XN - 2))
    f = t - i
    g = lambda a: max(0.0, float(a[i]) + (float(a[i + 1]) - float(a[i])) * f)
    return g(T["XI"]), g(T["XC"]), g(T["XL"])


G4_REF = {100: (0.024, 0.053), 300: (0.016, 0.028), 1000: (0.007, 0.012), 5000: (0.002, 0.003),
          10000: (0.001144, 0.001780)}


def test_reference_cross_section_assertions():
    XE = T["XE"]
    assert XE.size == 100 and T["XI"].size == 100 and T["XC"].size == 100 and T["XL"].size == 100
    assert round(float(XE[0])) == 8 and 10000 < XE[-1] < 50000
    assert interp(9)[0] == 0
    assert interp(100)[0] > interp(50)[0] and interp(100)[0] > interp(500)[0]
    for E, (ion, tot) in G4_REF.items():
        xi, xc, xl = interp(E)
        assert 0.85 < xi / ion < 1.15, E
        assert 0.80 < (xi + xc + xl) / tot < 1.20, E
    xi, xc, xl = interp(20)
    assert xl > xi and xl > xc
    xi, xc, xl = interp(500)
    assert xi > xl and xi > xc


def test_born_cdf_rows_are_monotone():
    """The CUDA path replaces the reference's linear CDF scan (helpers.wgsl:98-105)
    by a binary search; the two give the same breakpoint iff every row is
    non-decreasing."""
    for k in range(5):
        c = T[f"XWC{k}"].reshape(58, 250)
        assert (np.diff(c, axis=1) >= 0).all(), k


def test_grids_sorted_and_xef_quirk():
    for name in ("XE", "XWE", "XVE", "XAE"):
        assert (np.diff(T[name]) > 0).all(), name
    s = sum(T[f"XEF{k}"] for k in range(5))
    # helpers.wgsl:46-49: XEF rows past index 85 are corrupt (sum 5); the
    # kernels clamp to index 85 like the reference
    assert np.allclose(s[8:86], 1.0, atol=1e-4) and np.allclose(s[86:], 5.0)
    assert (s[1:8] > 0.9).all() and (s[1:8] <= 1.0 + 1e-6).all()
