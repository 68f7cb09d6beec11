#!/usr/bin/env python3
"""Generate ``cross_sections.bin`` and ``cross_sections.json`` from the
reference's WGSL cross-section table file.

Source: ``public/cross_sections.wgsl:9-72`` of allaunthefox/webgpu-dna. Every
``const NAME=array<f32,N>(...)`` literal list becomes one float32 array and
every scalar ``const NAME=<number>[u];`` becomes a one-element array (u32 when
the literal carries the ``u`` suffix, float32 otherwise).  Decimal literals are
rounded to float32 with correct round-to-nearest-even, which is what a WGSL
compiler does for an abstract-float literal used as f32 (and, for this file,
is bit-identical to the decimal -> f64 -> f32 route the reference's own unit
tests take; the generator checks that too).

Blob layout (little endian), read by ``webgpu-dna_b200/csrc/tables.cu`` and by
the oracle's loader:

    char     magic[8]   = "WGDNAXS1"
    uint32   n_entries
    uint32   data_bytes
    entry[n_entries]:   char name[24]; uint32 dtype (0=f32, 1=u32);
                        uint32 count; uint32 offset (bytes from data start);
                        uint32 reserved
    data                every array 16-byte aligned

The JSON manifest records count, dtype and SHA-256 of every array so that the
blob can be checked without the WGSL file.

Usage:  python gen_tables.py [path/to/cross_sections.wgsl]
"""
import ctypes
import hashlib
import json
import os
import re
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's table source: WGDNA_REFERENCE_WGSL, else public/cross_sections.wgsl
# under the checkout named by WGDNA_REFERENCE, else the command-line argument
DEFAULT_SRC = os.environ.get("WGDNA_REFERENCE_WGSL") or (
    os.path.join(os.environ["WGDNA_REFERENCE"], "public", "cross_sections.wgsl")
    if os.environ.get("WGDNA_REFERENCE") else None)
MAGIC = b"WGDNAXS1"
ENTRY_FMT = "<24sIIII"


def _strtof():
    libc = ctypes.CDLL("libc.so.6")
    f = libc.strtof
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return f


def parse_wgsl(text):
    """Return an ordered list of (name, numpy array) in file order."""
    strtof = _strtof()
    out = []
    pat = re.compile(
        r"const (\w+)=(?:array<f32,(\d+)>\(([^)]*)\)|([0-9.eE+-]+)(u?));")
    for m in pat.finditer(text):
        name = m.group(1)
        if m.group(2) is not None:
            toks = [t.strip() for t in m.group(3).split(",")]
            if len(toks) != int(m.group(2)):
                raise ValueError(f"{name}: {len(toks)} literals, declared {m.group(2)}")
            direct = np.array([strtof(t.encode(), None) for t in toks], dtype=np.float32)
            via64 = np.array([float(t) for t in toks], dtype=np.float64).astype(np.float32)
            if not np.array_equal(direct.view(np.uint32), via64.view(np.uint32)):
                raise ValueError(f"{name}: decimal rounding is ambiguous")
            out.append((name, direct))
        else:
            lit, usuf = m.group(4), m.group(5)
            if usuf:
                out.append((name, np.array([int(lit)], dtype=np.uint32)))
            else:
                out.append((name, np.array([strtof(lit.encode(), None)], dtype=np.float32)))
    return out


def build_blob(arrays):
    entries = []
    data = bytearray()
    for name, arr in arrays:
        while len(data) % 16:
            data.append(0)
        dtype = 1 if arr.dtype == np.uint32 else 0
        entries.append((name, dtype, arr.size, len(data)))
        data += arr.astype("<u4" if dtype else "<f4").tobytes()
    while len(data) % 16:
        data.append(0)
    head = MAGIC + struct.pack("<II", len(entries), len(data))
    for name, dtype, count, off in entries:
        head += struct.pack(ENTRY_FMT, name.encode().ljust(24, b"\0"), dtype, count, off, 0)
    while len(head) % 16:
        head += b"\0"
    return head + bytes(data)


def manifest(arrays):
    m = {}
    for name, arr in arrays:
        raw = arr.astype("<u4" if arr.dtype == np.uint32 else "<f4").tobytes()
        m[name] = {"dtype": "u32" if arr.dtype == np.uint32 else "f32",
                   "count": int(arr.size), "sha256": hashlib.sha256(raw).hexdigest()}
    return m


def main(argv):
    src = argv[1] if len(argv) > 1 else DEFAULT_SRC
    if not src:
        sys.exit("usage: gen_tables.py <reference>/public/cross_sections.wgsl "
                 "(or set WGDNA_REFERENCE to the reference checkout)")
    with open(src) as f:
        arrays = parse_wgsl(f.read())
    blob = build_blob(arrays)
    with open(os.path.join(HERE, "cross_sections.bin"), "wb") as f:
        f.write(blob)
    man = {"source": "public/cross_sections.wgsl", "arrays": manifest(arrays),
           "blob_sha256": hashlib.sha256(blob).hexdigest(), "blob_bytes": len(blob)}
    with open(os.path.join(HERE, "cross_sections.json"), "w") as f:
        json.dump(man, f, indent=1, sort_keys=True)
    nfl = sum(a.size for n, a in arrays if a.size > 1)
    print(f"{len(arrays)} entries, {nfl} table floats, blob {len(blob)} bytes")


if __name__ == "__main__":
    main(sys.argv)
