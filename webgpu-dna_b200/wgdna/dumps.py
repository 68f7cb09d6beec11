"""rad_buf dumps: the reference's on-disk format for a transport's radical
list, ``rad_E{E}_N{np}.bin`` -- raw little-endian float32 records
(x, y, z, pid * 8 + species code), no header (public/geant4dna.html:2234-2256
writes them, tools/dump_server.cjs:38-54 stores them, tools/run_irt.cjs:27-29
and experiments/lib/run-irt.mjs:23-122 read them back for the IRT)."""
import os
import re

import numpy as np

NAME = re.compile(r"rad_E(\d+)_N(\d+)\.bin$")


def dump_name(E_eV, n_primaries):
    return f"rad_E{int(E_eV)}_N{int(n_primaries)}.bin"


def write_rad_dump(directory, E_eV, n_primaries, rad):
    """Write rad (n x 4 float32) as ``rad_E{E}_N{np}.bin``; returns the path."""
    a = np.ascontiguousarray(rad, dtype="<f4").reshape(-1, 4)
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, dump_name(E_eV, n_primaries))
    with open(path, "wb") as f:
        f.write(a.tobytes())
    return path


def read_rad_dump(path):
    """(rad n x 4 float32, E_eV, n_primaries) of a dump; the size must be a
    multiple of 16 bytes (run_irt.cjs reads rad_n = bytes / 16)."""
    size = os.path.getsize(path)
    if size % 16:
        raise ValueError(f"{path}: {size} bytes is not a whole number of 16-byte records")
    rad = np.fromfile(path, dtype="<f4").reshape(-1, 4).astype(np.float32)
    m = NAME.search(os.path.basename(path))
    E, n = (int(m.group(1)), int(m.group(2))) if m else (None, None)
    return rad, E, n


def thermalised_primaries(rad):
    """Primaries present in a dump (the IRT's track count when every primary
    deposited its energy): distinct pid of the records."""
    w = np.rint(np.asarray(rad)[:, 3]).astype(np.int64)
    return int(np.unique(w // 8).size)
