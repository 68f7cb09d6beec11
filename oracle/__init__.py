"""CPU oracle of the transport -> IRT -> scoring path (ctypes binding).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this package, and only as the checker or
as the timed CPU baseline; the product path (``webgpu-dna_b200``) never calls
it.  The C sources beside this file restate the reference's algorithms (file
and line citations in each source); ``Makefile`` builds ``liboracle.so``.

Parity status: tables pinned bit for bit; geometry, constants, rad_buf
encoding and the IRT smoke case pinned by the reference's own unit tests;
transport / IRT statistics pinned against the reference's published 10 keV
outputs within statistical error (the reference's WebGPU shaders and JS worker
cannot run here).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BLOB = os.path.join(ROOT, "webgpu-dna_b200", "data", "cross_sections.bin")
_LIB = None


class TransportParams(C.Structure):
    _fields_ = [("np", C.c_uint32), ("box_nm", C.c_float), ("ce_eV", C.c_float),
                ("max_steps", C.c_uint32), ("E_eV", C.c_float), ("max_sec", C.c_uint32),
                ("vc", C.c_uint32), ("max_rad", C.c_uint32), ("start_half", C.c_float),
                ("dna_enable", C.c_uint32), ("dna_grid_n", C.c_uint32),
                ("dna_rise", C.c_float), ("dna_spacing", C.c_float), ("dna_x0", C.c_float),
                ("dna_r_bb", C.c_float), ("sec_steps", C.c_uint32), ("rng_mode", C.c_uint32),
                ("seed", C.c_uint64), ("pid_base", C.c_uint32), ("E_per_primary", C.c_void_p)]


class TransportOut(C.Structure):
    _fields_ = [("results", C.POINTER(C.c_float)), ("dose", C.POINTER(C.c_uint32)),
                ("counters", C.c_uint32 * 8), ("sec_stats", C.c_uint32 * 8), ("dbg", C.c_uint32 * 8),
                ("rad", C.POINTER(C.c_float)), ("rad_key", C.POINTER(C.c_uint64)),
                ("rad_n", C.c_uint64), ("dep_units", C.c_uint64), ("dep_eV_f64", C.c_double),
                ("sec_n", C.c_uint64), ("steps", C.c_uint64)]


class IrtOut(C.Structure):
    _fields_ = [("tl", (C.c_double * 5) * 7), ("G", (C.c_double * 5) * 7),
                ("rxn_counts", C.c_uint64 * 9), ("n_reacted", C.c_uint64),
                ("n_pairs", C.c_uint64), ("n_tracks", C.c_uint64), ("n_events", C.c_uint64),
                ("curves", C.POINTER(C.c_float)), ("curves_cap", C.c_uint64)]


class Dna(C.Structure):
    _fields_ = [("grid_N", C.c_uint32), ("n_bp_per", C.c_uint32), ("n_fibers", C.c_uint32),
                ("n_bp", C.c_uint32), ("rise", C.c_double), ("r_bb", C.c_double),
                ("spacing_nm", C.c_double), ("x0", C.c_double), ("L_nm", C.c_double),
                ("fy", C.POINTER(C.c_float)), ("fz", C.POINTER(C.c_float)),
                ("rbb0", C.POINTER(C.c_float)), ("rbb1", C.POINTER(C.c_float))]


class SsbOut(C.Structure):
    _fields_ = [("ssb", C.c_uint64), ("ssb0", C.c_uint64), ("ssb1", C.c_uint64),
                ("candidates", C.c_uint64), ("in_reach", C.c_uint64), ("lcg_state", C.c_uint32)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.POINTER
        L.orc_load_tables.argtypes = [C.c_char_p]
        L.orc_transport.argtypes = [P(TransportParams), P(TransportOut), C.c_int]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_irt.argtypes = [P(C.c_float), C.c_uint64, C.c_uint32, C.c_double, C.c_uint64,
                              P(IrtOut), C.c_int]
        L.orc_irt_rxn_table.argtypes = [P(C.c_double)]
        L.orc_build_dna.argtypes = [C.c_double, C.c_uint32, C.c_double, P(Dna)]
        L.orc_free_dna.argtypes = [P(Dna)]
        L.orc_score_direct.argtypes = [P(Dna), P(C.c_float), C.c_uint64, C.c_uint32,
                                       P(C.c_uint8), P(SsbOut)]
        L.orc_score_indirect.argtypes = [P(Dna), P(C.c_float), P(C.c_uint32), C.c_uint64,
                                         C.c_uint32, P(C.c_uint8), P(SsbOut)]
        L.orc_cluster_dsb.argtypes = [P(Dna), P(C.c_uint8), P(C.c_uint64), P(C.c_double),
                                      P(C.c_uint64), P(C.c_uint64)]
        L.orc_voxel_ssb.argtypes = [P(Dna), P(C.c_uint32), C.c_uint32, C.c_double, P(C.c_float)]
        L.orc_voxel_ssb.restype = C.c_double
        L.orc_expected_dsb_local.argtypes = [P(Dna), P(C.c_float), P(C.c_uint8)]
        L.orc_expected_dsb_local.restype = C.c_double
        L.orc_dose_sum_ev.argtypes = [P(C.c_uint32), C.c_uint64]
        L.orc_dose_sum_ev.restype = C.c_double
        L.orc_dose_projection.argtypes = [P(C.c_uint32), C.c_uint32, C.c_int, P(C.c_float)]
        L.orc_chem_grid.argtypes = [P(C.c_float), C.c_uint32, C.c_uint64, P(C.c_float), P(C.c_uint32),
                                    P(C.c_uint32)]
        rc = L.orc_load_tables(BLOB.encode())
        if rc != 0:
            raise RuntimeError(f"oracle: cannot load tables {BLOB} (rc={rc})")
        _LIB = L
    return _LIB


def _fp(a, t=C.c_float):
    return a.ctypes.data_as(C.POINTER(t))


DNA_DEFAULT = dict(grid_n=21, rise=0.34, spacing=150.0, r_bb=1.0)


def dna_x0(L_nm=3000.0, rise=0.34):
    n = int(np.floor(L_nm / rise))
    return np.float32(-(n - 1) * rise * 0.5)


def transport(np_, E_eV, seed=0, box_nm=15000.0, ce_eV=7.5, dna_enable=None, rng_mode=0,
              max_sec=5_000_000, max_rad=16_000_000, sec_steps=2000, max_steps=65536,
              start_half=0.0, vc=128, nthreads=None, want_dose=True, pid_base=0, E_per_primary=None):
    """Phase A + B on the CPU.  Returns a dict of numpy arrays and counters.

    rng_mode 0 = Philox streams (bit-exact with the CUDA path), 1 = the
    reference's xoshiro generator seeded with ``seed`` (normally floor(E))."""
    L = lib()
    if dna_enable is None:
        dna_enable = 1 if E_eV == 10000 else 0
    p = TransportParams(np_, box_nm, ce_eV, max_steps, E_eV, max_sec, vc, max_rad, start_half,
                        dna_enable, DNA_DEFAULT["grid_n"], DNA_DEFAULT["rise"],
                        DNA_DEFAULT["spacing"], float(dna_x0()), DNA_DEFAULT["r_bb"],
                        sec_steps, rng_mode, seed, pid_base, None)
    if E_per_primary is not None:
        E_arr = np.ascontiguousarray(E_per_primary, dtype=np.float32)
        assert E_arr.size == np_
        p.E_per_primary = E_arr.ctypes.data
    res = np.zeros(np_ * 8, dtype=np.float32)
    dose = np.zeros(vc ** 3, dtype=np.uint32) if want_dose else None
    o = TransportOut()
    o.results = _fp(res)
    o.dose = _fp(dose, C.c_uint32) if want_dose else None
    rc = L.orc_transport(C.byref(p), C.byref(o), nthreads or os.cpu_count())
    if rc < 0:
        raise RuntimeError(f"oracle transport rc={rc}")
    n = o.rad_n
    rad = np.ctypeslib.as_array(o.rad, shape=(n * 4,)).copy() if n else np.zeros(0, np.float32)
    key = np.ctypeslib.as_array(o.rad_key, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
    L.orc_free(C.cast(o.rad, C.c_void_p))
    L.orc_free(C.cast(o.rad_key, C.c_void_p))
    return dict(results=res, dose=dose, counters=np.array(o.counters[:], dtype=np.uint32),
                sec_stats=np.array(o.sec_stats[:], dtype=np.uint32),
                dbg=np.array(o.dbg[:], dtype=np.uint32), rad=rad.reshape(-1, 4), rad_key=key,
                dep_units=o.dep_units, dep_eV_f64=o.dep_eV_f64, sec_n=o.sec_n, steps=o.steps,
                capped=(rc == 1))


def irt(rad, n_therm, E_eV, seed=0, nthreads=None, curves=False):
    """IRT to 1 us.  With curves=True also returns per-track counts (max pid + 1,
    16, 5) of OH, eaq, H, H2O2, H2 at t_k = 10^(-3 + 0.4 k) ns."""
    L = lib()
    rad = np.ascontiguousarray(rad, dtype=np.float32).reshape(-1)
    o = IrtOut()
    cv = None
    if curves:
        npid = int(np.rint(rad[3::4]).astype(np.int64).max() // 8) + 1 if rad.size else 0
        cv = np.zeros((max(npid, 1), 16, 5), dtype=np.float32)
        o.curves = _fp(cv)
        o.curves_cap = cv.shape[0]
    L.orc_irt(_fp(rad), rad.size // 4, n_therm, E_eV, seed, C.byref(o), nthreads or os.cpu_count())
    out = dict(tl=np.array(o.tl), G=np.array(o.G), rxn_counts=np.array(o.rxn_counts[:], dtype=np.uint64),
               n_reacted=o.n_reacted, n_pairs=o.n_pairs, n_tracks=o.n_tracks, n_events=o.n_events)
    if curves:
        out["curves"] = cv
    return out


def irt_rxn_table():
    L = lib()
    out = np.zeros((9, 6), dtype=np.float64)
    L.orc_irt_rxn_table(_fp(out, C.c_double))
    return out


class DnaTarget:
    def __init__(self, L_nm=3000.0, grid_N=21, spacing_nm=150.0):
        self._d = Dna()
        lib().orc_build_dna(L_nm, grid_N, spacing_nm, C.byref(self._d))
        d = self._d
        self.n_bp_per, self.n_fibers, self.n_bp, self.grid_N = d.n_bp_per, d.n_fibers, d.n_bp, d.grid_N
        self.x0, self.rise, self.r_bb, self.spacing_nm = d.x0, d.rise, d.r_bb, d.spacing_nm
        self.fy = np.ctypeslib.as_array(d.fy, shape=(d.n_fibers,)).copy()
        self.fz = np.ctypeslib.as_array(d.fz, shape=(d.n_fibers,)).copy()
        self.rbb0 = np.ctypeslib.as_array(d.rbb0, shape=(2 * d.n_bp_per,)).copy()
        self.rbb1 = np.ctypeslib.as_array(d.rbb1, shape=(2 * d.n_bp_per,)).copy()

    def __del__(self):
        try:
            lib().orc_free_dna(C.byref(self._d))
        except Exception:
            pass


def score_direct(dna, rad, lcg_state=0x12345678, hits=None):
    rad = np.ascontiguousarray(rad, dtype=np.float32).reshape(-1)
    if hits is None:
        hits = np.zeros(2 * dna.n_bp, dtype=np.uint8)
    o = SsbOut()
    lib().orc_score_direct(C.byref(dna._d), _fp(rad), rad.size // 4, lcg_state, _fp(hits, C.c_uint8), C.byref(o))
    return dict(hits=hits, ssb=o.ssb, ssb0=o.ssb0, ssb1=o.ssb1, candidates=o.candidates,
                in_reach=o.in_reach, lcg_state=o.lcg_state)


def score_indirect(dna, pos, alive, lcg_state=0x12345678, hits=None):
    pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1)
    alive = np.ascontiguousarray(alive, dtype=np.uint32)
    if hits is None:
        hits = np.zeros(2 * dna.n_bp, dtype=np.uint8)
    o = SsbOut()
    lib().orc_score_indirect(C.byref(dna._d), _fp(pos), _fp(alive, C.c_uint32), alive.size, lcg_state,
                             _fp(hits, C.c_uint8), C.byref(o))
    return dict(hits=hits, ssb=o.ssb, ssb0=o.ssb0, ssb1=o.ssb1, candidates=o.candidates,
                in_reach=o.in_reach, lcg_state=o.lcg_state)


def cluster_dsb(dna, hits):
    hits = np.ascontiguousarray(hits, dtype=np.uint8)
    dsb, s0, s1 = C.c_uint64(), C.c_uint64(), C.c_uint64()
    de = C.c_double()
    lib().orc_cluster_dsb(C.byref(dna._d), _fp(hits, C.c_uint8), C.byref(dsb), C.byref(de),
                          C.byref(s0), C.byref(s1))
    return dict(dsb=dsb.value, dsb_expected=de.value, ssb0=s0.value, ssb1=s1.value)


def voxel_ssb(dna, dose, box_nm=15000.0, vc=128):
    """scoreDirectSSB (ssb-dsb.ts:227-283): (direct_expected, lambda)."""
    dose = np.ascontiguousarray(dose, dtype=np.uint32)
    lam = np.zeros(2 * dna.n_bp, np.float32)
    e = lib().orc_voxel_ssb(C.byref(dna._d), _fp(dose, C.c_uint32), vc, box_nm, _fp(lam))
    return e, lam


def expected_dsb_local(dna, lam, hits=None):
    """expectedDSBLocal (ssb-dsb.ts:285-334)."""
    lam = np.ascontiguousarray(lam, dtype=np.float32)
    h = None if hits is None else _fp(np.ascontiguousarray(hits, dtype=np.uint8), C.c_uint8)
    return lib().orc_expected_dsb_local(C.byref(dna._d), _fp(lam), h)


def dose_sum_ev(dose):
    dose = np.ascontiguousarray(dose, dtype=np.uint32)
    return lib().orc_dose_sum_ev(_fp(dose, C.c_uint32), dose.size)


def dose_projection(dose, axis, vc=128):
    dose = np.ascontiguousarray(dose, dtype=np.uint32)
    out = np.zeros(vc * vc, np.float32)
    lib().orc_dose_projection(_fp(dose, C.c_uint32), vc, axis, _fp(out))
    return out.reshape(vc, vc)


def chem_grid(rad, seed=0, n=None):
    """Grid-hash chemistry on the first n entries of rad: (counts 8 x 5, pos, alive)."""
    rad = np.ascontiguousarray(rad, dtype=np.float32).reshape(-1, 4)
    n = rad.shape[0] if n is None else min(n, rad.shape[0])
    pos = np.zeros((n, 4), np.float32)
    alive = np.zeros(n, np.uint32)
    counts = np.zeros((8, 5), np.uint32)
    rc = lib().orc_chem_grid(_fp(rad), n, seed, _fp(pos), _fp(alive, C.c_uint32), _fp(counts, C.c_uint32))
    if rc:
        raise MemoryError("oracle chem_grid")
    return counts, pos, alive
