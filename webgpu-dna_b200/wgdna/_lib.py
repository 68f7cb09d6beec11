"""ctypes binding of libwgdna.so (declarations in include/wgdna.h).

The product path always goes through this library; there is no CPU fallback.
If the library is missing or no CUDA device is present, the calls raise.
"""
import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libwgdna.so")
TABLES_PATH = os.path.join(PKG_ROOT, "data", "cross_sections.bin")

WGDNA_OK = 0
WGDNA_ERR_ARG, WGDNA_ERR_CUDA, WGDNA_ERR_TABLES, WGDNA_ERR_CAPACITY = -1, -2, -3, -4
WGDNA_ERR_DEVICE, WGDNA_ERR_NOMEM, WGDNA_ERR_STATE = -5, -6, -7
ERRORS = {-1: "WGDNA_ERR_ARG", -2: "WGDNA_ERR_CUDA", -3: "WGDNA_ERR_TABLES", -4: "WGDNA_ERR_CAPACITY",
          -5: "WGDNA_ERR_DEVICE", -6: "WGDNA_ERR_NOMEM", -7: "WGDNA_ERR_STATE"}

# every entry point declared in include/wgdna.h
EXPORTS = ["wgdna_default_cfg", "wgdna_create", "wgdna_destroy", "wgdna_last_error", "wgdna_version",
           "wgdna_set_stream", "wgdna_transport", "wgdna_transport_copy_out", "wgdna_run_transport",
           "wgdna_run_irt", "wgdna_irt", "wgdna_build_dna_target", "wgdna_set_dna_target",
           "wgdna_score_direct", "wgdna_score_indirect", "wgdna_cluster_dsb", "wgdna_score",
           "wgdna_score_direct_noalloc", "wgdna_reaction_table", "wgdna_irt_record_curves", "wgdna_irt_curves",
           "wgdna_track_descriptors", "wgdna_surrogate_init", "wgdna_surrogate_params", "wgdna_surrogate_norm",
           "wgdna_surrogate_load", "wgdna_surrogate_train", "wgdna_surrogate_grad", "wgdna_surrogate_predict",
           "wgdna_surrogate_chemistry", "wgdna_dose_sum", "wgdna_dose_projection", "wgdna_score_voxel_ssb",
           "wgdna_expected_dsb_local", "wgdna_chem_grid", "wgdna_device_views", "wgdna_score_draws",
           "wgdna_cluster_device", "wgdna_set_wait_limits", "wgdna_default_tuning", "wgdna_get_tuning",
           "wgdna_set_tuning"]
SG_IN, SG_OUT, SG_NPARAM = 64, 80, 51664
# test switches of wgdna_set_wait_limits
WGDNA_TEST_UNPUBLISHED, WGDNA_TEST_MMA_WAIT = 1, 2


class WgdnaError(RuntimeError):
    def __init__(self, func, code, msg):
        super().__init__(f"{func} failed ({ERRORS.get(code, code)}): {msg}")
        self.code = code


class Cfg(C.Structure):
    _fields_ = [("device", C.c_int), ("tables_path", C.c_char_p), ("max_primaries", C.c_uint32),
                ("max_sec", C.c_uint32), ("max_rad", C.c_uint64), ("vc", C.c_uint32), ("reserved", C.c_uint32)]


class Tuning(C.Structure):
    """wgdna_tuning: launch and scheduling shapes (results never depend on them)."""
    _fields_ = [("transport_ctas_per_sm", C.c_uint32), ("prim_take", C.c_uint32), ("stash_keep", C.c_uint32),
                ("stash_spill", C.c_uint32), ("queue_poll", C.c_uint32), ("irt_init_blocks_per_sm", C.c_uint32),
                ("irt_loop_blocks_per_sm", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class TransportParams(C.Structure):
    _fields_ = [("np", C.c_uint32), ("E_eV", C.c_float), ("box_nm", C.c_float), ("ce_eV", C.c_float),
                ("max_steps", C.c_uint32), ("sec_steps", C.c_uint32), ("start_half", C.c_float),
                ("dna_enable", C.c_uint32), ("dna_grid_n", C.c_uint32), ("dna_rise", C.c_float),
                ("dna_spacing", C.c_float), ("dna_x0", C.c_float), ("dna_r_bb", C.c_float),
                ("pid_base", C.c_uint32), ("seed", C.c_uint64), ("E_per_primary", C.c_void_p)]


class TransportStats(C.Structure):
    _fields_ = [("counters", C.c_uint32 * 8), ("sec_stats", C.c_uint32 * 8), ("dbg", C.c_uint32 * 8),
                ("rad_n_raw", C.c_uint64), ("rad_n_stored", C.c_uint64), ("rad_dropped", C.c_uint64),
                ("sec_n_raw", C.c_uint64), ("sec_n", C.c_uint64), ("sec_dropped", C.c_uint64),
                ("dep_units", C.c_uint64), ("dep_eV_f64", C.c_double), ("steps", C.c_uint64),
                ("ms_transport", C.c_float), ("ms_canon", C.c_float), ("device_error", C.c_uint32),
                ("n_therm", C.c_uint32)]


class IrtResult(C.Structure):
    _fields_ = [("counts", (C.c_double * 5) * 7), ("G", (C.c_double * 5) * 7), ("rxn_counts", C.c_uint64 * 9),
                ("n_reacted", C.c_uint64), ("n_tracks", C.c_uint64), ("n_pairs", C.c_uint64),
                ("n_events", C.c_uint64), ("n_particles", C.c_uint64), ("n_init_events", C.c_uint64),
                ("chem_n", C.c_uint64), ("ms", C.c_float),
                ("ms_load", C.c_float), ("ms_pairing", C.c_float), ("ms_events", C.c_float),
                ("device_error", C.c_uint32), ("ms_sort", C.c_float)]


class ChemGridResult(C.Structure):
    _fields_ = [("counts", (C.c_uint32 * 5) * 8), ("G", (C.c_double * 5) * 8), ("chem_n", C.c_uint64),
                ("deposited_eV", C.c_double), ("ms", C.c_float)]


class DeviceView(C.Structure):
    _fields_ = [("dose", C.c_void_p), ("dose_words", C.c_uint64), ("hits", C.c_void_p), ("hits_bytes", C.c_uint64),
                ("rad", C.c_void_p), ("rad_n", C.c_uint64), ("results", C.c_void_p), ("n_primaries", C.c_uint32),
                ("stream", C.c_void_p)]


class DnaInfo(C.Structure):
    _fields_ = [("grid_N", C.c_uint32), ("n_bp_per", C.c_uint32), ("n_fibers", C.c_uint32), ("n_bp", C.c_uint32),
                ("rise", C.c_double), ("r_bb", C.c_double), ("spacing_nm", C.c_double), ("x0", C.c_double),
                ("L_nm", C.c_double)]


class SsbResult(C.Structure):
    _fields_ = [("ssb", C.c_uint64), ("ssb0", C.c_uint64), ("ssb1", C.c_uint64), ("candidates", C.c_uint64),
                ("in_reach", C.c_uint64), ("lcg_state", C.c_uint32), ("ms", C.c_float)]


class DsbResult(C.Structure):
    _fields_ = [("dsb", C.c_uint64), ("ssb0", C.c_uint64), ("ssb1", C.c_uint64), ("dsb_expected", C.c_double),
                ("ms", C.c_float)]


_LIB = None


def lib():
    """Load libwgdna.so (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python webgpu-dna_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "wgdna_default_cfg": (None, [P(Cfg)]),
        "wgdna_create": (C.c_int, [P(Cfg), P(vp)]),
        "wgdna_destroy": (None, [vp]),
        "wgdna_last_error": (C.c_char_p, []),
        "wgdna_version": (C.c_int, []),
        "wgdna_set_stream": (C.c_int, [vp, vp]),
        "wgdna_transport": (C.c_int, [vp, P(TransportParams), P(TransportStats)]),
        "wgdna_transport_copy_out": (C.c_int, [vp, vp, vp, vp, C.c_uint64, P(C.c_uint64)]),
        "wgdna_run_transport": (C.c_int, [vp, P(TransportParams), vp, vp, vp, C.c_uint64, P(C.c_uint64),
                                          P(TransportStats)]),
        "wgdna_run_irt": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32, C.c_double, C.c_uint64, P(IrtResult)]),
        "wgdna_irt": (C.c_int, [vp, C.c_uint32, C.c_double, C.c_uint64, P(IrtResult)]),
        "wgdna_build_dna_target": (C.c_int, [C.c_double, C.c_uint32, C.c_double, vp, vp, vp, vp, P(DnaInfo)]),
        "wgdna_set_dna_target": (C.c_int, [vp, C.c_double, C.c_uint32, C.c_double]),
        "wgdna_score_direct": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32, vp, P(SsbResult)]),
        "wgdna_score_indirect": (C.c_int, [vp, vp, vp, C.c_uint64, C.c_uint32, vp, P(SsbResult)]),
        "wgdna_cluster_dsb": (C.c_int, [vp, vp, P(DsbResult)]),
        "wgdna_score": (C.c_int, [vp, C.c_uint32, P(SsbResult), P(DsbResult)]),
        "wgdna_reaction_table": (C.c_int, [vp]),
        "wgdna_score_direct_noalloc": (C.c_int, [vp, C.c_uint64, vp, vp, vp, vp, P(DnaInfo), C.c_uint32, vp, vp,
                                                 P(SsbResult)]),
        "wgdna_irt_record_curves": (C.c_int, [vp, C.c_int]),
        "wgdna_irt_curves": (C.c_int, [vp, vp, C.c_uint64, P(C.c_uint64)]),
        "wgdna_track_descriptors": (C.c_int, [vp, vp, C.c_uint64, P(C.c_uint64)]),
        "wgdna_surrogate_init": (C.c_int, [vp, C.c_uint64]),
        "wgdna_surrogate_params": (C.c_int, [vp, vp, vp]),
        "wgdna_surrogate_norm": (C.c_int, [vp, vp, vp]),
        "wgdna_surrogate_load": (C.c_int, [vp, vp, vp, C.c_uint64]),
        "wgdna_surrogate_train": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_float, C.c_uint64, vp]),
        "wgdna_surrogate_grad": (C.c_int, [vp, C.c_uint64, vp, P(C.c_double)]),
        "wgdna_surrogate_predict": (C.c_int, [vp, vp, C.c_uint64, vp]),
        "wgdna_surrogate_chemistry": (C.c_int, [vp, vp, P(C.c_float)]),
        "wgdna_dose_sum": (C.c_int, [vp, vp, P(C.c_double)]),
        "wgdna_dose_projection": (C.c_int, [vp, vp, C.c_int, vp]),
        "wgdna_score_voxel_ssb": (C.c_int, [vp, vp, C.c_double, vp, P(C.c_double)]),
        "wgdna_expected_dsb_local": (C.c_int, [vp, vp, vp, P(C.c_double)]),
        "wgdna_chem_grid": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32, C.c_double, C.c_uint64, P(ChemGridResult),
                                      vp, vp, C.c_uint64]),
        "wgdna_device_views": (C.c_int, [vp, P(DeviceView)]),
        "wgdna_score_draws": (C.c_int, [vp, C.c_uint32, P(SsbResult)]),
        "wgdna_cluster_device": (C.c_int, [vp, P(DsbResult)]),
        "wgdna_set_wait_limits": (C.c_int, [vp, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32]),
        "wgdna_default_tuning": (None, [P(Tuning)]),
        "wgdna_get_tuning": (C.c_int, [vp, P(Tuning)]),
        "wgdna_set_tuning": (C.c_int, [vp, P(Tuning)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def check(func, rc):
    if rc != WGDNA_OK:
        msg = lib().wgdna_last_error()
        raise WgdnaError(func, rc, msg.decode() if msg else "")


def ptr(a):
    """Host pointer of a numpy array or a (pinned) torch tensor, or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return C.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    raise TypeError(f"unsupported buffer type {type(a)}")


class Context:
    """Owns a wgdna_ctx (device buffers of one call at a time, one stream)."""

    def __init__(self, max_primaries=4096, max_sec=5_000_000, max_rad=16_000_000, vc=128, device=0,
                 tables_path=None):
        L = lib()
        cfg = Cfg()
        L.wgdna_default_cfg(C.byref(cfg))
        cfg.device = device
        cfg.max_primaries = max_primaries
        cfg.max_sec = max_sec
        cfg.max_rad = max_rad
        cfg.vc = vc
        cfg.tables_path = tables_path.encode() if tables_path else None
        h = C.c_void_p()
        check("wgdna_create", L.wgdna_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.max_primaries, self.max_sec, self.max_rad, self.vc = max_primaries, max_sec, max_rad, vc

    def close(self):
        if getattr(self, "h", None):
            lib().wgdna_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        check("wgdna_set_stream", lib().wgdna_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def tuning(self):
        t = Tuning()
        check("wgdna_get_tuning", lib().wgdna_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t=None, **fields):
        """Apply a Tuning (or the current one with ``fields`` changed)."""
        t = t if t is not None else self.tuning()
        for k, v in fields.items():
            setattr(t, k, int(v))
        check("wgdna_set_tuning", lib().wgdna_set_tuning(self.h, C.byref(t)))
        return t


def reaction_table():
    """Per-reaction constants (irt-worker.js:240-279) as a (9, 6) array:
    sigma, sigma_eff, rc, kdif, kact, prob."""
    out = np.zeros((9, 6), np.float64)
    check("wgdna_reaction_table", lib().wgdna_reaction_table(ptr(out)))
    return out
