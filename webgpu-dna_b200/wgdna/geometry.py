"""B-DNA fibre-grid target (src/physics/dna-geometry.ts:16-68, types.ts:23-37)."""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class DNATarget:
    rise: float
    r_bb: float
    n_bp_per: int
    n_fibers: int
    n_bp: int
    grid_N: int
    spacing_nm: float
    x0: float
    L_nm: float
    fy: np.ndarray        # float32[grid_N^2]
    fz: np.ndarray
    rbb0: np.ndarray      # float32[2*n_bp_per]: (y0, z0, y1, z1, ...)
    rbb1: np.ndarray

    @property
    def key(self):
        return (self.L_nm, self.grid_N, self.spacing_nm)


def build_dna_target(L_nm=3000.0, grid_N=21, spacing_nm=150.0):
    """buildDNATarget: grid_N x grid_N straight fibres along X (host only)."""
    L = _lib.lib()
    info = _lib.DnaInfo()
    _lib.check("wgdna_build_dna_target",
               L.wgdna_build_dna_target(float(L_nm), int(grid_N), float(spacing_nm), None, None, None, None,
                                        C.byref(info)))
    fy = np.zeros(info.n_fibers, np.float32)
    fz = np.zeros(info.n_fibers, np.float32)
    rbb0 = np.zeros(2 * info.n_bp_per, np.float32)
    rbb1 = np.zeros(2 * info.n_bp_per, np.float32)
    _lib.check("wgdna_build_dna_target",
               L.wgdna_build_dna_target(float(L_nm), int(grid_N), float(spacing_nm), _lib.ptr(fy), _lib.ptr(fz),
                                        _lib.ptr(rbb0), _lib.ptr(rbb1), C.byref(info)))
    return DNATarget(rise=info.rise, r_bb=info.r_bb, n_bp_per=info.n_bp_per, n_fibers=info.n_fibers,
                     n_bp=info.n_bp, grid_N=info.grid_N, spacing_nm=info.spacing_nm, x0=info.x0,
                     L_nm=info.L_nm, fy=fy, fz=fz, rbb0=rbb0, rbb1=rbb1)


buildDNATarget = build_dna_target
