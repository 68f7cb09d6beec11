"""The reference's unit tests (tests/unit/*.test.ts), restated against this
package's host surface and the oracle."""
import math

import numpy as np

import oracle
import wgdna
from wgdna import constants as K


def test_app_defaults():                                   # app-defaults.test.ts:12-16
    assert K.DEFAULT_CHEM_BACKEND == "worker"


def test_constants():                                      # constants.test.ts:1-62
    assert len(K.BIND) == 5
    assert [round(b, 2) for b in K.BIND] == [10.79, 13.39, 16.05, 32.30, 539.0]
    assert len(K.EXC_E) == 5 and K.EXC_E[0] == 8.22 and K.EXC_E[4] == 13.77
    assert len(K.VIB_LEV) == 9 and K.VIB_LEV[0] == 0.01 and K.VIB_LEV[8] == 0.835
    assert K.NW == 33.4
    assert (K.DIFFUSION["OH"], K.DIFFUSION["eaq"], K.DIFFUSION["H"], K.DIFFUSION["H3O"]) == (2.2, 4.9, 7.0, 9.0)
    assert len(K.IRT_REACTIONS) == 7
    assert K.IRT_REACTIONS[0][:2] == (0, 0) and K.IRT_REACTIONS[0][4] == 1
    assert K.IRT_REACTIONS[5][:2] == (1, 3) and K.IRT_REACTIONS[5][4] == 3
    assert K.KARAMITROS_2011 == {"G_OH": 2.50, "G_eaq": 2.50, "G_H": 0.57, "G_H2O2": 0.73, "G_H2": 0.42}


def test_dna_geometry():                                   # dna-geometry.test.ts:1-40
    for dna in (wgdna.build_dna_target(3000, 21, 150), oracle.DnaTarget(3000, 21, 150)):
        assert dna.n_fibers == 441 and dna.grid_N == 21
        bp = math.floor(3000 / 0.34)
        assert dna.n_bp_per == bp and dna.n_bp == 441 * bp and dna.n_bp > 3_000_000
        assert dna.spacing_nm == 150 and dna.r_bb == 1.0 and abs(dna.rise - 0.34) < 1e-9
        assert dna.rbb0.size == 2 * dna.n_bp_per and dna.rbb1.size == 2 * dna.n_bp_per
        assert abs(dna.x0 - (-(dna.n_bp_per - 1) * dna.rise * 0.5)) < 1e-9


def test_dna_geometry_host_equals_oracle():
    a, b = wgdna.build_dna_target(), oracle.DnaTarget()
    for f in ("fy", "fz", "rbb0", "rbb1"):
        np.testing.assert_array_equal(getattr(a, f).view(np.uint32), getattr(b, f).view(np.uint32))


def decode(w):                                             # rad-buf-encoding.test.ts:20-24
    i = int(np.floor(float(w) + 0.5))
    return i // 8, i % 8


def test_rad_buf_encoding():                               # rad-buf-encoding.test.ts:26-84
    for s in (0, 1, 2, 3, 5, 6, 7):
        assert decode(np.float32(0 * 8 + s)) == (0, s)
    for pid, s in ((1, 0), (7, 5), (4095, 2), (4095, 7)):
        assert decode(np.float32(pid * 8 + s)) == (pid, s)
    for pid in range(1, 4096, 137):
        for s in (0, 1, 2, 3, 5, 6, 7):
            assert decode(np.float32(pid * 8 + s))[1] == s
    # the f32 w stays exact up to pid 2,097,151 (the batch limit of the C ABI)
    assert decode(np.float32(2_097_151 * 8 + 7)) == (2_097_151, 7)


def test_reaction_table():                                 # reactions.test.ts:1-54
    def find(a, b):
        lo, hi = min(a, b), max(a, b)
        return next((r for r in K.IRT_REACTIONS if r[0] == lo and r[1] == hi), None)
    assert abs(find(1, 0)[3] - 0.98) < 0.005
    assert all(r[2] > 0 for r in K.IRT_REACTIONS)
    assert all(0 < r[3] <= 1 for r in K.IRT_REACTIONS)
    assert all(0 <= r[4] <= 3 for r in K.IRT_REACTIONS)
    assert abs(find(1, 3)[2] - 0.47) < 0.005
    rx = find(0, 0)
    k_si = 4 * math.pi * rx[2] * (2 * K.DIFFUSION["OH"]) * rx[3] * 6.022e23 * 1e-24 * 1e9
    assert 0.5 < k_si / 4.4e9 < 2.0


def test_worker_reaction_constants():
    """irt-worker.js:240-279: TDC sigma = k/(4 pi D) (x2 for self), PDC contact
    radius = sum of VdW radii, Onsager rc = q1 q2 * 0.711 nm."""
    t = oracle.irt_rxn_table()
    kc = 1e24 / (6.022e23 * 1e9)
    assert abs(t[3, 0] - 2 * 0.636e10 * kc / (4 * math.pi * 9.8)) < 1e-15   # eaq+eaq
    assert abs(t[0, 0] - 0.44) < 1e-15                                        # OH+OH contact
    assert abs(t[5, 2] - (-1.44 / (0.02527 * 80.1))) < 1e-15                 # eaq+H3O+ rc
    assert t[3, 2] > 0 and t[8, 2] < 0                                        # repulsive / attractive
    assert all(0 < p <= 1 for p in t[:, 5])
