"""The benchmark workloads beside the 4096 x 10 keV pipeline:

* single synthetic 10 keV-like track through the IRT (510 spurs of six
  species on a 2.7 um random walk, 2550 tracked species);
* mixed primary energies, log-uniform over 100 eV - 30 keV, in one transport
  launch, then the IRT over tracks of very different species counts.

CPU tests check the inputs and the oracle on them; GPU tests check the CUDA
path against the oracle bit for bit on the same inputs."""
import ctypes as C

import numpy as np
import pytest

import oracle
import wgdna
from wgdna import _lib, synthetic


def test_synthetic_track_shape_and_codes():
    rad = synthetic.synthetic_track()
    assert rad.shape == (510 * 6, 4) and rad.dtype == np.float32
    codes = np.rint(rad[:, 3]).astype(int) % 8
    assert sorted(np.unique(codes)) == [0, 2, 3, 5, 6, 7]
    assert synthetic.tracked_species(rad) == 2550
    # same key, same track; another key, another track
    np.testing.assert_array_equal(rad, synthetic.synthetic_track())
    assert not np.array_equal(rad, synthetic.synthetic_track(key=2))
    # the walk is 2.7 um long: spur centres about 5.3 nm apart
    c = rad[::6, :3].astype(np.float64)
    assert 2.0 < np.median(np.linalg.norm(np.diff(c, axis=0), axis=1)) < 9.0


def test_oracle_on_synthetic_track():
    rad = synthetic.synthetic_track()
    r = oracle.irt(rad, 1, 10000.0, seed=1)
    assert r["n_tracks"] == 1
    g = r["G"]
    # 510 spurs per 100 eV-units of 10 keV: every radical starts at G = 5.1
    # and decays; H2 markers (510) plus H2 made by reactions 3, 4, 6 grow
    assert (np.diff(g[:, 0]) <= 0).all() and (np.diff(g[:, 1]) <= 0).all()
    assert (np.diff(g[:, 4]) >= 0).all() and g[0, 4] >= 5.1
    assert r["n_pairs"] > 1_000_000 and r["n_reacted"] > 500


def test_mixed_energies_are_log_uniform():
    e = synthetic.mixed_energies(65536)
    assert e.min() >= 100.0 and e.max() <= 30000.0
    h, _ = np.histogram(np.log(e), bins=8)
    assert h.min() > 0.9 * h.mean()


@pytest.mark.gpu
def test_irt_synthetic_track_bit_exact(ctx):
    rad = synthetic.synthetic_track()
    ref = oracle.irt(rad, 1, 10000.0, seed=1)
    r = _lib.IrtResult()
    _lib.check("wgdna_run_irt", _lib.lib().wgdna_run_irt(ctx.h, _lib.ptr(rad), rad.shape[0], 1, 10000.0, 1,
                                                         C.byref(r)))
    assert r.device_error == 0 and r.n_tracks == 1
    # more initial events than the sort keeps in shared memory: the device-memory sort runs
    assert r.n_init_events > 4096
    np.testing.assert_array_equal(np.array(r.counts), ref["tl"])
    np.testing.assert_array_equal(np.array(r.rxn_counts[:]), ref["rxn_counts"])
    assert (r.n_reacted, r.n_pairs, r.n_events) == (ref["n_reacted"], ref["n_pairs"], ref["n_events"])


@pytest.mark.gpu
@pytest.mark.parametrize("n,key", [(192, 5), (2048, 6)])
def test_mixed_energies_transport_and_irt_bit_exact(ctx, n, key):
    E = synthetic.mixed_energies(n, key=key)
    o = oracle.transport(n, 10000.0, seed=13, rng_mode=0, dna_enable=0, E_per_primary=E)
    p = wgdna.transport_params(n, 10000.0, 15000.0, 7.5, seed=13, dna_enable=0)
    Eh = np.ascontiguousarray(E, np.float32)
    p.E_per_primary = Eh.ctypes.data
    L = _lib.lib()
    st = _lib.TransportStats()
    _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    res = np.zeros(n * 8, np.float32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    k = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), None, _lib.ptr(rad),
                                                       st.rad_n_stored, C.byref(k)))
    np.testing.assert_array_equal(res.view(np.uint32), o["results"].view(np.uint32))
    np.testing.assert_array_equal(rad.view(np.uint32), o["rad"].view(np.uint32))
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    ref = oracle.irt(o["rad"], nth, float(E.mean()), seed=3)
    r = _lib.IrtResult()
    _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, nth, float(E.mean()), 3, C.byref(r)))
    np.testing.assert_array_equal(np.array(r.counts), ref["tl"])
    np.testing.assert_array_equal(np.array(r.rxn_counts[:]), ref["rxn_counts"])
    assert r.n_pairs == ref["n_pairs"] and r.n_events == ref["n_events"]
