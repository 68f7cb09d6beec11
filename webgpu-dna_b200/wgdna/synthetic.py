"""Seeded synthetic inputs for the benchmark workloads.

* ``synthetic_track``: one 10 keV-like track for the single-track IRT case --
  a 3-D random walk of ``length_nm`` with ``n_spurs`` spur centres evenly
  spaced along it; each spur emits OH (code 0), a pre-thermalised e-aq (5, no
  further displacement), H3O+ (3), H (2), an H2 marker (7, counted, not
  tracked) and OH- (6), each at an independent N(0, sigma^2) offset per axis
  with sigma ~ U[1, 2] nm per spur.  Entries are float32 rad_buf records
  (x, y, z, pid * 8 + code) of primary 0, the format of
  tests/unit/rad-buf-encoding.test.ts:5-11.
* ``mixed_energies``: primary energies log-uniform over [lo, hi] eV.

Both draw from numpy's Philox bit generator with the given key, so the inputs
are reproducible across machines.
"""
import numpy as np

SPUR_CODES = (0, 5, 3, 2, 7, 6)


def _rng(key):
    return np.random.Generator(np.random.Philox(key=int(key)))


def synthetic_track(key=1, n_spurs=510, length_nm=2700.0, sigma_lo=1.0, sigma_hi=2.0, pid=0):
    g = _rng(key)
    step = length_nm / n_spurs
    d = g.normal(size=(n_spurs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    centres = np.cumsum(d * step, axis=0)
    sig = g.uniform(sigma_lo, sigma_hi, size=n_spurs)
    k = len(SPUR_CODES)
    off = g.normal(size=(n_spurs, k, 3)) * sig[:, None, None]
    pos = centres[:, None, :] + off
    w = np.broadcast_to(np.array(SPUR_CODES, np.float64) + 8.0 * pid, (n_spurs, k))
    rad = np.concatenate([pos.reshape(-1, 3), w.reshape(-1, 1)], axis=1).astype(np.float32)
    return rad


def mixed_energies(n, lo=100.0, hi=30000.0, key=3):
    g = _rng(key)
    return np.exp(g.uniform(np.log(lo), np.log(hi), size=n)).astype(np.float32)


def tracked_species(rad):
    """Entries the IRT tracks (codes other than 4 and 7, irt-worker.js:475-537)."""
    code = np.rint(np.asarray(rad)[:, 3]).astype(np.int64) % 8
    return int(((code != 4) & (code != 7)).sum())
