"""The oracle's scoring against a direct Python transcription of the
reference's JavaScript loops (src/scoring/ssb-dsb.ts:43-427), evaluated with
JS number semantics, on small lists: a second, independent restatement that
pins the oracle's scoring bit for bit."""
import math

import numpy as np

import oracle

R_D = 0.29


def js_round(x):
    f = math.floor(x)
    return f + 1 if x - f >= 0.5 else f


def make_rng(seed=0x12345678):
    s = [seed & 0xFFFFFFFF]

    def rng():
        s[0] = (s[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return s[0] / 4294967296

    return rng, s


def nearest(d, x, y, z):
    x_half = (d.n_bp_per - 1) * d.rise * 0.5
    grid_off = -((d.grid_N - 1) * d.spacing_nm) * 0.5
    if x < -x_half - R_D or x > x_half + R_D:
        return None, 0
    fi = js_round((y - grid_off) * (1 / d.spacing_nm))
    fj = js_round((z - grid_off) * (1 / d.spacing_nm))
    if fi < 0 or fi >= d.grid_N or fj < 0 or fj >= d.grid_N:
        return None, 0
    fib = fi * d.grid_N + fj
    y_rel = y - float(d.fy[fib])
    z_rel = z - float(d.fz[fib])
    if y_rel * y_rel + z_rel * z_rel > (d.r_bb + R_D) * (d.r_bb + R_D):
        return None, 0
    bp_est = js_round((x + x_half) * (1 / d.rise))
    best, bb, bs = math.inf, -1, -1
    for b in range(max(0, bp_est - 2), min(d.n_bp_per - 1, bp_est + 2) + 1):
        dx = x - (d.x0 + b * d.rise)
        dy0, dz0 = y_rel - float(d.rbb0[2 * b]), z_rel - float(d.rbb0[2 * b + 1])
        d20 = dx * dx + dy0 * dy0 + dz0 * dz0
        if d20 < best:
            best, bb, bs = d20, b, 0
        dy1, dz1 = y_rel - float(d.rbb1[2 * b]), z_rel - float(d.rbb1[2 * b + 1])
        d21 = dx * dx + dy1 * dy1 + dz1 * dz1
        if d21 < best:
            best, bb, bs = d21, b, 1
    if best < R_D * R_D:
        return fib * d.n_bp_per + bb + bs * d.n_bp, 1
    return None, 1


def js_score_direct(d, rad, seed):
    """scoreDirectSSB_events (ssb-dsb.ts:135-217)."""
    rng, st = make_rng(seed)
    hits = np.zeros(2 * d.n_bp, np.uint8)
    cand = reach = ssb = 0
    n = len(rad)
    i = 0
    while i < n:
        x, y, z = (float(v) for v in rad[i, :3])
        skip = 2 if (i + 1 < n and rad[i + 1, 0] == rad[i, 0] and rad[i + 1, 1] == rad[i, 1]
                     and rad[i + 1, 2] == rad[i, 2]) else 1
        i += skip
        h, c = nearest(d, x, y, z)
        cand += c
        if h is None:
            continue
        reach += 1
        if rng() < 0.15 and hits[h] == 0:
            hits[h] = 1
            ssb += 1
    return hits, ssb, cand, reach, st[0]


def js_cluster(d, hits):
    """clusterDSB integer part (ssb-dsb.ts:370-396)."""
    W, n, dsb = 10, d.n_bp, 0
    for f in range(d.n_fibers):
        base = f * d.n_bp_per
        s0 = np.flatnonzero(hits[base: base + d.n_bp_per] == 1)
        s1 = np.flatnonzero(hits[base + n: base + n + d.n_bp_per] == 1)
        used = np.zeros(len(s1), bool)
        jlo = 0
        for b0 in s0:
            while jlo < len(s1) and s1[jlo] < b0 - W:
                jlo += 1
            j = jlo
            while j < len(s1) and s1[j] <= b0 + W:
                if not used[j]:
                    used[j] = True
                    dsb += 1
                    break
                j += 1
    return dsb


def sites(d, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        if rng.random() < 0.5:
            f, b, s = rng.integers(d.n_fibers), rng.integers(d.n_bp_per), rng.integers(2)
            off = (d.rbb0 if s == 0 else d.rbb1)[2 * b: 2 * b + 2]
            p = (d.x0 + b * d.rise + rng.normal(0, 0.12), d.fy[f] + off[0] + rng.normal(0, 0.12),
                 d.fz[f] + off[1] + rng.normal(0, 0.12))
        else:
            p = tuple(rng.uniform(-1600, 1600, 3))
        for _ in range(int(rng.choice([1, 1, 2, 3]))):
            out.append(p + (0.0,))
    return np.array(out[:n], np.float32)


def test_lcg_first_values():
    rng, st = make_rng()
    assert st[0] == 0x12345678
    v1 = rng()
    assert st[0] == (0x12345678 * 1664525 + 1013904223) % 2 ** 32
    assert v1 == st[0] / 2 ** 32


def test_js_round_ties_up():
    assert js_round(2.5) == 3 and js_round(-2.5) == -2 and js_round(0.49999999999999994) == 0


def test_oracle_direct_scoring_equals_js_transcription():
    d = oracle.DnaTarget()
    for n, seed, s0 in ((4000, 1, 0x12345678), (2500, 2, 0xCAFEBABE)):
        rad = sites(d, n, seed)
        hits, ssb, cand, reach, st = js_score_direct(d, rad, s0)
        o = oracle.score_direct(d, rad, s0)
        assert (o["ssb"], o["candidates"], o["in_reach"], o["lcg_state"]) == (ssb, cand, reach, st)
        np.testing.assert_array_equal(o["hits"], hits)
        assert reach > 100 and ssb > 5


def test_oracle_cluster_equals_js_transcription():
    d = oracle.DnaTarget()
    hits = (np.random.default_rng(3).random(2 * d.n_bp) < 0.002).astype(np.uint8)
    assert oracle.cluster_dsb(d, hits)["dsb"] == js_cluster(d, hits)


def test_dedupe_walk_visits_alternate_entries_of_a_run():
    """[A, A, B, B, B, C]: the walk visits indices 0, 2, 4, 5 (ssb-dsb.ts:155-168)."""
    d = oracle.DnaTarget()
    b = 4000
    A = (d.x0 + b * d.rise, float(d.fy[220] + d.rbb0[2 * b]), float(d.fz[220] + d.rbb0[2 * b + 1]), 0)
    B = (A[0] + 0.34, A[1], A[2], 0)
    Cc = (A[0] + 0.68, A[1], A[2], 0)
    rad = np.array([A, A, B, B, B, Cc], np.float32)
    o = oracle.score_direct(d, rad, 7)
    _, _, cand, reach, _ = js_score_direct(d, rad, 7)
    assert o["candidates"] == cand == 4
