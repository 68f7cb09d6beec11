"""Primary sharding over two gloo ranks on CPU (the N > 1 path without GPUs).

Each rank runs its block of global primary ids through the oracle; the
all-reduced counters, dose grid and IRT counts, and the sharded scoring
protocol (wgdna.sharded), must equal a single run over all primaries bit for
bit.  A rank that fails makes the other rank's next collective fail within
the process group's timeout instead of hanging."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG, ROOT

NP_TOTAL = 48


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _init(rank, world, port, timeout_s=60):
    sys.path[:0] = [ROOT, PKG]
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _sites(n, seed):
    import oracle
    d = oracle.DnaTarget()
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        f, b, s = rng.integers(d.n_fibers), rng.integers(d.n_bp_per), rng.integers(2)
        off = (d.rbb0 if s == 0 else d.rbb1)[2 * b: 2 * b + 2]
        p = (d.x0 + b * d.rise + rng.normal(0, 0.12), d.fy[f] + off[0] + rng.normal(0, 0.12),
             d.fz[f] + off[1] + rng.normal(0, 0.12), 0.0)
        out += [p] * int(rng.choice([1, 2]))
    return np.array(out[:n], np.float32), d


def _worker(rank, world, port, q):
    try:
        dist = _init(rank, world, port)
        import oracle
        from wgdna import sharded
        base, n = sharded.shard(NP_TOTAL, rank, world)
        o = oracle.transport(n, 10000.0, seed=3, rng_mode=0, pid_base=base, nthreads=2)
        counters = sharded.allreduce_sum(dist, o["counters"].astype(np.int64))
        dose = sharded.reduce_dose(dist, o["dose"])
        nth_local = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
        nth = int(sharded.allreduce_sum(dist, np.array([nth_local]))[0])
        ir = oracle.irt(o["rad"], nth, 10000.0, seed=9, nthreads=2)
        tl = sharded.allreduce_sum(dist, ir["tl"])
        rxn = sharded.allreduce_sum(dist, ir["rxn_counts"].astype(np.int64))
        # scoring on a synthetic list split at a run boundary
        rad_all, d = _sites(6000, 17)
        cut = 3001 if rad_all[3000, 0] != rad_all[3001, 0] else 3002
        mine = rad_all[:cut] if rank == 0 else rad_all[cut:]

        def score_fn(rad, state):
            r = oracle.score_direct(d, rad, state)
            return r["hits"], r["in_reach"], r["candidates"]

        sc = sharded.sharded_score(dist, score_fn, mine, 0x12345678, d.n_bp)
        res = {"counters": counters, "dose_sum": int(dose.astype(np.uint64).sum()), "dose_nz": int((dose > 0).sum()),
               "tl": tl, "rxn": rxn, "nth": nth, "ssb": sc["ssb_count"], "in_reach": sc["in_reach"],
               "lcg": sc["lcg_state"], "hits_sum": int(sc["hits"].sum()), "cand": sc["candidates"],
               "rad": o["rad"] if rank == 0 else None, "rad1": o["rad"] if rank == 1 else None}
        q.put((rank, res))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put((rank, repr(e)))
        raise


def test_two_rank_sharding_equals_single_run():
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert not isinstance(got[0], str), got[0]
    assert not isinstance(got[1], str), got[1]
    ref = oracle.transport(NP_TOTAL, 10000.0, seed=3, rng_mode=0)
    np.testing.assert_array_equal(got[0]["counters"], ref["counters"].astype(np.int64))
    assert got[0]["dose_sum"] == int(ref["dose"].astype(np.uint64).sum())
    assert got[0]["dose_nz"] == int((ref["dose"] > 0).sum())
    # shards concatenated in rank order == the single canonical rad_buf
    np.testing.assert_array_equal(np.concatenate([got[0]["rad"], got[1]["rad1"]]).view(np.uint32),
                                  ref["rad"].view(np.uint32))
    nth = int((ref["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    assert got[0]["nth"] == nth
    ir = oracle.irt(ref["rad"], nth, 10000.0, seed=9)
    np.testing.assert_array_equal(got[0]["tl"], ir["tl"])
    np.testing.assert_array_equal(got[0]["rxn"], ir["rxn_counts"].astype(np.int64))
    rad_all, d = _sites(6000, 17)
    sref = oracle.score_direct(d, rad_all, 0x12345678)
    for r in (0, 1):
        assert got[r]["ssb"] == sref["ssb"] and got[r]["in_reach"] == sref["in_reach"]
        assert got[r]["lcg"] == sref["lcg_state"] and got[r]["hits_sum"] == int(sref["hits"].sum())
        assert got[r]["cand"] == sref["candidates"]


def _failing_worker(rank, world, port, q):
    import torch
    dist = _init(rank, world, port, timeout_s=5)
    if rank == 1:
        q.put((rank, "raised"))
        raise RuntimeError("injected failure on rank 1 between steps")
    t = torch.ones(4)
    try:
        dist.all_reduce(t)
        q.put((rank, "completed"))
    except Exception as e:
        q.put((rank, "error:" + type(e).__name__))


def test_failed_rank_is_detected_by_the_next_collective():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert got[1] == "raised"
    assert got[0].startswith("error:")
    assert procs[1].exitcode != 0
