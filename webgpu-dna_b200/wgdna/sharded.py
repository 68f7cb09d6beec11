"""Primary-sharded runs over torch.distributed ranks (one process per GPU).

Primaries are independent histories keyed by their global id (Philox counter
(block, secondary, pid, .)), so rank r simply runs the global ids
[r*n, (r+1)*n) with pid_base = r*n: transport and IRT need no data exchange,
only sums of integer counters.  Direct SSB scoring is sequential in the
reference (one LCG draw per in-reach site, in rad_buf order, ssb-dsb.ts:203);
the sharded protocol reproduces the single-device result exactly:

  1. every rank scores its shard once to learn its number of draws n_r
     (the count does not depend on the LCG state);
  2. all-gather n_r; rank r starts from the LCG state advanced by
     sum_{q<r} n_q draws (affine jump-ahead) and scores again;
  3. the hit bytes are OR-reduced (MAX on uint8); SSB counts are the set bytes
     of the combined array, DSBs are clustered once.

A run of identical positions spanning a shard boundary (two primaries
producing bit-identical f32 sites at the boundary) would change which entry
the reference's dedupe walk visits; shards are contiguous in primary id, so
this needs two different histories to coincide bit for bit.
"""
import numpy as np

LCG_A, LCG_C = 1664525, 1013904223


def lcg_jump(state, k):
    """State of makeSsbRng (ssb-dsb.ts:421-427) after k draws."""
    ra, rc, pa, pc = 1, 0, LCG_A, LCG_C
    k = int(k)
    while k:
        if k & 1:
            ra, rc = (pa * ra) & 0xFFFFFFFF, (pa * rc + pc) & 0xFFFFFFFF
        pa, pc = (pa * pa) & 0xFFFFFFFF, (pa * pc + pc) & 0xFFFFFFFF
        k >>= 1
    return (ra * state + rc) & 0xFFFFFFFF


def shard(np_total, rank, world):
    """Contiguous block of global primary ids for a rank: (pid_base, count)."""
    per = np_total // world
    extra = np_total % world
    base = rank * per + min(rank, extra)
    return base, per + (1 if rank < extra else 0)


def allreduce_sum(dist, arr, group=None):
    """Sum an integer or float numpy array over ranks (int64 / float64)."""
    import torch
    a = np.asarray(arr)
    t = torch.from_numpy(a.astype(np.int64 if a.dtype.kind in "iu" else np.float64))
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, group=group)
    return t.cpu().numpy()


def reduce_dose(dist, dose_u32, group=None):
    """Dose grids add per voxel; u32 arithmetic wraps as the single-device atomics do."""
    return (allreduce_sum(dist, dose_u32.astype(np.int64), group) & 0xFFFFFFFF).astype(np.uint32)


def sharded_score(dist, score_fn, rad_local, lcg_state, n_bp, group=None):
    """Exact sharded scoreDirectSSB_events.

    score_fn(rad, lcg_state) -> (hits uint8[2*n_bp], in_reach, candidates)
    scores one list from a fresh zero hit array."""
    import torch
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    _, n_r, cand = score_fn(rad_local, lcg_state)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    cnt = torch.tensor([int(n_r), int(cand)], dtype=torch.int64, device=dev)
    allc = [torch.zeros_like(cnt) for _ in range(world)]
    dist.all_gather(allc, cnt, group=group)
    counts = [int(c[0]) for c in allc]
    cands = [int(c[1]) for c in allc]
    offset = sum(counts[:rank])
    hits, n2, _ = score_fn(rad_local, lcg_jump(lcg_state, offset))
    assert n2 == n_r
    h = torch.from_numpy(np.ascontiguousarray(hits, dtype=np.uint8)).to(dev)
    dist.all_reduce(h, op=dist.ReduceOp.MAX, group=group)
    hits_all = h.cpu().numpy()
    ssb0 = int(np.count_nonzero(hits_all[:n_bp]))
    ssb1 = int(np.count_nonzero(hits_all[n_bp:]))
    total = sum(counts)
    return {"hits": hits_all, "ssb_count": ssb0 + ssb1, "ssb0": ssb0, "ssb1": ssb1, "in_reach": total,
            "candidates": sum(cands), "lcg_state": lcg_jump(lcg_state, total), "offset": offset}


# ---------------------------------------------------------------- device path
class _CudaArray:
    """A device buffer of the library seen by torch (zero copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def device_tensor(ptr, n, typestr, device):
    import torch
    return torch.as_tensor(_CudaArray(ptr, n, typestr), device=device)


def device_step_exchange(ctx, dist, lcg_state, device, irt_counts=None, group=None):
    """The exchange steps of a sharded pipeline step on the device, after every
    rank ran wgdna_transport (and wgdna_irt) on its block of primaries:

      * dose grid: NCCL sum (the u32 grid summed as int32 wraps the same way);
      * IRT checkpoint counts: sum;
      * direct SSB scoring, exactly as on one device: each rank scores its
        rad_buf once to learn its LCG draws, the draws are all-gathered,
        each rank scores again from the LCG state advanced past the lower ranks'
        draws, the hit bytes are MAX-reduced and every rank clusters DSBs on
        the combined hits.

    Returns (ssb, dsb, in_reach, counts) of the whole job."""
    import ctypes as C
    import numpy as np
    import torch
    from . import _lib
    L = _lib.lib()
    v = _lib.DeviceView()
    _lib.check("wgdna_device_views", L.wgdna_device_views(ctx.h, C.byref(v)))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dose = device_tensor(v.dose, v.dose_words, "<i4", device)
    dist.all_reduce(dose, group=group)
    counts = None
    if irt_counts is not None:
        t = torch.tensor(np.asarray(irt_counts, np.float64).reshape(-1), device=device)
        dist.all_reduce(t, group=group)
        counts = t.cpu().numpy()
    s1 = _lib.SsbResult()
    _lib.check("wgdna_score_draws", L.wgdna_score_draws(ctx.h, lcg_state, C.byref(s1)))
    n = torch.tensor([int(s1.in_reach)], dtype=torch.int64, device=device)
    alln = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(alln, n, group=group)
    draws = [int(x.item()) for x in alln]
    s2 = _lib.SsbResult()
    _lib.check("wgdna_score_draws", L.wgdna_score_draws(ctx.h, lcg_jump(lcg_state, sum(draws[:rank])), C.byref(s2)))
    hits = device_tensor(v.hits, v.hits_bytes, "|u1", device)
    dist.all_reduce(hits, op=dist.ReduceOp.MAX, group=group)
    d = _lib.DsbResult()
    _lib.check("wgdna_cluster_device", L.wgdna_cluster_device(ctx.h, C.byref(d)))
    return int(d.ssb0 + d.ssb1), int(d.dsb), sum(draws), counts
