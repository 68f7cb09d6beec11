#!/usr/bin/env python3
"""Benchmark: 10 keV primaries/s through transport + IRT + scoring on B200.

A step is one pass of the hot path over one batch: 4096 primary electrons at
10 keV in liquid water (box +-15 um, cutoff 7.5 eV, Philox key = seed), Phase A
+ B transport, rad_buf canonicalisation, IRT chemistry to 1 us, direct SSB
scoring and DSB clustering on the 21x21 B-DNA fibre grid.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

value    device time of K steps (CUDA events on the library's stream), inputs
         resident in HBM; L2 is flushed (256 MB write) between steps, outside
         the timed events.
e2e      the same work through the public host API with pinned host buffers:
         per-primary source energies uploaded, results / dose grid / rad_buf
         read back every step (runAtEnergy's contract), IRT + scoring results
         returned.
N > 1    one process per GPU (torchrun); each rank runs its own 4096 primaries
         (global ids rank*4096 + i, weak scaling); per-step summaries are
         all-reduced with NCCL; timing is the max over ranks.
--impl reference  times the CPU restatement of the reference's path (the
         oracle; the WebGPU shaders / JS worker cannot run here) on all host
         cores on a bounded sample per step.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "webgpu-dna_b200")]

METRIC = "10 keV primaries/s (transport+IRT+scoring)"
UNIT = "primaries/s"
NP = 4096
E_EV = 10000.0
WORKLOAD = ("4096 x 10 keV e- in liquid water, box +-15 um, cutoff 7.5 eV, Philox seed 0 -> "
            "IRT to 1 us -> direct SSB + DSB on 21x21 B-DNA fibres")
CPU_SAMPLE_PRIMARIES = 512
# library kernels per step: transport 1, rad_buf canonical order 5 (histogram,
# scan, scatter, segment sort, reduce), IRT 7 (segment max, load, scan,
# pairing, order, initial-event sort, events), scoring 5 (prep, tiles, tile
# scan, apply, cluster)
LAUNCHES_PER_STEP = 18


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 4 + k and r[4 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def cpu_reference_step(nthreads, sample, seed):
    """One bounded sample of the path on the host cores (the oracle)."""
    import numpy as np
    import oracle
    t0 = time.perf_counter()
    o = oracle.transport(sample, E_EV, seed=seed, rng_mode=0, dna_enable=1, nthreads=nthreads)
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    oracle.irt(o["rad"], nth, E_EV, seed=seed, nthreads=nthreads)
    oracle.score_direct(_odna(), o["rad"])
    return time.perf_counter() - t0


_ODNA = None


def _odna():
    global _ODNA
    if _ODNA is None:
        import oracle
        _ODNA = oracle.DnaTarget()
    return _ODNA


def run_reference(args, ws, rank):
    """The reference arm: the CPU restatement of the path (the oracle) on all
    host cores, each timed step the benchmark's whole workload (4096 x 10 keV,
    seed 0: transport, IRT, scoring); warm-up steps use 64 primaries.  A
    one-core figure on 64 primaries is reported beside it."""
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    for w in range(args.warmup):
        cpu_reference_step(nthreads, 64, 1000 + w)
    dts = [cpu_reference_step(nthreads, args.np, args.seed) for _ in range(args.steps)]
    t = sum(dts)
    value = args.np * args.steps / t
    one = 64 / cpu_reference_step(1, 64, args.seed)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 transport / f64 IRT", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD if args.np == NP else WORKLOAD.replace("4096", str(args.np)),
                       "np_per_gpu": args.np, "E_eV": E_EV, "seed": args.seed},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"the whole workload ({args.np} x 10 keV, seed {args.seed}) per step, "
                                       f"{args.steps} steps, through transport+IRT+scoring",
                             "single_core": {"value": one, "unit": UNIT, "cores": 1,
                                             "sample": "64 x 10 keV primaries, one thread"}},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


class Slot:
    """One pipeline slot: a library context on its own stream, its transport
    parameters (its own primary ids), an L2-flush buffer and pinned host
    buffers for the end-to-end path."""

    def __init__(self, i, NPr, rank, P, dev, args, dna):
        import ctypes as C
        import torch
        import wgdna
        from wgdna import _lib
        self.i = i
        self.ctx = wgdna.Context(max_primaries=NPr, device=dev.index, max_rad=max(NPr * 1600, 1_000_000),
                                 max_sec=max(NPr * 250, 100_000))
        self.stream = torch.cuda.Stream(device=dev)
        self.ctx.set_stream(self.stream.cuda_stream)
        if args.tuning:
            self.ctx.set_tuning(**dict(kv.split("=") for kv in args.tuning.split(",")))
        self.p = wgdna.transport_params(NPr, E_EV, 15000.0, 7.5, dna=dna, seed=args.seed, dna_enable=1)
        self.p.pid_base = (rank * P + i) * NPr
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        self.st, self.ir = _lib.TransportStats(), _lib.IrtResult()
        self.ssb, self.dsb = _lib.SsbResult(), _lib.DsbResult()
        self.E_host = torch.full((NPr,), E_EV, dtype=torch.float32, pin_memory=True)
        self.res_h = torch.empty(NPr * 8, dtype=torch.float32, pin_memory=True)
        self.dose_h = torch.empty(self.ctx.vc ** 3, dtype=torch.int32, pin_memory=True)
        self.rad_cap = self.ctx.max_rad
        self.rad_h = torch.empty(self.rad_cap * 4, dtype=torch.float32, pin_memory=True)
        self.p_e2e = wgdna.transport_params(NPr, E_EV, 15000.0, 7.5, dna=dna, seed=args.seed, dna_enable=1)
        self.p_e2e.pid_base = self.p.pid_base
        self.p_e2e.E_per_primary = self.E_host.data_ptr()
        self.rad_n = C.c_uint64()
        self.times = {k: [] for k in ("tr", "canon", "irt", "pair", "evl", "sort", "sc")}

    def record(self):
        self.times["tr"].append(self.st.ms_transport)
        self.times["canon"].append(self.st.ms_canon)
        self.times["irt"].append(self.ir.ms)
        self.times["pair"].append(self.ir.ms_pairing)
        self.times["evl"].append(self.ir.ms_events)
        self.times["sort"].append(self.ir.ms_sort)
        self.times["sc"].append(self.ssb.ms + self.dsb.ms)


def _run_threads(fns):
    """Run the callables concurrently (ctypes calls release the GIL); re-raise the first error."""
    errs = []

    def wrap(f):
        try:
            f()
        except BaseException as e:  # noqa: BLE001 - surfaced below
            errs.append(e)
    ts = [threading.Thread(target=wrap, args=(f,)) for f in fns]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]


def run_native(args, ws, rank, local):
    import ctypes as C
    import numpy as np
    import torch
    import wgdna
    from wgdna import _lib, sharded

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    NPr = args.np
    # batches in flight at once (one context, stream and host thread each); the
    # sharded exchange of a multi-GPU step runs collectives, so one slot there
    P = max(1, args.pipeline) if ws == 1 else 1
    dna = wgdna.build_dna_target()
    slots = [Slot(i, NPr, rank, P, dev, args, dna) for i in range(P)]
    ctx, stream, p = slots[0].ctx, slots[0].stream, slots[0].p
    job = {}

    def step_device(sl):
        _lib.check("wgdna_transport", L.wgdna_transport(sl.ctx.h, C.byref(sl.p), C.byref(sl.st)))
        _lib.check("wgdna_irt", L.wgdna_irt(sl.ctx.h, sl.st.n_therm, E_EV, args.seed + 1, C.byref(sl.ir)))
        if ws == 1:
            _lib.check("wgdna_score", L.wgdna_score(sl.ctx.h, 0x12345678, C.byref(sl.ssb), C.byref(sl.dsb)))
            return
        # exchange steps of the sharded job: dose grid and IRT counts summed, direct
        # SSB scored exactly as on one device (draw counts all-gathered, hits MAX-reduced)
        with torch.cuda.stream(sl.stream):
            job["ssb"], job["dsb"], job["reach"], job["counts"] = sharded.device_step_exchange(
                sl.ctx, torch.distributed, 0x12345678, dev,
                irt_counts=np.concatenate([np.array(sl.ir.counts).reshape(-1), [float(sl.st.n_therm)]]))

    e2e_bytes = {"h2d": 0, "d2h": 0}

    def step_e2e(sl):
        _lib.check("wgdna_run_transport",
                   L.wgdna_run_transport(sl.ctx.h, C.byref(sl.p_e2e), C.c_void_p(sl.res_h.data_ptr()),
                                         C.c_void_p(sl.dose_h.data_ptr()), C.c_void_p(sl.rad_h.data_ptr()),
                                         sl.rad_cap, C.byref(sl.rad_n), C.byref(sl.st)))
        _lib.check("wgdna_irt", L.wgdna_irt(sl.ctx.h, sl.st.n_therm, E_EV, args.seed + 1, C.byref(sl.ir)))
        _lib.check("wgdna_score", L.wgdna_score(sl.ctx.h, 0x12345678, C.byref(sl.ssb), C.byref(sl.dsb)))
        e2e_bytes["h2d"] = NPr * 4 + C.sizeof(sl.p_e2e)
        e2e_bytes["d2h"] = (NPr * 32 + sl.ctx.vc ** 3 * 4 + min(sl.rad_n.value, sl.rad_cap) * 16 + C.sizeof(sl.st) +
                            C.sizeof(sl.ir) + C.sizeof(sl.ssb) + C.sizeof(sl.dsb))

    # batch k runs on slot k % P
    share = [len(range(i, args.steps, P)) for i in range(P)]
    for sl in slots:
        for _ in range(args.warmup):
            step_device(sl)
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    launches = LAUNCHES_PER_STEP * args.steps
    with Clocks(local) as clk:
        barrier()
        if P == 1:
            sl = slots[0]
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
            for k in range(args.steps):
                with torch.cuda.stream(stream):
                    sl.flush.fill_(float(k))
                    ev[k][0].record(stream)
                step_device(sl)
                with torch.cuda.stream(stream):
                    ev[k][1].record(stream)
                sl.record()
            barrier()
            tot_ms = sum(a.elapsed_time(b) for a, b in ev)
        else:
            # one start event; every slot's stream waits for it, then runs its
            # batches (L2 flush, transport, IRT, scoring) from its own thread
            t_start = torch.cuda.Event(enable_timing=True)
            ends = [torch.cuda.Event(enable_timing=True) for _ in slots]
            t_start.record(slots[0].stream)
            for sl in slots[1:]:
                sl.stream.wait_event(t_start)

            def run(sl):
                def f():
                    for k in range(share[sl.i]):
                        with torch.cuda.stream(sl.stream):
                            sl.flush.fill_(float(k))
                        step_device(sl)
                        sl.record()
                    ends[sl.i].record(sl.stream)
                return f
            _run_threads([run(sl) for sl in slots])
            barrier()
            tot_ms = max(t_start.elapsed_time(e) for e in ends)
        barrier()
    if ws > 1:
        t = torch.tensor([tot_ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        tot_ms = float(t.item())
    value = ws * NPr * args.steps / (tot_ms / 1000.0)

    # end-to-end through the public host API (the slots' host threads, as above)
    for sl in slots:
        for _ in range(2):
            step_e2e(sl)
    barrier()
    t0 = time.perf_counter()
    if P == 1:
        for _ in range(args.steps):
            step_e2e(slots[0])
    else:
        _run_threads([(lambda sl=sl: [step_e2e(sl) for _ in range(share[sl.i])]) for sl in slots])
    barrier()
    e2e_s = time.perf_counter() - t0
    if ws > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = ws * NPr * args.steps / e2e_s
    st, ir, ssb, dsb = slots[0].st, slots[0].ir, slots[0].ssb, slots[0].dsb
    tt = {k: sum((sl.times[k] for sl in slots), []) for k in slots[0].times}
    t_tr, t_canon, t_irt, t_pair, t_evl, t_sort, t_sc = (tt[k] for k in ("tr", "canon", "irt", "pair", "evl",
                                                                        "sort", "sc"))

    physics = physics_fields(ctx, L, p, NPr) if rank == 0 else None
    # the second half of the metric: the learned chemistry against the IRT
    # (trained in this run by the library's kernels; untimed by the step clock)
    surrogate = surrogate_block(ctx, 3, 1) if ws == 1 and not args.no_surrogate else None
    # the other workloads of the benchmark table, untimed by the step clock:
    # one synthetic track (C1), mixed energies (C3), the DNA-damage sweep (C5,
    # on the network the surrogate block trained)
    workloads = None
    if ws == 1 and not args.no_workloads:
        workloads = {"track": track_block(), "mixed": mixed_block()}
        if surrogate is not None:
            workloads["sweep"] = sweep_block(ctx, args.sweep_n)

    # roofline of the dominant kernel: algorithmic bytes per launch / its mean duration
    pk = peaks()
    mean = lambda a: sum(a) / len(a)
    stages = {"irt": mean(t_irt), "transport": mean(t_tr), "canon": mean(t_canon), "scoring": mean(t_sc)}
    kernels = {"k_transport": mean(t_tr), "k_irt_init": mean(t_pair), "k_irt_loop": mean(t_evl),
               "k_track_order+k_irt_sort": mean(t_sort)}
    dom = max(("k_transport", "k_irt_init", "k_irt_loop"), key=kernels.get)
    R, S, D = st.rad_n_stored, st.sec_n, st.dbg[5]
    Np, Ei, Et = ir.n_particles, ir.n_init_events, ir.n_events
    alg = {
        # rad_buf 16 B/entry, secondaries pushed + popped 48 B each, R struct 32 B, dose atomics 4 B
        "k_transport": 16 * R + 96 * S + 32 * NPr + 4 * D,
        # tracked species (x, y, z f64 + species) read once, initial events (t f64, ids u32) written once
        "k_irt_init": 25 * Np + 12 * Ei,
        # initial events read once, species state read, product events pushed and popped
        "k_irt_loop": 12 * Ei + 25 * Np + 24 * max(Et - Ei, 0),
    }[dom]
    achieved = alg / (kernels[dom] / 1000.0) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            t = json.load(open(tf)).get(dom)
            # dram bytes per full launch, scaled from the profiled case by the units processed
            if t:
                unit = {"k_transport": NPr, "k_irt_init": Np, "k_irt_loop": Np}[dom]
                traffic = t["bytes_per_unit"] * unit
        except Exception:
            traffic = None
    clocks = clk.summary()
    # the binding resource of these kernels is issue slots (divergent Monte
    # Carlo and f64 event chains, not bytes): warp instructions per launch (from
    # one ncu capture, per unit processed, profiles/issue.json) / (duration x SM
    # clock x SMs) against 4 warp instructions per cycle per SM
    issue = None
    isf = os.path.join(ROOT, "profiles", "issue.json")
    if os.path.exists(isf):
        try:
            t = json.load(open(isf)).get(dom)
            if t:
                unit = {"k_transport": NPr, "k_irt_init": Np, "k_irt_loop": Np}[dom]
                inst = t["inst_per_unit"] * unit
                mhz = clocks.get("sm_mhz") or 1965.0
                sms = torch.cuda.get_device_properties(dev).multi_processor_count
                ach = inst / (kernels[dom] / 1000.0) / (mhz * 1e6) / sms
                issue = {"achieved": ach, "peak": 4.0, "unit": "warp instructions / cycle / SM", "frac": ach / 4.0,
                         "inst_per_launch": inst, "sm_mhz": mhz, "sms": sms, "source": "profiles/issue.json"}
        except Exception:
            issue = None
    hbm = {"achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
           "traffic": traffic, "alg_bytes": int(alg), "peak_source": "fallback" if pk.get("fallback") else "measured"}
    if issue is not None:
        roofline = {"bound": "issue", "kernel": dom, "achieved": issue["achieved"], "peak": issue["peak"],
                    "unit": issue["unit"], "frac": issue["frac"], "traffic": traffic, "issue": issue, "hbm": hbm}
    else:
        roofline = {"bound": "hbm", "kernel": dom, **hbm}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 transport / f64 IRT", "data": "synthetic",
            "config": {"workload": WORKLOAD if NPr == NP else WORKLOAD.replace("4096", str(NPr)),
                       "np_per_gpu": NPr, "E_eV": E_EV, "seed": args.seed,
                       "l2": ("256 MB write before each batch (outside the events)" if P == 1 else
                              "256 MB write before each batch, inside the timed span"),
                       "parallelism": f"primary shards x{ws}",
                       "pipeline": (f"{P} batches in flight (one context, stream and host thread each; batch k on "
                                    f"slot k mod {P}); value = all batches' primaries / the span from the first "
                                    f"batch's start to the last one's end, each batch's L2 flush inside it")
                       if P > 1 else "batches one after another",
                       **({"tuning": args.tuning} if args.tuning else {})},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": e2e_bytes["h2d"],
                    "d2h_bytes_per_step": e2e_bytes["d2h"]},
            "gpu_launches": launches,
            "stage_ms": {k: round(v, 4) for k, v in stages.items()},
            "kernel_ms": {k: round(v, 4) for k, v in kernels.items()},
            "roofline": roofline,
            "clocks": clocks,
            "physics": physics,
            "surrogate": surrogate,
            "workloads": workloads,
            "job": {"ssb": job.get("ssb"), "dsb": job.get("dsb"), "in_reach": job.get("reach")} if ws > 1 else None,
            "work": {"rad_n": int(R), "sec_n": int(S), "steps": int(st.steps), "irt_pairs": int(ir.n_pairs),
                     "irt_events": int(ir.n_events), "irt_init_events": int(Ei), "irt_species": int(Np),
                     "dose_atomics": int(D), "ssb": int(ssb.ssb), "dsb": int(dsb.dsb)},
        }
        if ws == 1 and not args.no_cpu:
            nthreads = os.cpu_count() or 1
            cpu_reference_step(nthreads, 64, 99)
            dt = cpu_reference_step(nthreads, CPU_SAMPLE_PRIMARIES, 7)
            one = 64 / cpu_reference_step(1, 64, 7)
            line["cpu_baseline"] = {"value": CPU_SAMPLE_PRIMARIES / dt, "unit": UNIT, "cores": nthreads,
                                    "kind": "port",
                                    "sample": f"{CPU_SAMPLE_PRIMARIES} x 10 keV primaries through "
                                              f"transport+IRT+scoring (oracle, {nthreads} threads)",
                                    "single_core": {"value": one, "unit": UNIT, "cores": 1,
                                                    "sample": "64 x 10 keV primaries, one thread"}}
        print(json.dumps(line), flush=True)
    for sl in slots:
        sl.ctx.close()


PUBLISHED_10KEV = os.path.join(ROOT, "tests", "golden", "reference_outputs.json")


def physics_fields(ctx, L, p, npr):
    """The physics of one more (untimed) step of the same workload, against the
    reference's published 10 keV run (validation/webgpu-results.json:6-30):
    CSDA, ions per primary, initial G, G(1 us), SSB_dir, DSB, kernel hits, each
    with z = (ours - published) / sigma, sigma = the per-track standard
    deviation times sqrt(1/n + 1/4096) (Poisson for SSB_dir and DSB)."""
    import ctypes as C
    import numpy as np
    from wgdna import _lib
    pub = json.load(open(PUBLISHED_10KEV))["webgpu_10keV"]
    st, ir, ssb, dsb = _lib.TransportStats(), _lib.IrtResult(), _lib.SsbResult(), _lib.DsbResult()
    _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
    res = np.zeros(npr * 8, np.float32)
    rad = np.zeros((st.rad_n_stored, 4), np.float32)
    n = C.c_uint64()
    _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, _lib.ptr(res), None, _lib.ptr(rad), st.rad_n_stored,
                                                       C.byref(n)))
    L.wgdna_irt_record_curves(ctx.h, 1)
    try:
        _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, E_EV, 1 + p.seed, C.byref(ir)))
        cv = np.zeros((npr, 16, 5), np.float32)
        _lib.check("wgdna_irt_curves", L.wgdna_irt_curves(ctx.h, _lib.ptr(cv), npr, C.byref(n)))
    finally:
        L.wgdna_irt_record_curves(ctx.h, 0)
    _lib.check("wgdna_score", L.wgdna_score(ctx.h, 0x12345678, C.byref(ssb), C.byref(dsb)))
    r = res.reshape(-1, 8)
    ru = r.view(np.uint32)
    th = ru[:, 5] == 0
    nth = int(th.sum())
    f = math.sqrt(1.0 / max(nth, 1) + 1.0 / 4096)
    out = {"n_therm": nth, "e_conservation": st.dep_units / 100.0 / (nth * E_EV) if nth else None}

    def put(name, val, ref, sig):
        out[name] = {"value": round(float(val), 4), "published": ref,
                     "z": round(float((val - ref) / sig), 3) if sig > 0 else None}

    path, ions = r[th, 0].astype(np.float64), ru[th, 3].astype(np.float64)
    put("csda_nm", path.mean(), pub["tracking"]["csdaNm"], path.std() * f)
    put("ions_per_primary", ions.mean(), pub["tracking"]["ionsPerPriPrimaryOnly"], ions.std() * f)
    per100 = st.dep_units / 1e4
    w = np.rint(rad[:, 3]).astype(np.int64)
    pid, code = w >> 3, w & 7
    for k, name, codes in ((0, "G_OH_init", [0]), (1, "G_eaq_init", [1, 5]), (2, "G_H_init", [2])):
        cnt = np.bincount(pid[np.isin(code, codes)], minlength=npr).astype(np.float64)
        put(name, st.counters[k] / per100, pub["pre_chemistry"][name], cnt.std() / 100.0 * f)
    per_track = cv[:, 15, :].astype(np.float64) / (E_EV / 100.0)
    for j, sp in enumerate(("G_OH", "G_eaq", "G_H", "G_H2O2", "G_H2")):
        put(sp + "_1us", ir.G[6][j], pub["chemistry_1us"][sp], per_track[:, j].std() * f)
    d = pub["dna_damage"]
    for name, got, ref in (("SSB_dir", ssb.ssb, d["SSB_dir"]), ("DSB", dsb.dsb, d["DSB"])):
        put(name, got, ref, math.sqrt(got + ref))
    out["kernel_hits"] = {"value": int(st.counters[4]), "published": d["kernelHits"]}
    zs = [abs(v["z"]) for v in out.values() if isinstance(v, dict) and v.get("z") is not None]
    out["max_abs_z"] = max(zs) if zs else None
    out["source"] = ("published: validation/webgpu-results.json:6-30 (4096 x 10 keV, cutoff 7.4 eV, the "
                     "reference's own generator); ours: one untimed step of this workload")
    return out


def _irt_alg_bytes(ir):
    """Algorithmic bytes of the dominant IRT kernel (species read once, events written / read once)."""
    if ir.ms_pairing >= ir.ms_events:
        return "k_irt_init", ir.ms_pairing, 25 * ir.n_particles + 12 * ir.n_init_events
    return "k_irt_loop", ir.ms_events, 12 * ir.n_init_events + 25 * ir.n_particles + \
        24 * max(ir.n_events - ir.n_init_events, 0)


def run_track(args):
    """Single synthetic 10 keV-like track (510 spurs x 6 species, 2.7 um walk) through
    the IRT to 1 us: rad_buf from pinned host memory, counts back to the host."""
    import ctypes as C
    import numpy as np
    import torch
    import oracle
    import wgdna
    from wgdna import _lib, synthetic
    L = _lib.lib()
    ctx = wgdna.Context(max_primaries=16, max_rad=1_000_000, max_sec=100_000)
    rad = synthetic.synthetic_track()
    rad_h = torch.from_numpy(rad).pin_memory()
    ir = _lib.IrtResult()

    def step():
        _lib.check("wgdna_run_irt", L.wgdna_run_irt(ctx.h, C.c_void_p(rad_h.data_ptr()), rad.shape[0], 1, 1e4, 1,
                                                    C.byref(ir)))
    for _ in range(args.warmup):
        step()
    dev_ms, kern = [], []
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
            dev_ms.append(ir.ms)
            kern.append(_irt_alg_bytes(ir))
        wall = time.perf_counter() - t0
    ms = sum(dev_ms) / len(dev_ms)
    name, kms, alg = kern[-1]
    pk = peaks()
    nthreads = 1
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        oracle.irt(rad, 1, 1e4, seed=1, nthreads=nthreads)
    cpu = reps / (time.perf_counter() - t0)
    line = {"metric": "single-track IRT to 1 us (2550 species)", "value": 1000.0 / ms, "unit": "tracks/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "none", "vs_baseline": None, "dtype": "f64 IRT", "data": "synthetic",
            "config": {"workload": "one synthetic track: 510 spurs of OH, e-aq, H3O+, H, H2, OH- "
                                   "(sigma U[1,2] nm) on a 2.7 um random walk, Philox key 1; IRT to 1 us",
                       "species": synthetic.tracked_species(rad), "l2": "input far below L2 (one track)"},
            "e2e": {"value": args.steps / wall, "unit": "tracks/s", "h2d_bytes_per_step": int(rad.nbytes),
                    "d2h_bytes_per_step": C.sizeof(ir)},
            "gpu_launches": 9 * (args.steps),
            "roofline": {"bound": "hbm", "kernel": name, "achieved": alg / (kms / 1000.0) / 1e9,
                         "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": alg / (kms / 1000.0) / 1e9 / pk["hbm_gbs"],
                         "traffic": None},
            "clocks": clk.summary(),
            "work": {"pairs": int(ir.n_pairs), "events": int(ir.n_events), "reacted": int(ir.n_reacted)},
            "cpu_baseline": {"value": cpu, "unit": "tracks/s", "cores": nthreads, "kind": "port",
                             "sample": "the same track, oracle IRT on one thread (the reference worker is "
                                       "single-threaded)"}}
    print(json.dumps(line), flush=True)
    ctx.close()


MIXED_N = 65536


def run_mixed(args):
    """65,536 primaries, energies log-uniform over 100 eV - 30 keV, in one transport
    launch, then the IRT over all tracks (species counts from a few to ~4000)."""
    import ctypes as C
    import numpy as np
    import oracle
    import wgdna
    from wgdna import _lib, synthetic
    L = _lib.lib()
    N = args.np if args.np != NP else MIXED_N
    E = synthetic.mixed_energies(N)
    ctx = wgdna.Context(max_primaries=N, max_rad=max(N * 1100, 1_000_000), max_sec=max(N * 130, 100_000))
    import torch
    E_h = torch.from_numpy(E).pin_memory()
    p = wgdna.transport_params(N, 10000.0, 15000.0, 7.5, seed=args.seed, dna_enable=0)
    p.E_per_primary = E_h.data_ptr()
    st, ir = _lib.TransportStats(), _lib.IrtResult()
    Emean = float(np.mean(E.astype(np.float64)))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)

    def step():
        _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
        _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, Emean, args.seed + 1, C.byref(ir)))
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kt, ki = [], []
    with Clocks(0) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
                ev[k][0].record(stream)
            step()
            with torch.cuda.stream(stream):
                ev[k][1].record(stream)
            kt.append(st.ms_transport)
            ki.append(_irt_alg_bytes(ir))
        torch.cuda.synchronize()
    tot = sum(a.elapsed_time(b) for a, b in ev)
    value = N * args.steps / (tot / 1000.0)
    pk = peaks()
    name, kms, alg = ki[-1]
    R, S, D = st.rad_n_stored, st.sec_n, st.dbg[5]
    if sum(kt) / len(kt) > kms:
        name, kms, alg = "k_transport", sum(kt) / len(kt), 16 * R + 96 * S + 32 * N + 4 * D
    sample = 1024
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    o = oracle.transport(sample, 10000.0, seed=7, rng_mode=0, dna_enable=0, E_per_primary=E[:sample],
                         nthreads=nthreads)
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    oracle.irt(o["rad"], nth, Emean, seed=7, nthreads=nthreads)
    cpu = sample / (time.perf_counter() - t0)
    # per species-count bucket: the IRT alone on the tracks of that bucket (host rad_buf
    # of the same transport, re-run through wgdna_run_irt); results per track do not
    # depend on which other tracks share the launch
    rad = np.empty(st.rad_n_stored * 4, np.float32)
    rn = C.c_uint64()
    _lib.check("wgdna_transport_copy_out", L.wgdna_transport_copy_out(ctx.h, None, None, _lib.ptr(rad),
                                                                      st.rad_n_stored, C.byref(rn)))
    rad = rad[:4 * min(rn.value, st.rad_n_stored)].reshape(-1, 4)
    w = rad[:, 3].astype(np.int64)
    pid, code = w >> 3, w & 7
    tracked = np.bincount(pid[code != 7], minlength=N)
    buckets = []
    edges = (1, 100, 500, 1000, 2000, 5000, 1 << 30)
    irb = _lib.IrtResult()
    for lo, hi in zip(edges[:-1], edges[1:]):
        sel = np.nonzero((tracked >= lo) & (tracked < hi))[0]
        if sel.size == 0:
            continue
        sub = np.ascontiguousarray(rad[np.isin(pid, sel)])
        ms = []
        for k in range(3):
            _lib.check("wgdna_run_irt", L.wgdna_run_irt(ctx.h, _lib.ptr(sub), sub.shape[0], int(sel.size), Emean,
                                                        args.seed + 1, C.byref(irb)))
            ms.append(irb.ms)
        ms = sorted(ms)[1]
        buckets.append({"species": f"{lo}-{hi - 1}" if hi < (1 << 30) else f">={lo}", "tracks": int(sel.size),
                        "irt_species": int(irb.n_particles), "pairs": int(irb.n_pairs), "events": int(irb.n_events),
                        "irt_ms": round(ms, 3), "pairs_per_s": irb.n_pairs / (ms / 1000.0)})
    line = {"metric": "mixed-energy primaries/s (transport+IRT)", "value": value, "unit": "primaries/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 transport / f64 IRT",
            "data": "synthetic",
            "config": {"workload": f"{N} primaries, E log-uniform 100 eV - 30 keV (Philox key 3), one transport "
                                   "launch, IRT to 1 us over all tracks", "np": N,
                       "l2": "256 MB write between timed steps"},
            "stage_ms": {"transport": sum(kt) / len(kt), "irt_init": ir.ms_pairing, "irt_loop": ir.ms_events},
            "roofline": {"bound": "hbm", "kernel": name, "achieved": alg / (kms / 1000.0) / 1e9,
                         "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": alg / (kms / 1000.0) / 1e9 / pk["hbm_gbs"],
                         "traffic": None},
            "clocks": clk.summary(),
            "work": {"rad_n": int(R), "sec_n": int(S), "tracks": int(ir.n_tracks), "irt_species": int(ir.n_particles),
                     "irt_pairs": int(ir.n_pairs), "irt_events": int(ir.n_events)},
            "irt_buckets": buckets,
            "cpu_baseline": {"value": cpu, "unit": "primaries/s", "cores": nthreads, "kind": "port",
                             "sample": f"first {sample} primaries of the same energy list, oracle transport + IRT"}}
    print(json.dumps(line), flush=True)
    ctx.close()


def track_block(steps=5, warmup=2):
    """C1 in the default line: one synthetic 10 keV-like track (510 spurs x 6
    species on a 2.7 um walk) through the IRT to 1 us from pinned host memory;
    device ms per track and the oracle's one-thread time on the same track."""
    import ctypes as C
    import torch
    import oracle
    import wgdna
    from wgdna import _lib, synthetic
    L = _lib.lib()
    ctx = wgdna.Context(max_primaries=16, max_rad=1_000_000, max_sec=100_000)
    try:
        rad = synthetic.synthetic_track()
        rad_h = torch.from_numpy(rad).pin_memory()
        ir = _lib.IrtResult()
        ms = []
        for k in range(warmup + steps):
            _lib.check("wgdna_run_irt", L.wgdna_run_irt(ctx.h, C.c_void_p(rad_h.data_ptr()), rad.shape[0], 1, 1e4, 1,
                                                        C.byref(ir)))
            if k >= warmup:
                ms.append(ir.ms)
        t0 = time.perf_counter()
        oracle.irt(rad, 1, 1e4, seed=1, nthreads=1)
        cpu_s = time.perf_counter() - t0
        m = sum(ms) / len(ms)
        return {"workload": "one synthetic track, 510 spurs x 6 species (2550 tracked) on a 2.7 um walk, IRT to 1 us",
                "ms_per_track": round(m, 4), "tracks_per_s": round(1000.0 / m, 2), "pairs": int(ir.n_pairs),
                "events": int(ir.n_events), "reacted": int(ir.n_reacted),
                "cpu_one_thread_s": round(cpu_s, 4), "speedup_vs_one_thread": round(cpu_s * 1000.0 / m, 1)}
    finally:
        ctx.close()


def mixed_block(steps=2, warmup=1, seed=0):
    """C3 in the default line: 65,536 primaries, E log-uniform 100 eV - 30 keV,
    one transport launch, the IRT over all tracks; then the IRT alone on each
    species-count bucket's tracks (pairs per second per bucket)."""
    import ctypes as C
    import numpy as np
    import torch
    import wgdna
    from wgdna import _lib, synthetic
    L = _lib.lib()
    N = MIXED_N
    E = synthetic.mixed_energies(N)
    ctx = wgdna.Context(max_primaries=N, max_rad=max(N * 1100, 1_000_000), max_sec=max(N * 130, 100_000))
    try:
        E_h = torch.from_numpy(E).pin_memory()
        p = wgdna.transport_params(N, 10000.0, 15000.0, 7.5, seed=seed, dna_enable=0)
        p.E_per_primary = E_h.data_ptr()
        st, ir = _lib.TransportStats(), _lib.IrtResult()
        Emean = float(np.mean(E.astype(np.float64)))
        tr, pa, ev, tot = [], [], [], []
        for k in range(warmup + steps):
            _lib.check("wgdna_transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
            _lib.check("wgdna_irt", L.wgdna_irt(ctx.h, st.n_therm, Emean, seed + 1, C.byref(ir)))
            if k >= warmup:
                tr.append(st.ms_transport)
                pa.append(ir.ms)
                tot.append(st.ms_transport + st.ms_canon + ir.ms)
        rad = np.empty(st.rad_n_stored * 4, np.float32)
        rn = C.c_uint64()
        _lib.check("copy_out", L.wgdna_transport_copy_out(ctx.h, None, None, _lib.ptr(rad), st.rad_n_stored,
                                                           C.byref(rn)))
        rad = rad[:4 * min(rn.value, st.rad_n_stored)].reshape(-1, 4)
        w = rad[:, 3].astype(np.int64)
        pid, code = w >> 3, w & 7
        tracked = np.bincount(pid[code != 7], minlength=N)
        buckets = []
        irb = _lib.IrtResult()
        edges = (1, 100, 500, 1000, 2000, 5000, 1 << 30)
        for lo, hi in zip(edges[:-1], edges[1:]):
            sel = np.nonzero((tracked >= lo) & (tracked < hi))[0]
            if sel.size == 0:
                continue
            sub = np.ascontiguousarray(rad[np.isin(pid, sel)])
            _lib.check("wgdna_run_irt", L.wgdna_run_irt(ctx.h, _lib.ptr(sub), sub.shape[0], int(sel.size), Emean,
                                                        seed + 1, C.byref(irb)))
            buckets.append({"species": f"{lo}-{hi - 1}" if hi < (1 << 30) else f">={lo}", "tracks": int(sel.size),
                            "irt_ms": round(irb.ms, 3), "pairs_per_s": irb.n_pairs / (irb.ms / 1000.0)})
        m = sum(tot) / len(tot)
        return {"workload": f"{N} primaries, E log-uniform 100 eV - 30 keV, one transport launch, IRT to 1 us "
                            "over all tracks",
                "primaries_per_s": round(N / (m / 1000.0), 1), "ms_per_step": round(m, 3),
                "transport_ms": round(sum(tr) / len(tr), 3), "irt_ms": round(sum(pa) / len(pa), 3),
                "tracks": int(ir.n_tracks), "irt_species": int(ir.n_particles), "irt_buckets": buckets}
    finally:
        ctx.close()


SURROGATE_ENERGIES = (1000.0, 3000.0, 10000.0)


def surrogate_block(ctx, steps, warmup, train_batches=None):
    """The learned chemistry against the IRT it replaces, on held-out 4096-track
    batches at 1, 3 and 10 keV: the network is trained here, by the library's
    own tcgen05 kernels, on ~2e5 IRT tracks (train_batches x 4096 per energy,
    wgdna.surrogate.train_on_irt).  Per batch (wgdna.surrogate.held_out): one
    transport, the IRT with per-track curves, four runs with different seeds
    on the same tracks (their mean is the reference G(t) at the 16 curve
    times), the plain batched IRT timed on its own, and the surrogate
    chemistry timed on the same tracks (CUDA events of each call).  Errors: the
    largest relative error of the batch G over 5 species x 16 times (where
    G > 0.05) and at 1 us."""
    import numpy as np
    from wgdna import surrogate as S
    train = S.train_on_irt(ctx, train_batches or S.TRAIN_BATCHES)
    per_E = {}
    for E in SURROGATE_ENERGIES:
        t_irt, t_sg, e1, eall, gis, gcs = [], [], [], [], [], []
        for k in range(warmup + steps):
            gi, gc, irt_ms, sg_ms, _ = S.held_out(ctx, E, 777 + 13 * k + int(E))
            if k >= warmup:
                t_irt.append(irt_ms)
                t_sg.append(sg_ms)
                a, b = S.g_errors(gi, gc)
                e1.append(a)
                eall.append(b)
                gis.append(gi)
                gcs.append(gc)
        # the held-out batches pooled (same tracks for both paths): the IRT's
        # own sampling noise shrinks, the surrogate's bias does not
        gi, gc = np.mean(gis, axis=0), np.mean(gcs, axis=0)
        p1, pall = S.g_errors(gi, gc)
        rel = np.abs(gc - gi) / np.maximum(np.abs(gi), 1e-12)
        rel[gi <= 0.05] = 0.0
        kt, ks = np.unravel_index(int(np.argmax(rel)), rel.shape)
        per_E[int(E)] = {"irt_ms": round(sum(t_irt) / len(t_irt), 4),
                         "surrogate_ms": round(sum(t_sg) / len(t_sg), 4),
                         "speedup": round(sum(t_irt) / sum(t_sg), 2),
                         "G_err_1us": round(p1, 5), "G_err_max": round(pall, 5),
                         "G_err_max_at": {"t_ns": float(S.TIMES_NS[kt]), "species": S.SPECIES[ks],
                                          "G_irt": round(float(gi[kt, ks]), 4), "G_surrogate": round(float(gc[kt, ks]), 4)},
                         "G_err_max_single_batch": round(max(eall), 5), "G_err_1us_single_batch": round(max(e1), 5),
                         "tracks_compared": 4096 * len(gis)}
    return {"per_energy": per_E,
            "min_speedup": min(v["speedup"] for v in per_E.values()),
            "max_G_err": max(v["G_err_max"] for v in per_E.values()),
            "training": train,
            "method": "MLP 64-128-128-128-80 GELU, bf16 weights / f32 accumulate (tcgen05), trained in this run "
                      "on the IRT's per-track G(t); speedup = batched IRT device time / surrogate device time "
                      "(descriptors + forward with fused reduction) on the same held-out 4096-track batches"}


def run_surrogate(args):
    """The surrogate block alone (see surrogate_block), with the CPU oracle's IRT
    beside it."""
    import numpy as np
    import oracle
    import wgdna
    ctx = wgdna.Context(max_primaries=4096, max_rad=8_000_000, max_sec=1_200_000)
    pk = peaks()
    with Clocks(0) as clk:
        blk = surrogate_block(ctx, args.steps, args.warmup)
    nthreads = os.cpu_count() or 1
    o = oracle.transport(256, 10000.0, seed=3, rng_mode=0, dna_enable=0, nthreads=nthreads)
    nth = int((o["results"].view(np.uint32).reshape(-1, 8)[:, 5] == 0).sum())
    t0 = time.perf_counter()
    oracle.irt(o["rad"], nth, 10000.0, seed=3, nthreads=nthreads)
    cpu = 256 / (time.perf_counter() - t0)
    r10 = blk["per_energy"][10000]
    line = {"metric": "surrogate vs IRT chemistry speedup (min over 1, 3, 10 keV; G error <= 2%)",
            "value": blk["min_speedup"], "unit": "x", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r10["surrogate_ms"], "higher_is_better": True, "scaling": "none", "vs_baseline": None,
            "dtype": "bf16 weights / f32 accumulate (surrogate), f64 (IRT)", "data": "synthetic",
            "config": {"workload": "4096-track batches at 1, 3, 10 keV; MLP 64-128-128-128-80 GELU trained on "
                                   "the IRT's per-track G(t) at 16 times (1 ps - 1 us)", "training": blk["training"]},
            "per_energy": blk["per_energy"], "max_G_err": blk["max_G_err"],
            "e2e": {"value": 4096 / (r10["surrogate_ms"] / 1000.0), "unit": "tracks/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 81 * 8},
            "gpu_launches": 2 * args.steps * 3,
            "roofline": {"bound": "hbm", "kernel": "k_descriptors", "achieved": None, "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": None, "traffic": None},
            "clocks": clk.summary(),
            "cpu_baseline": {"value": cpu, "unit": "tracks/s", "cores": nthreads, "kind": "port",
                             "sample": "oracle IRT on 256 tracks of a 10 keV batch (the chemistry the surrogate replaces)"}}
    print(json.dumps(line), flush=True)
    ctx.close()


def sweep_block(ctx, n_per=1_000_000, B=4096, energies=(1000.0, 3000.0, 10000.0)):
    """C5: n_per primaries at each energy in batches of B through transport,
    the surrogate chemistry (the context's trained network; the IRT checks 1 %
    of the batches) and direct SSB + DSB scoring (10 bp window) on the 21 x 21
    fibre grid; yields per Gy and per primary, device and wall throughput."""
    import ctypes as C
    import numpy as np
    import wgdna
    from wgdna import _lib
    L = _lib.lib()
    dna = wgdna.build_dna_target()
    box = 15000.0
    mass_kg = ((2 * box * 1e-9) ** 3) * 1000.0
    rows = {}
    stream_ms = wall_all = 0.0
    for E in energies:
        nb = (n_per + B - 1) // B
        st, ssb, dsb = _lib.TransportStats(), _lib.SsbResult(), _lib.DsbResult()
        ir = _lib.IrtResult()
        dep = 0.0
        n_ssb = n_dsb = 0
        checks = []
        Gsum = np.zeros(80)
        ms_tr = ms_sg = ms_sc = 0.0
        t0 = time.perf_counter()
        for b in range(nb):
            n = min(B, n_per - b * B)
            p = wgdna.transport_params(n, E, box, 7.5, dna=dna, seed=int(E) * 1000 + b, dna_enable=1)
            p.pid_base = b * B
            _lib.check("transport", L.wgdna_transport(ctx.h, C.byref(p), C.byref(st)))
            Gc = np.zeros(80)
            ms = C.c_float()
            _lib.check("chem", L.wgdna_surrogate_chemistry(ctx.h, _lib.ptr(Gc), C.byref(ms)))
            if b % 100 == 50 or nb < 100 and b == nb // 2:                      # the IRT checks 1 %
                L.wgdna_irt_record_curves(ctx.h, 1)
                _lib.check("irt", L.wgdna_irt(ctx.h, st.n_therm, E, b + 1, C.byref(ir)))
                L.wgdna_irt_record_curves(ctx.h, 0)
                # 1 ps, 100 ps, 10 ns and 1 us are both IRT checkpoints and curve times
                gi = np.array(ir.G)[[0, 2, 4, 6]]
                gs = Gc.reshape(16, 5)[[0, 5, 10, 15]]
                checks.append(float((np.abs(gs - gi) / np.maximum(gi, 1e-12))[gi > 0.05].max()))
            _lib.check("score", L.wgdna_score(ctx.h, 0x12345678, C.byref(ssb), C.byref(dsb)))
            dep += st.dep_eV_f64
            n_ssb += ssb.ssb
            n_dsb += dsb.dsb
            Gsum += Gc * n * E
            ms_tr += st.ms_transport
            ms_sg += ms.value
            ms_sc += ssb.ms + dsb.ms
        wall = time.perf_counter() - t0
        dose = dep * 1.602e-19 / mass_kg
        gbp = dna.n_bp * 1e-9
        rows[int(E)] = {"primaries": n_per, "batches": nb, "dose_Gy": dose,
                        "SSB_per_primary": n_ssb / n_per, "DSB_per_primary": n_dsb / n_per,
                        "DSB_per_Gy_Gbp": n_dsb / (dose * gbp) if dose > 0 else 0.0,
                        "SSB_per_Gy_Gbp": n_ssb / (dose * gbp) if dose > 0 else 0.0,
                        "G_1us": [round(float(v), 4) for v in (Gsum / (n_per * E)).reshape(16, 5)[15]],
                        "irt_check_max_rel_err": max(checks) if checks else None, "irt_checked_batches": len(checks),
                        "device_ms": {"transport": round(ms_tr, 2), "surrogate": round(ms_sg, 2),
                                      "scoring": round(ms_sc, 2)},
                        "primaries_per_s_device": n_per / ((ms_tr + ms_sg + ms_sc) / 1000.0),
                        "primaries_per_s_wall": n_per / wall}
        stream_ms += ms_tr + ms_sg + ms_sc
        wall_all += wall
    tot = len(energies) * n_per
    return {"workload": f"{n_per} primaries at each of {', '.join(str(int(e)) for e in energies)} eV, batches of "
                        f"{B}, box +-15 um, DNA 21 x 21 fibres, DSB window 10 bp; transport + surrogate chemistry "
                        "+ scoring (the IRT checks 1 % of batches)",
            "primaries_per_s_device": tot / (stream_ms / 1000.0), "primaries_per_s_wall": tot / wall_all,
            "device_ms": stream_ms, "yields": rows}


def run_sweep(args):
    """DNA-damage sweep (see sweep_block) with the surrogate trained first."""
    import wgdna
    from wgdna import surrogate as S
    n_per = args.np if args.np != NP else 1_000_000
    ctx = wgdna.Context(max_primaries=4096, max_rad=8_000_000, max_sec=1_200_000)
    train = S.train_on_irt(ctx)
    with Clocks(0) as clk:
        blk = sweep_block(ctx, n_per)
    line = {"metric": "DNA-damage sweep primaries/s (1, 3, 10 keV; transport + surrogate + scoring)",
            "value": blk["primaries_per_s_device"], "unit": "primaries/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": blk["device_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 transport / bf16-f32 surrogate", "data": "synthetic",
            "config": {"workload": blk["workload"], "training": train},
            "e2e": {"value": blk["primaries_per_s_wall"], "unit": "primaries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "yields": blk["yields"], "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--np", type=int, default=NP, help="primaries per GPU per step (4096 = the benchmark)")
    ap.add_argument("--pipeline", type=int, default=1,
                    help="batches in flight on one GPU (one context, stream and host thread each)")
    ap.add_argument("--tuning", default="",
                    help="launch-shape overrides for every context, e.g. transport_ctas_per_sm=1,irt_loop_blocks_per_sm=2 "
                         "(fields of wgdna_tuning; the rest from the tuning table)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate block of the default line")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the track / mixed / sweep blocks of the default line")
    ap.add_argument("--sweep-n", type=int, default=1_000_000, help="primaries per energy of the sweep block")
    ap.add_argument("--workload", choices=["pipeline", "track", "mixed", "surrogate", "sweep"], default="pipeline",
                    help="pipeline = 4096 x 10 keV transport+IRT+scoring (the benchmark); track = one "
                         "synthetic track through the IRT; mixed = 65,536 primaries of mixed energy; "
                         "surrogate = learned chemistry against the IRT; sweep = 1e6 primaries at 1, 3, 10 keV "
                         "with surrogate chemistry and DNA scoring")
    args = ap.parse_args()
    if args.workload != "pipeline":
        {"track": run_track, "mixed": run_mixed, "surrogate": run_surrogate, "sweep": run_sweep}[args.workload](args)
        return
    if args.impl == "reference":
        # host cores only: no device and no process group; under torchrun rank 0
        # alone measures and prints, the other ranks exit at once
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_init(args)
    try:
        run_native(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
