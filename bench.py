#!/usr/bin/env python3
"""Benchmark of the B200 equi-join engine.

Default workload: the full-size single join, |R| = |S| = 640,000,000 uint32 (key, value) tuples,
10% of S matching (64M output pairs, each materialised as (r_val, s_val)), Bloom filter 10 bits/key
with 7 hashes. A step is one complete join (partition R and S, build and probe the Bloom filter,
shared-memory hash build and probe, pair materialisation) over inputs resident in HBM.

  python bench.py [--gpus N --steps K --warmup W] [--workload c1|c0|batch|serve|sweep|shard] [--impl reference]

One JSON line on rank 0. `value` is the device-timed join throughput (|R|+|S|)/t over all ranks;
`e2e` the same metric through the host-array C entry point (H2D inputs, join, D2H pairs; S in
16 chunks against R partitioned once when |S| >= 2^26, so each chunk's passes overlap the next
chunk's copy);
`roofline` the dominant pipeline stage's algorithmic bytes over its CUDA-event duration;
`cpu_baseline` the reference's own CPU join (run_sanity_check) on a bounded sample on this host.
With N > 1 every rank runs an independent replica of the join (the path is single-GPU).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "brig-join_b200"))
sys.path.insert(0, ROOT)

METRIC = "join tuples/s ((|R|+|S|)/t)"
UNIT = "tuples/s"
WORKLOADS = {
    "c1": dict(name="join 640M x 640M, 10% match, Bloom 10 bits/key k=7", n_r=640_000_000,
               n_s=640_000_000, match=0.1, bloom=1, bpk=10.0, k=7, mode=0, p1=0),
    # the reference's README preset: --partition_size 512, i.e. first-level fan-out 512 by key % 512
    # (second level auto: 67, the reference's starting odd fan-out)
    "c0": dict(name="join 16M x 16M, 10% match, Bloom 10 bits/key k=7, fan-out 512 (key % 512)",
               n_r=1 << 24, n_s=1 << 24, match=0.1, bloom=1, bpk=10.0, k=7, mode=1, p1=512),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- clocks sampled during the timed region --------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="brig_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---- CPU baseline and reference arm: the reference's run_sanity_check on the benchmark's inputs ----
def workload_config(wl, world):
    """The workload's `config` object, identical in both arms."""
    nr, ns = wl["n_r"], wl["n_s"]
    return {"workload": wl["name"], "n_r": nr, "n_s": ns, "match_frac": wl["match"],
            "bloom_bits_per_key": wl["bpk"] if wl["bloom"] else 0, "bloom_hashes": wl["k"] if wl["bloom"] else 0,
            "partition_mode": "modulo" if wl["mode"] == 1 else "hash",
            "partition_size": wl["p1"] if wl["p1"] else "auto",
            "l2": f"no flush: each step streams {8 * (nr + ns) / 1e9:.2f} GB of inputs"
                  + (", far above the 126 MB L2" if 8 * (nr + ns) > 4 * 126e6 else ", a few times the 126 MB L2"),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def cpu_join_runs(rk, sk, reps, min_seconds=0.0):
    """Times the reference's own run_sanity_check (oracle/_ref, built from its sources) on int32
    views of the keys, or the oracle's restatement of it where the reference was not built:
    (kind, cores, seconds per run, count)."""
    from oracle import oracle as o
    times, count = [], None
    t_end = time.time() + min_seconds
    while len(times) < reps or (time.time() < t_end and len(times) < 4 * reps):
        if o.ref_available():
            count, sec = o.ref_count(rk, sk)
        else:
            t0 = time.perf_counter()
            count = o.count(rk, sk)
            sec = time.perf_counter() - t0
        times.append(sec)
    if o.ref_available():
        return "reference", o.ref_threads(), times, count
    return "port", 1, times, count


def run_reference_arm(args, wl):
    """The reference's CPU join on the full workload: inputs from the oracle's restatement of the
    generator (row-identical to the engine's, checked in the tests), W untimed and K timed runs of
    run_sanity_check. Loads no engine library."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    from oracle import oracle as o
    nr, ns = wl["n_r"], wl["n_s"]
    rk, _, sk, _ = o.gen(42, nr, ns, wl["match"], want_vals=False)
    m = int(math.floor(wl["match"] * ns))
    kind, cores, _, c = cpu_join_runs(rk, sk, max(args.warmup, 0))
    assert args.warmup == 0 or c == m, f"reference count {c} != {m}"
    kind, cores, secs, c = cpu_join_runs(rk, sk, args.steps)
    assert c == m, f"reference count {c} != {m}"
    t = sum(secs)
    value = args.steps * (nr + ns) / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": workload_config(wl, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"the full workload ({nr} x {ns} rows, {m} matches), one run_sanity_check "
                                   f"(count only, as the reference) per step on {cores} host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- multi-rank aggregation (replicas: one independent join per GPU) -------------------------------
def max_over_ranks(x: float, dist, device) -> float:
    """The largest x over all ranks (the job's time is its slowest rank's); x itself on one rank."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world: int, steps: int, nr: int, ns: int, ms_total: float) -> float:
    """Tuples per second over all ranks: every rank joins its own |R| + |S| tuples per step."""
    return world * steps * (nr + ns) / (ms_total / 1e3)


# ---- per-stage algorithmic bytes ------------------------------------------------------------------
def stage_bytes(nr, ns, surv, matches, bloom_bits, bloom_level):
    """Minimum bytes each stage must move in this layout: inputs read once, outputs written once.

    Partitioned buffers hold packed 8-byte (key, value) tuples, so a pass that only needs the keys
    still reads 8 bytes per tuple. bloom_level is the S pass that probes the filter (0: no filter).
    Level-1 probes read one random 32-byte sector per S tuple from HBM; level-2 probes read the
    filter from L2 (a partition's segments), which is not HBM traffic."""
    s_l1 = bloom_level == 1
    return {
        "r_hist": 4 * nr,
        "r_scan": 0,
        "r_scatter": 16 * nr,
        "r_l2_hist": 8 * nr,
        "r_l2_scatter": 16 * nr,
        "bloom_build": 8 * nr + bloom_bits // 8,
        "s_hist_probe": (4 * ns + 32 * ns + 12 * surv) if s_l1 else 4 * ns,
        "s_scan": 0,
        "s_scatter": 16 * (surv if s_l1 else ns),
        "s_l2_hist": 8 * surv if s_l1 else (8 * ns + 8 * surv if bloom_level == 2 else 8 * ns),
        "s_l2_scatter": 16 * surv,
        "tasks": 0,
        "probe": 8 * nr + 8 * surv + 8 * matches,
    }


# DRAM bytes (read + write) per tuple of each stage's main kernel, from ncu captures of the same
# kernels on 2^26 x 2^26 (inputs 4x the L2, fan-outs 512 x 512 and the filter probed at level 2 as at
# 640M) summarised in the profiles directory: (bytes per tuple, which count the stage's launch processes). Used to scale the
# measured traffic to the benchmarked launch; the per-tuple traffic of these streaming kernels does
# not depend on the relation size once the inputs exceed the L2.
NCU_TRAFFIC_PER_TUPLE = {
    "r_hist": (4.05, "nr"), "r_scatter": (15.93, "nr"), "r_l2_hist": (8.05, "nr"), "r_l2_scatter": (16.30, "nr"),
    "bloom_build": (9.01, "nr"), "s_hist_probe": (4.01, "ns"), "s_scatter": (15.94, "ns"),
    "s_l2_hist": (9.99, "ns"), "probe": (9.87, "nr"),
}


def stage_traffic(stage, nr, ns, bloom_level):
    """ncu-measured DRAM bytes of the stage's main kernel scaled to this launch, or None."""
    if stage not in NCU_TRAFFIC_PER_TUPLE:
        return None
    if stage in ("s_hist_probe", "s_scatter") and bloom_level == 1:
        return None  # captured with the filter probed in the second pass
    per, unit = NCU_TRAFFIC_PER_TUPLE[stage]
    return per * (nr if unit == "nr" else ns)


def gather_peak(bj, torch, stream, table_bytes=2 << 20, loads=1 << 30):
    """Random 8-byte reads per second from an L2-resident table (brig_join_gather_rate): the ceiling of
    the level-2 Bloom probe, one such read per key. Median of 5 timed launches after 2 warm-ups."""
    table = torch.randint(0, 1 << 30, (table_bytes // 4,), dtype=torch.int32, device="cuda")
    sink = torch.zeros(1, dtype=torch.int32, device="cuda")
    sp = stream.cuda_stream
    for _ in range(2):
        bj.gather_rate(table, loads, sink, stream=sp)
    rates = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n = bj.gather_rate(table, loads, sink, stream=sp)
        e1.record(stream)
        e1.synchronize()
        rates.append(n / (e0.elapsed_time(e1) / 1e3))
    rates.sort()
    return {"peak_reads_per_s": rates[len(rates) // 2], "unit": "reads/s",
            "peak_kind": f"measured in this run: brig_join_gather_rate, {loads} random 8-byte reads from a "
                         f"{table_bytes >> 20} MB L2-resident table"}


# ---- batched uneven joins -------------------------------------------------------------------------
def batch_shapes(n_joins, seed, lo=4096, hi=1 << 24):
    """|R_j| log-uniform in [lo, hi], |S_j| = 4 |R_j| (the 256-join uneven batch)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    nr = np.exp(rng.uniform(math.log(lo), math.log(hi), n_joins)).astype(np.int64)
    return [(int(r), int(4 * r)) for r in nr]


def batch_measure(joins, steps, warmup, fixed_cfg=None):
    """256 independent joins, S = 10% Zipf(1.0) matches over R's row order: one batched pipeline
    (autotuned, CUDA-graph replayed) against one single-join call per join. Returns the result dict;
    the batched and sequential pairs of every join are compared as sorted multisets."""
    import torch
    import brig_join as bj
    torch.cuda.set_device(0)
    shapes = batch_shapes(joins, 7)
    tot_r = sum(r for r, _ in shapes)
    tot_s = sum(s for _, s in shapes)
    i32 = torch.int32
    big = [torch.empty(n, dtype=i32, device="cuda") for n in (tot_r, tot_r, tot_s, tot_s)]
    ms = [int(math.floor(0.1 * s)) for _, s in shapes]
    caps = [m + 64 for m in ms]
    out_r = torch.empty(sum(caps), dtype=i32, device="cuda")
    out_s = torch.empty(sum(caps), dtype=i32, device="cuda")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    items, ro, so, oo, offs = [], 0, 0, 0, []
    for j, (nr, ns) in enumerate(shapes):
        v = [big[0][ro:ro + nr], big[1][ro:ro + nr], big[2][so:so + ns], big[3][so:so + ns]]
        bj.gen_device(1000 + j, nr, ns, 0.1, 1.0, *v, stream=sp)
        items.append(dict(r_key=v[0], r_val=v[1], n_r=nr, s_key=v[2], s_val=v[3], n_s=ns,
                          out_r=out_r[oo:oo + caps[j]], out_s=out_s[oo:oo + caps[j]], capacity=caps[j]))
        offs.append(oo)
        ro += nr; so += ns; oo += caps[j]
    torch.cuda.synchronize()
    tuples = tot_r + tot_s

    def timed(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    def sorted_pairs(counts):
        # every join's (r_val, s_val) pairs as one sorted int64 tensor per join
        res = []
        for j, c in enumerate(counts):
            a = out_r[offs[j]:offs[j] + int(c)].to(torch.int64) & 0xffffffff
            b = out_s[offs[j]:offs[j] + int(c)].to(torch.int64) & 0xffffffff
            res.append(torch.sort((a << 32) | b).values)
        return res

    # batched: autotune once (outside the timed region), then graph replays
    if fixed_cfg:
        jb = bj.Join(use_cuda_graph=1, **fixed_cfg)
        tuned, tune_s = dict(fixed_cfg), 0.0
    else:
        jb = bj.Join(use_cuda_graph=1)
        t0 = time.time()
        tuned = jb.autotune(items, stream=sp)
        tune_s = time.time() - t0
    for _ in range(max(warmup, 1)):
        jb.run_batch(items, stream=sp)
    counts = jb.batch_counts(len(items))
    assert list(counts) == ms, "batched counts differ from the constructed match counts"
    batched_pairs = sorted_pairs(counts)
    launches0 = bj.kernel_launches()
    with ClockSampler(0) as clk:
        ms_batch = timed(lambda: jb.run_batch(items, stream=sp), steps)
    launches = bj.kernel_launches() - launches0
    jb.batch_counts(len(items))
    # per-stage device times of the tuned configuration (a profiled handle launches directly)
    cfg = dict(tuned)
    cfg = {k: v for k, v in cfg.items() if k in dict(bj.Config._fields_)}
    with bj.Join(profile_stages=1, **cfg) as jp:
        jp.run_batch(items, stream=sp)
        jp.run_batch(items, stream=sp)
        jp.batch_counts(len(items))
        jp.stage_times()
        jp.run_batch(items, stream=sp)
        jp.batch_counts(len(items))
        stages = jp.stage_times()
    jb.close()
    # sequential: the same joins, one plain join call each
    js = bj.Join()

    def seq():
        for it in items:
            js.run(it["r_key"], it["r_val"], it["n_r"], it["s_key"], it["s_val"], it["n_s"], it["out_r"], it["out_s"],
                   it["capacity"], stream=sp)
    seq()
    seq_counts = []
    for it in items:
        js.run(it["r_key"], it["r_val"], it["n_r"], it["s_key"], it["s_val"], it["n_s"], it["out_r"], it["out_s"],
               it["capacity"], stream=sp)
        seq_counts.append(js.stats().count)
    assert seq_counts == ms, "sequential counts differ"
    seq_pairs = sorted_pairs(seq_counts)
    identical = all(torch.equal(a, b) for a, b in zip(batched_pairs, seq_pairs))
    del batched_pairs, seq_pairs
    ms_seq = timed(seq, max(1, steps // 4))
    js.close()
    return {
        "metric": "batched join tuples/s (sum |R|+|S| over %d joins / t)" % joins, "value": tuples / (ms_batch / 1e3),
        "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": ms_batch,
        "higher_is_better": True, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"{joins} joins, |R| log-uniform [4K, 16M], |S| = 4|R|, 10% Zipf(1.0) matches",
                   "total_r": tot_r, "total_s": tot_s, "autotuned": tuned, "autotune_s": round(tune_s, 2),
                   "graph": True},
        "stage_ms": {k: round(v, 3) for k, v in stages.items()},
        "sequential": {"ms_per_batch": ms_seq, "value": tuples / (ms_seq / 1e3)},
        "speedup_vs_sequential": ms_seq / ms_batch, "gpu_launches": launches, "clocks": clk.summary(),
        "identical_results": identical,
        "identical_results_check": "per join, the sorted (r_val, s_val) multisets of the batched and the "
                                   "sequential runs compared on the device",
    }


def run_batch_workload(args):
    fixed = json.loads(args.batch_config) if args.batch_config else None
    print(json.dumps(batch_measure(args.joins, args.steps, args.warmup, fixed)), flush=True)
    return 0


# ---- selectivity and Bloom sweep ------------------------------------------------------------------
def run_sweep_workload(args):
    """|R| = 2^26, |S| = 2^30, a fraction of S drawn from R (0.1%, 1%, 10%, 100%), the filter off or on
    at 8, 10 and 14 bits/key: device time per join, survivors and the chosen probe level. Every
    count is checked against the constructed match count."""
    import torch
    import brig_join as bj
    torch.cuda.set_device(0)
    nr, ns = 1 << 26, 1 << 30
    if args.rows > 0:
        nr, ns = args.rows, 16 * args.rows
    i32 = torch.int32
    rk, rv = (torch.empty(nr, dtype=i32, device="cuda") for _ in range(2))
    sk, sv = (torch.empty(ns, dtype=i32, device="cuda") for _ in range(2))
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    rows = []
    fracs = [float(x) for x in args.fracs.split(",")] if args.fracs else [0.001, 0.01, 0.1, 1.0]
    bpks = [float(x) for x in args.bpks.split(",")] if args.bpks else [0, 8.0, 10.0, 14.0]
    for frac in fracs:
        bj.gen_device(7, nr, ns, frac, 0.0, rk, rv, sk, sv, stream=sp)
        m = int(math.floor(frac * ns))
        cap = m + 4096
        out_r = torch.empty(cap, dtype=i32, device="cuda")
        out_s = torch.empty(cap, dtype=i32, device="cuda")
        for bpk in bpks:
            kw = dict(use_bloom=1, bloom_bits_per_key=bpk) if bpk else dict(use_bloom=0)
            with bj.Join(**kw) as j:
                for _ in range(max(args.warmup, 1)):
                    j.run(rk, rv, nr, sk, sv, ns, out_r, out_s, cap, stream=sp)
                st = j.stats()
                assert st.count == m, (frac, bpk, st.count, m)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                steps = max(1, min(args.steps, 5))
                e0.record(stream)
                for _ in range(steps):
                    j.run(rk, rv, nr, sk, sv, ns, out_r, out_s, cap, stream=sp)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / steps
                rows.append({"match": frac, "bloom_bits_per_key": bpk, "ms": round(ms, 3),
                             "g_tuples_per_s": round((nr + ns) / ms / 1e6, 2), "count": st.count,
                             "s_survivors": st.s_survivors, "bloom_num_hashes": st.bloom_num_hashes})
        del out_r, out_s
    line = {"metric": "join tuples/s ((|R|+|S|)/t) across selectivity and Bloom size", "unit": UNIT,
            "n_r": nr, "n_s": ns, "data": "synthetic", "dtype": "u32", "sweep": rows}
    print(json.dumps(line), flush=True)
    return 0


# ---- served joins ---------------------------------------------------------------------------------
def serve_measure(pool_n, requests, rates, streams):
    """Poisson stream of join requests against a 120 GB budget: p50/p99 latency and aggregate
    tuples/s per offered load, continuous batching against one request at a time. Returns the
    result dict; every request's count is checked against its constructed match count."""
    import numpy as np
    import threading
    import torch
    import brig_join as bj
    torch.cuda.set_device(0)
    rng = np.random.default_rng(11)
    pool = []
    for i in range(pool_n):
        nr = int(math.exp(rng.uniform(math.log(1 << 16), math.log(1 << 26))))
        ratio = int(rng.choice([1, 4, 16]))
        frac = float(rng.choice([0.01, 0.1, 0.5]))
        ns = nr * ratio
        t = [torch.empty(n, dtype=torch.int32, device="cuda") for n in (nr, nr, ns, ns)]
        bj.gen_device(5000 + i, nr, ns, frac, 0.0, *t)
        pool.append((t, nr, ns, int(math.floor(frac * ns))))
    torch.cuda.synchronize()
    seq = [int(x) for x in rng.integers(0, len(pool), requests)]

    # pinned host outputs: the pairs come back by asynchronous copies, as a client that hands the
    # server page-locked buffers would receive them
    outs = {i: tuple(torch.empty(pool[i][3] + 16, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
                     for _ in range(2)) for i in range(len(pool))}

    def one_load(srv, rate):
        lat, queue, phases = [], [], []
        gaps = np.random.default_rng(3).exponential(1.0 / rate, len(seq)) if rate > 0 else np.zeros(len(seq))
        tickets = []
        t0 = time.perf_counter()

        def submitter():
            nxt = t0
            for k, i in enumerate(seq):
                nxt += gaps[k]
                d = nxt - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                t, nr, ns, m = pool[i]
                tickets.append((srv.submit(t[0], t[1], t[2], t[3], capacity=m + 16, out=outs[i], on_device=True), i))
        th = threading.Thread(target=submitter)
        th.start()
        done = 0
        while done < len(seq):
            while len(tickets) <= done:
                time.sleep(0.0005)
            tk, i = tickets[done]
            res, a, b = srv.poll(tk)
            assert res.status == bj.BRIG_OK and res.count == pool[i][3]
            lat.append(res.submit_to_done_ms)
            queue.append(res.queue_ms)
            phases.append((res.setup_ms, res.join_ms, res.wave))
            done += 1
        th.join()
        wall = time.perf_counter() - t0
        tuples = sum(pool[i][1] + pool[i][2] for i in seq)
        worst = sorted(range(len(seq)), key=lambda k: -lat[k])[:3]
        return {"offered_req_per_s": rate, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_queue_ms": float(np.mean(queue)), "tuples_per_s": tuples / wall, "wall_s": wall,
                "slowest": [{"ms": round(lat[k], 2), "queue_ms": round(queue[k], 2),
                             "setup_ms": round(phases[k][0], 2), "join_ms": round(phases[k][1], 2),
                             "wave": phases[k][2], "tuples": pool[seq[k]][1] + pool[seq[k]][2]} for k in worst]}

    def run_mode(streams, max_wave):
        # One long-running server per mode. A warm-up pass over the whole pool sizes every slot's
        # workspace (growing it maps fresh device memory, which a running server pays once), then
        # each offered load replays the same Poisson request sequence.
        with bj.Server(hbm_budget_bytes=120 * 10**9, max_wave=max_wave, streams=streams) as srv:
            for _ in range(2):
                tk = [srv.submit(t[0], t[1], t[2], t[3], capacity=m + 16, out=outs[i], on_device=True)
                      for i, (t, nr, ns, m) in enumerate(pool)]
                for x in tk:
                    srv.poll(x)
            return [one_load(srv, r) for r in rates]

    sweep = run_mode(streams, 16)
    base = run_mode(1, 1)
    return {
        "metric": "served join tuples/s and p50/p99 latency", "value": max(x["tuples_per_s"] for x in sweep),
        "unit": UNIT, "n_gpus": 1, "dtype": "u32", "data": "synthetic", "higher_is_better": True,
        "config": {"workload": f"{requests} Poisson requests from a pool of {len(pool)}: |R| log-uniform "
                               "[64K, 64M], |S|/|R| in {1,4,16}, match in {1%,10%,50%}, budget 120 GB",
                   "streams": streams, "max_wave": 16},
        "continuous_batching": sweep, "one_at_a_time": base,
    }


# ---- sharded join across GPUs ---------------------------------------------------------------------
def shard_measure(rows, steps, warmup):
    """The sharded join (brig_join.shard) on every rank of the job: one global pair of relations of
    |R| = |S| = rows x ranks tuples (the device generator, 10% of S matching), each rank holding a
    contiguous slice of both. A step is one ShardedJoin.run on every rank: R grouped by owner and
    exchanged over NCCL, the owners' filters (10 bits/key, k = 7) built and gathered, S prefiltered,
    grouped and exchanged, the local joins. Weak scaling: the rows per rank stay fixed. The first
    run's global pair count is checked against the constructed match count, and its pairs against
    the keys. Also reported: the R grouping kernels' bandwidth (key read for the counts; key and
    value read and written for the scatter: 20 bytes per tuple) and the plain single-GPU join of one
    rank's slices. Joins the job's process group, or makes a one-rank NCCL group for itself.
    Returns rank 0's line (None on the other ranks)."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    import brig_join as bj
    import brig_join.shard as sh
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    own_group = not dist.is_initialized()
    if own_group:
        if "MASTER_ADDR" not in os.environ or world == 1:
            with socket.socket() as so:
                so.bind(("127.0.0.1", 0))
                os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(so.getsockname()[1])
        dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    try:
        n = rows
        total = n * world
        i32 = torch.int32
        stream = torch.cuda.current_stream()
        g = [torch.empty(total, dtype=i32, device="cuda") for _ in range(4)]
        bj.gen_device(42, total, total, 0.1, 0.0, *g, stream=stream.cuda_stream)
        rk, rv, sk, sv = (t[rank * n:(rank + 1) * n].clone() for t in g)
        m = int(math.floor(0.1 * total))
        job = sh.ShardedJoin(sh.TorchComm(), bits_per_key=10.0, num_hashes=7)
        ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
        for w in range(max(warmup, 1)):
            x = job.run(rk, rv, sk, sv)
            if w == 0:  # values are global row numbers: every pair key-equal, every S row at most once
                assert x.total == m, f"global count {x.total} != {m}"
                r, s_ = x.r_val.long(), x.s_val.long()
                assert bool((g[0][r] == g[2][s_]).all().item()), "pair check failed"
                assert int(torch.unique(s_).numel()) == x.count, "an S row matched twice"
                del r, s_, g
            del x
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(steps):
            x = job.run(rk, rv, sk, sv)
            del x
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda") / steps
        # the R grouping kernels alone
        ops = job.ops
        for _ in range(3):
            ops.split(world, rk, rv)
        torch.cuda.synchronize()
        a0, a1 = ev(), ev()
        reps = 10
        a0.record(stream)
        for _ in range(reps):
            ops.split(world, rk, rv)
        a1.record(stream)
        torch.cuda.synchronize()
        split_ms = a0.elapsed_time(a1) / reps
        # the plain join of this rank's slices
        cap = n + 4096
        out_r = torch.empty(cap, dtype=i32, device="cuda")
        out_s = torch.empty(cap, dtype=i32, device="cuda")
        with bj.Join(use_bloom=1, bloom_bits_per_key=10.0, bloom_num_hashes=7) as jn:
            for _ in range(3):
                jn.run(rk, rv, n, sk, sv, n, out_r, out_s, cap, stream=stream.cuda_stream)
            b0, b1 = ev(), ev()
            b0.record(stream)
            for _ in range(5):
                jn.run(rk, rv, n, sk, sv, n, out_r, out_s, cap, stream=stream.cuda_stream)
            b1.record(stream)
            torch.cuda.synchronize()
            plain_ms = b0.elapsed_time(b1) / 5
        if rank != 0:
            return None
        peak, peak_kind = peaks()
        split_gbs = 20.0 * n / (split_ms * 1e-3) / 1e9
        return {"metric": "sharded join tuples/s ((|R|+|S|)/t)", "value": 2 * total * 1e3 / ms, "unit": UNIT,
                "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": round(ms, 3),
                "higher_is_better": True, "scaling": "weak", "dtype": "u32", "data": "synthetic",
                "config": {"workload": f"sharded join {total} x {total} over {world} rank(s), 10% match, "
                                       "owner filters 10 bits/key k=7", "rows_per_rank": n},
                "r_split_ms": round(split_ms, 3),
                "r_split_roofline": {"bound": "hbm", "achieved": round(split_gbs, 1), "peak": peak,
                                     "unit": "GB/s", "frac": round(split_gbs / peak, 3), "bytes_per_tuple": 20,
                                     "peak_kind": peak_kind},
                "plain_join_ms_one_rank_slices": round(plain_ms, 3)}
    finally:
        if own_group:
            dist.destroy_process_group()


def run_shard_workload(args):
    line = shard_measure(args.rows if args.rows > 0 else 1 << 26, args.steps, args.warmup)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def run_serve_workload(args):
    rates = [float(x) for x in args.rates.split(",")]
    print(json.dumps(serve_measure(args.pool, args.requests, rates, args.streams)), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS) + ["batch", "serve", "sweep", "shard"])
    ap.add_argument("--joins", type=int, default=256, help="batch workload: number of joins")
    ap.add_argument("--batch-config", default="",
                    help="batch workload: a JSON object of configuration fields to use instead of autotuning")
    ap.add_argument("--pool", type=int, default=24, help="serve workload: distinct requests")
    ap.add_argument("--requests", type=int, default=64, help="serve workload: requests per load point")
    ap.add_argument("--rates", default="20,80,320,1280", help="serve workload: offered loads (requests/s)")
    ap.add_argument("--fracs", default="", help="sweep workload: match fractions (comma-separated)")
    ap.add_argument("--bpks", default="", help="sweep workload: Bloom bits per key, 0 = no filter (comma-separated)")
    ap.add_argument("--streams", type=int, default=3, help="serve workload: concurrent waves")
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and served measurements that follow the join's")
    ap.add_argument("--bloom", type=int, default=None, help="override Bloom on/off")
    ap.add_argument("--bloom-level", type=int, default=0,
                    help="S pass that probes the filter (1 first, 2 second, 0 planner's choice)")
    ap.add_argument("--rows", type=int, default=0,
                    help="override |R| = |S| (a smaller case of the same generator, e.g. for ncu)")
    ap.add_argument("--p1", type=int, default=0, help="override the level-1 fan-out")
    ap.add_argument("--p2", type=int, default=0, help="override the level-2 fan-out")
    ap.add_argument("--mode", type=int, default=None, help="override the partition mode (0 hash, 1 modulo)")
    ap.add_argument("--table", type=int, default=0, help="override table_capacity")
    ap.add_argument("--s-chunks", type=int, default=-1,
                    help="e2e: copy and join S in this many chunks against R partitioned once (s_chunks); "
                         "-1: 16 when |S| >= 2^26, else one piece")
    args = ap.parse_args()
    if args.steps > 64:
        ap.error("--steps above 64: per-stage events keep the last 64 runs")
    if args.workload == "batch":
        return run_batch_workload(args)
    if args.workload == "sweep":
        return run_sweep_workload(args)
    if args.workload == "serve":
        return run_serve_workload(args)
    if args.workload == "shard":
        return run_shard_workload(args)
    wl = dict(WORKLOADS[args.workload])
    if args.bloom is not None:
        wl["bloom"] = args.bloom
    if args.p1:
        wl["p1"] = args.p1
    if args.mode is not None:
        wl["mode"] = args.mode
    if args.rows > 0:
        wl["n_r"] = wl["n_s"] = args.rows
        wl["name"] = f"join {args.rows} x {args.rows}, 10% match" + (
            f", Bloom {wl['bpk']:g} bits/key k={wl['k']}" if wl["bloom"] else "")
    if args.impl == "reference":
        return run_reference_arm(args, wl)

    import torch
    import brig_join as bj

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    nr, ns = wl["n_r"], wl["n_s"]
    i32 = torch.int32
    rk = torch.empty(nr, dtype=i32, device="cuda")
    rv = torch.empty(nr, dtype=i32, device="cuda")
    sk = torch.empty(ns, dtype=i32, device="cuda")
    sv = torch.empty(ns, dtype=i32, device="cuda")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    bj.gen_device(42 + rank, nr, ns, wl["match"], 0.0, rk, rv, sk, sv, stream=sp)
    m = int(math.floor(wl["match"] * ns))
    cap = m + m // 50 + 4096
    out_r = torch.empty(cap, dtype=i32, device="cuda")
    out_s = torch.empty(cap, dtype=i32, device="cuda")
    jcfg = dict(use_bloom=wl["bloom"], bloom_bits_per_key=wl["bpk"], bloom_num_hashes=wl["k"],
                bloom_probe_level=args.bloom_level, partition_mode=wl["mode"], partition_size=wl["p1"],
                second_partition_size=args.p2, table_capacity=args.table)
    j = bj.Join(use_cuda_graph=1, profile_stages=1, **jcfg)

    def step():
        j.run(rk, rv, nr, sk, sv, ns, out_r, out_s, cap, stream=sp)

    # warm-up; the first run is checked: exact count, every pair key-equal, every matching S row once
    for w in range(max(args.warmup, 1)):
        step()
        st = j.stats()
        j.stage_times()  # discard warm-up stage times
        if w == 0:
            assert st.count == m, f"count {st.count} != {m}"
            r = out_r[:st.count].long()
            s = out_s[:st.count].long()
            ok = bool((rk[r] == sk[s]).all().item())
            uniq = int(torch.unique(s).numel())
            assert ok and uniq == m, "pair check failed"
            del r, s
    torch.cuda.synchronize()

    # timed region: inputs (8*(|R|+|S|) bytes) are far larger than L2, so no flush is needed
    stages = {}
    launches0 = bj.kernel_launches()
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        stages = j.stage_times()  # mean per-stage CUDA-event time over exactly these K steps
        if dist:
            dist.barrier()
    launches = bj.kernel_launches() - launches0
    ms_total = ev0.elapsed_time(ev1)
    st = j.stats()
    ms_total = max_over_ranks(ms_total, dist, "cuda")
    ms_step = ms_total / args.steps
    value = whole_job_value(world, args.steps, nr, ns, ms_total)

    peak, peak_kind = peaks()
    avg = stages
    blvl = 0
    if wl["bloom"]:
        blvl = args.bloom_level or (1 if st.bloom_num_bits // 8 <= (96 << 20) or st.second_partition_size <= 1
                                    else 2)
    sb = stage_bytes(nr, ns, st.s_survivors, st.count, st.bloom_num_bits, blvl)
    dom = max(avg, key=avg.get)
    achieved = sb[dom] / (avg[dom] / 1e3) / 1e9
    join_bytes = 8 * (nr + ns) + 8 * st.count
    join_gbs = join_bytes / (ms_step / 1e3) / 1e9
    # The level-2 Bloom pass reads one filter word pair per S key from L2 at a hashed position: its
    # ceiling is the rate of such reads, measured here outside the timed region (2 MB table).
    gather = None
    if blvl == 2 and "s_l2_hist" in avg:
        gather = gather_peak(bj, torch, stream)
        keys_per_s = ns / (avg["s_l2_hist"] / 1e3)
        gather.update({"kernel": "s_l2_hist", "achieved_reads_per_s": keys_per_s,
                       "frac": keys_per_s / gather["peak_reads_per_s"]})

    # end to end through the host-array entry point: pinned host inputs in, pairs out
    e2e = None
    if args.e2e_steps > 0:
        hk = [torch.empty(n, dtype=i32, pin_memory=True) for n in (nr, nr, ns, ns)]
        for h, d in zip(hk, (rk, rv, sk, sv)):
            h.copy_(d)
        ho_r = torch.empty(cap, dtype=i32, pin_memory=True)
        ho_s = torch.empty(cap, dtype=i32, pin_memory=True)
        torch.cuda.synchronize()
        times = []
        cnt = None
        jh = j
        if args.s_chunks < 0:
            args.s_chunks = 16 if ns >= (1 << 26) else 0
        if args.s_chunks > 1:
            jh = bj.Join(s_chunks=args.s_chunks, **jcfg)
        for it in range(args.e2e_steps + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cnt, _, _ = jh.run_host(hk[0].numpy(), hk[1].numpy(), hk[2].numpy(), hk[3].numpy(), capacity=cap,
                                    out=(ho_r.numpy(), ho_s.numpy(), None), stream=sp)
            e1.record(stream)
            torch.cuda.synchronize()
            if it > 0:
                times.append(e0.elapsed_time(e1))
        assert cnt == m
        e2e_ms = sum(times) / len(times)
        if dist:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": world * (nr + ns) / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": 8 * (nr + ns), "d2h_bytes_per_step": 8 * cnt + 8}
        if args.s_chunks > 1:
            e2e["s_chunks"] = args.s_chunks

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference's CPU join on this run's own inputs (the keys, as the int32 it takes)
        if e2e is not None:
            hr, hs = hk[0].numpy(), hk[2].numpy()
        else:
            hr, hs = rk.cpu().numpy(), sk.cpu().numpy()
        kind, cores, secs, c = cpu_join_runs(hr, hs, 2, min_seconds=10.0)
        assert c == m, f"CPU join count {c} != {m}"
        cpu = {"value": (nr + ns) / (sum(secs) / len(secs)), "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"the full workload ({nr} x {ns} rows), {len(secs)} runs of run_sanity_check "
                         f"(count only) on {cores} host threads"}
        del hr, hs

    # the batched and served forms on the same GPU, after the join's buffers are released
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        if e2e is not None:
            del hk, ho_r, ho_s
            if jh is not j:
                jh.close()
        j.close()
        del rk, rv, sk, sv, out_r, out_s
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        b = batch_measure(args.joins, 10, 3)
        extras["batch"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "speedup_vs_sequential",
                                            "identical_results", "gpu_launches", "stage_ms")}
        extras["batch"]["sequential_ms"] = b["sequential"]["ms_per_batch"]
        extras["batch"]["workload"] = b["config"]["workload"]
        extras["batch"]["autotuned"] = b["config"]["autotuned"]
        torch.cuda.empty_cache()
        sv_ = serve_measure(16, 48, [20.0, 640.0], 3)
        extras["serve"] = {"workload": sv_["config"]["workload"],
                           "continuous_batching": [{k: x[k] for k in ("offered_req_per_s", "p50_ms", "p99_ms",
                                                                      "tuples_per_s")}
                                                   for x in sv_["continuous_batching"]],
                           "one_at_a_time": [{k: x[k] for k in ("offered_req_per_s", "p50_ms", "p99_ms",
                                                                "tuples_per_s")}
                                             for x in sv_["one_at_a_time"]]}
        torch.cuda.empty_cache()
        try:  # the sharded join's path on this one GPU (a one-rank NCCL group)
            sh_ = shard_measure(1 << 25, 5, 3)
            extras["shard"] = {k: sh_[k] for k in ("value", "unit", "ms_per_step", "r_split_ms", "r_split_roofline",
                                                   "plain_join_ms_one_rank_slices")}
            extras["shard"]["workload"] = sh_["config"]["workload"]
        except Exception as e:  # noqa: BLE001 - reported in the line; the join's figures stand
            extras["shard"] = {"error": f"{type(e).__name__}: {e}"[:300]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(wl, world),
            "plan": {"partition_size": st.partition_size, "second_partition_size": st.second_partition_size,
                     "bloom_hashes": st.bloom_num_hashes, "bloom_num_bits": st.bloom_num_bits,
                     "bloom_probe_level": blvl},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": stage_traffic(dom, nr, ns, blvl),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per tuple on "
                                           "2^26 x 2^26, scaled to this launch",
                         "peak_kind": peak_kind},
            "join_roofline": {"algorithmic_bytes": join_bytes, "achieved": join_gbs, "peak": peak,
                              "frac": join_gbs / peak, "unit": "GB/s"},
            "bloom_read_roofline": gather,
            "stage_ms": {k: round(v, 4) for k, v in avg.items()},
            "matches": st.count, "s_survivors": st.s_survivors,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    j.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
