#!/usr/bin/env python
"""Benchmark of the batched banded affine-gap DP path (fills + tracebacks).

Default workload (one step = one batch): 1,000,000 short-read pairs,
rlength U{75..300}, lband/uband U{3..30}, 3% substitutions, 1% indels, 5%
random non-matching windows, 8-bit fills with the 16-bit rerun on overflow,
traceback of every pair.  Synthetic, seeded.  Metric: GCUPS over the
in-band cells of the reference's compare domain, whole job, fill +
traceback.  `value` is measured with pairs and sequences resident in HBM;
`e2e` goes through the host-buffer C-ABI call gdp_align_batch (host->device
copies, planning, kernels, device->host copies of results and Pair records
all inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gdp|reference]

For N > 1 launch with torchrun; each rank aligns its own shard of the same
size (weak scaling, no data-path collective: pairs are independent).
`--impl reference` times the reference's own CPU code (oracle/_ref, built
from the reference sources) on the host cores over a bounded sample.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gdp  # noqa: E402

WORKLOADS = {
    "short": (gdp.WL_SHORT, 1_000_000, "short reads r U{75..300}, bands U{3..30}, 8-bit + 16-bit rerun"),
    "fixed": (gdp.WL_FIXED, 10_000, "fixed 150x160, lband=uband=10, 16-bit"),
    "mix": (gdp.WL_MIX, 20_000, "70/25/5 short/long/cdna mix"),
    "cdna": (gdp.WL_CDNA, 2_000, "cDNA upper fill, r log-U[200,5000]"),
    "long": (gdp.WL_LONG, 2_000, "long reads r U{1000..10000}, bands U{50..200}, 16-bit"),
}
OPS_PER_CELL = 9          # E: 2 add + 1 max, F: 2 add + 1 max, H: 1 add + 2 max
DIR_BYTES_PER_CELL = 0.5  # 4 direction bits per cell


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons while the
    timed region runs: NVML read-only queries every 5 ms from a thread, with
    one sample at start and one at stop, so even a region of a few tens of
    milliseconds has samples.  Falls back to `nvidia-smi -lms 200`."""

    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.rows = []            # (sm_mhz, max_mhz, reason bits or names)
        self.proc = None
        self.thread = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def _handle(self, pynvml):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            for u in (uuid, "GPU-" + uuid):
                try:
                    return pynvml.nvmlDeviceGetHandleByUUID(u)
                except Exception:
                    pass
        except Exception:
            pass
        return pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_sample(self):
        p, h = self.nvml
        sm = p.nvmlDeviceGetClockInfo(h, p.NVML_CLOCK_SM)
        mx = p.nvmlDeviceGetMaxClockInfo(h, p.NVML_CLOCK_SM)
        try:
            bits = p.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            bits = p.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.rows.append((float(sm), float(mx), int(bits)))

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = (pynvml, self._handle(pynvml))
            self._nvml_sample()
        except Exception:
            self.nvml = None
        if self.nvml:
            def poll():
                while not self.stop_flag.wait(0.005):
                    try:
                        self._nvml_sample()
                    except Exception:
                        return
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) > 2 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                active = {n for k, n in enumerate(names) if len(r) > 5 + k and r[5 + k].lower() == "active"}
                self.rows.append((float(r[1]), float(r[2]), active))

    def stop(self):
        self.stop_flag.set()
        if self.nvml:
            if self.thread:
                self.thread.join(timeout=2)
            try:
                self._nvml_sample()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)
        reasons = set()
        for _, _, r in self.rows:
            if isinstance(r, int):
                reasons |= {n for n, b in self.REASONS.items() if r & b}
            else:
                reasons |= r
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nvml else "nvidia-smi"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(world, value, op):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(world, value):
    """The slowest rank's time: the whole job ends when it does."""
    import torch.distributed as dist
    return _reduce(world, value, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(world, value):
    import torch.distributed as dist
    return _reduce(world, value, dist.ReduceOp.SUM if world > 1 else None)


def make_workload(lib, name, npairs, seed, genome_len=1 << 24):
    kind = WORKLOADS[name][0]
    genome, blocks = gdp.make_genome(lib, 777, genome_len)
    pairs, arena = gdp.make_pairs(lib, kind, seed, genome, npairs)
    return genome, blocks, pairs, arena


def cpu_baseline(lib, name, seed, target_seconds, threads=None, genome=None):
    """The reference's own code (oracle/_ref) on a bounded sample of the same
    workload, all host threads (or the port when the reference is absent).
    `genome` = (sequence, genomecomp blocks) already set in the library."""
    import oracle
    kind = "reference" if oracle.reference_available() else "port"
    ref = oracle.reference() if kind == "reference" else oracle.restatement()
    threads = threads or os.cpu_count() or 1
    if genome is None:
        ref.init(0)
        genome, blocks = gdp.make_genome(lib, 777, 1 << 24)
        ref.set_genome(blocks, None, genome.size)
    else:
        genome, blocks = genome
    # calibration: rerun pairs in 16-bit, which costs about what the kept precisions do
    n = 200
    while True:
        pairs, arena = gdp.make_pairs(lib, WORKLOADS[name][0], seed + 99, genome, n)
        secs, _ = ref.bench(pairs, arena, threads)
        if secs >= target_seconds / 4 or n >= 2_000_000:
            break
        n = int(min(2_000_000, n * max(2.0, target_seconds / max(secs, 1e-3))))
    # the timed sample runs each pair at the precision the rerun contract keeps
    kept = kept_precisions(lib, genome, blocks, pairs, arena, threads)
    secs, _ = ref.bench(pairs, arena, threads, kept)
    cells = int(gdp.band_cells(pairs).sum())
    return {"value": round(cells / secs / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
            "sample": f"{n} pairs of the '{name}' workload ({cells} in-band cells), fill + traceback at the "
                      f"kept precision ({int((kept == 8).sum())} 8-bit), {secs:.2f} s wall on {threads} threads",
            "seconds": secs, "pairs": n, "cells": cells, "kept": kept, "data": (pairs, arena)}


def kept_precisions(lib, genome, blocks, pairs, arena, threads):
    """Per pair, the precision the rerun contract keeps (an 8-bit pair
    flagged RERUN16 keeps 8 unless its 8-bit fill saturates or its 8-bit
    traceback would read unwritten cells), from the restatement, untimed."""
    import oracle
    rest = oracle.restatement()
    rest.init(0)
    rest.set_genome(blocks, None, genome.size)
    return rest.kept_precision(pairs, arena, threads)


def endpoint_search(lib, ctx, seed, ngaps=200000):
    """End-gap endpoint search on the device: the short reads as end gaps
    (an upper and a lower fill per gap, extraband 14 as Dynprog_compute_bands
    gives end gaps), timed as one device-resident plan with and without the
    search flags; the search's cost is the difference."""
    import torch
    genome, blocks = gdp.make_genome(lib, 777, 1 << 24)
    base, arena = gdp.make_pairs(lib, gdp.WL_SHORT, seed, genome, ngaps)
    ctx.set_genome(blocks, None, genome.size)
    rl, gl = base["rlength"].astype(np.int64), base["glength"].astype(np.int64)
    pairs = np.repeat(base, 2)
    up, lo = pairs[0::2], pairs[1::2]
    up["variant"], lo["variant"] = gdp.UPPER, gdp.LOWER
    up["uband"], up["lband"] = np.maximum(gl - rl, 0) + 14, 0
    lo["lband"], lo["uband"] = np.maximum(rl - gl, 0) + 14, 0
    pairs["precision"] = 16
    keep = pairs["flags"] & gdp.FLAG_JUMP_LATE
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    d_arena = torch.from_numpy(arena).cuda()
    d_res = torch.empty(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    cells = int(gdp.band_cells(pairs).sum())
    out = {"gaps": ngaps, "fills": int(pairs.size), "cells": cells}
    for label, flags in (("plain", keep), ("endpoint", keep | gdp.FLAG_ENDPOINT)):
        pairs["flags"] = flags
        d_pairs.copy_(torch.from_numpy(pairs.view(np.uint8)))
        plan = ctypes.c_void_p()
        assert lib.gdp_plan_create(ctx.h, gdp._ptr(pairs), pairs.size, ctypes.byref(plan)) == 0, ctx.error()
        d_recs = torch.empty(16, dtype=torch.uint8, device="cuda")
        run = lambda: lib.gdp_plan_execute(ctx.h, plan, ctypes.c_void_p(d_pairs.data_ptr()),
                                           ctypes.c_void_p(d_arena.data_ptr()), ctypes.c_void_p(d_res.data_ptr()),
                                           ctypes.c_void_p(d_recs.data_ptr()))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(5):
            run()
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / 5
        lib.gdp_plan_destroy(plan)
        res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
        out[label] = {"ms": round(ms, 3), "gcups": round(cells / (ms * 1e-3) / 1e9, 2),
                      "bad_status": int((res["status"] != 0).sum())}
        if label == "endpoint":
            out[label]["halves_found"] = int(res["end_found"].sum())
    out["search_overhead_pct"] = round(100 * (out["endpoint"]["ms"] / out["plain"]["ms"] - 1), 1)
    return out


def stage3_gaps(genome, seed, ngaps, max_rlength, max_glength):
    """Single gaps as stage 3 sends them to Dynprog_single_gap: a query
    stretch between two aligned blocks (4..200 nt, log-uniform) against the
    genome stretch between them, half of equal length (substitutions only)
    and half with an indel of up to 10 nt; 1 % substitutions; plus strand;
    extraband_single = max(3, |glength - rlength|), widebandp, HIGHQ."""
    rng = np.random.default_rng(seed)
    rl = np.exp(rng.uniform(np.log(4), np.log(201), ngaps)).astype(np.int64)
    d = np.where(rng.random(ngaps) < 0.5, 0, rng.integers(-10, 11, ngaps))
    gl = np.maximum(rl + d, 1)
    goff = rng.integers(0, genome.size - 512, ngaps)
    # query = the genome stretch (its first rlength characters, padded with
    # random bases past glength), then 1 % substitutions
    tot = int(rl.sum())
    qoff = np.zeros(ngaps, np.int64)
    qoff[1:] = np.cumsum(rl)[:-1]
    idx = np.repeat(goff - qoff, rl) + np.arange(tot)
    q = genome[idx].copy()
    within = np.arange(tot) - np.repeat(qoff, rl) < np.repeat(gl, rl)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    q[~within] = rng.choice(acgt, size=int((~within).sum()))
    sub = rng.random(tot) < 0.01
    q[sub] = rng.choice(acgt, size=int(sub.sum()))
    q[q == ord("N")] = ord("A")
    arena = q   # rsequence and rsequenceuc are the same bytes
    gaps = np.zeros(ngaps, dtype=gdp.SINGLE_GAP_DTYPE)
    gaps["rseq"] = gaps["rseq_uc"] = qoff
    gaps["rlength"], gaps["glength"] = rl, gl
    gaps["roffset"] = rng.integers(0, 1000, ngaps)
    gaps["goffset"] = goff
    gaps["chroffset"], gaps["chrhigh"] = 0, genome.size
    gaps["watsonp"] = 1
    gaps["jump_late_p"] = rng.random(ngaps) < 0.5
    gaps["widebandp"] = 1
    gaps["extraband_single"] = np.maximum(3, np.abs(gl - rl))
    gaps["max_rlength"], gaps["max_glength"] = max_rlength, max_glength
    gaps["dynprogindex"] = 1
    return gaps, arena


def single_gap_batch(lib, ctx, seed, ngaps=200000, cpu_gaps=20000):
    """Dynprog_single_gap over a batch of stage-3 single gaps, end to end
    through gdp_single_gap_batch (host gaps and sequences in, host records
    out), against the reference's own Dynprog_single_gap on the host (one
    thread, a bounded sample of the same gaps)."""
    import torch
    genome, blocks = gdp.make_genome(lib, 778, 1 << 24)
    ctx.set_genome(blocks, None, genome.size)
    gaps, arena = stage3_gaps(genome, seed, ngaps, 500, 2000)
    res, path, recs = ctx.single_gaps(gaps, arena)
    dp = path == gdp.SINGLE_DP
    rl, gl = gaps["rlength"].astype(np.int64), gaps["glength"].astype(np.int64)
    xb = gaps["extraband_single"].astype(np.int64)
    lb = np.where(gl >= rl, xb, rl - gl + xb)
    ub = np.where(gl >= rl, gl - rl + xb, xb)
    # in-band cells of the fills: rows max(1, c - uband)..min(r, c + lband) per column c
    cells = 0
    for i in np.nonzero(dp)[0]:
        c = np.arange(1, gl[i] + 1)
        cells += int(np.maximum(0, np.minimum(rl[i], c + lb[i]) - np.maximum(1, c - ub[i]) + 1).sum())
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    def pinned(arr):
        t = torch.empty(max(arr.nbytes, 1), dtype=torch.uint8, pin_memory=True)
        a = t.numpy()[:arr.nbytes].view(arr.dtype).reshape(arr.shape)
        a[...] = arr
        return t, a

    keep = [pinned(gaps), pinned(arena), pinned(np.zeros(ngaps, dtype=gdp.RESULT_DTYPE)),
            pinned(np.zeros(ngaps, dtype=np.int8)), pinned(np.zeros(recs.size, dtype=gdp.REC_DTYPE))]
    h_gaps, h_arena, h_res, h_path, h_recs = (k[1] for k in keep)
    used = ctypes.c_int64(0)
    times = []
    for _ in range(4):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = lib.gdp_single_gap_batch(ctx.h, gdp._ptr(h_gaps), ngaps, gdp._ptr(h_arena), h_arena.size,
                                      gdp._ptr(h_res), gdp._ptr(h_path), gdp._ptr(h_recs), h_recs.size,
                                      ctypes.byref(used))
        b.record(stream)
        b.synchronize()
        assert rc == 0 and used.value == recs.size, ctx.error()
        times.append(a.elapsed_time(b))
    ms = statistics.median(times[1:])
    assert np.array_equal(h_res, res) and np.array_equal(h_recs, recs)
    out = {"gaps": ngaps, "simple": int((path == gdp.SINGLE_SIMPLE).sum()), "filled": int(dp.sum()),
           "filled_8bit": int((res["precision"][dp] == 8).sum()), "fill_cells": cells,
           "records": int(recs.size), "ms": round(ms, 3), "gaps_per_s": round(ngaps / (ms * 1e-3), 1),
           "fill_gcups": round(cells / (ms * 1e-3) / 1e9, 3), "bad_status": int((res["status"] != 0).sum()),
           "h2d_bytes": int(gaps.nbytes + arena.nbytes),
           "d2h_bytes": int(res.nbytes + path.nbytes + recs.nbytes),
           "timing": "host gaps and sequences to host records (gdp_single_gap_batch, pinned host "
                     "buffers), median of 3 after one warm-up, CUDA events on the context stream"}
    import oracle
    if cpu_gaps > 0 and oracle.reference_available():
        ref = oracle.reference()
        ref.init(0)
        ref.set_genome(blocks, None, genome.size)
        rs = oracle.ReferenceSingleGap(ref, 200, 40)
        sample = gaps[:cpu_gaps]
        t0 = time.perf_counter()
        st, off, rrecs = rs.run(sample, arena)
        secs = time.perf_counter() - t0
        same = (np.array_equal(st[:, 0], res["tb_score"][:cpu_gaps]) and
                np.array_equal(st[:, 5], res["nrecs"][:cpu_gaps]) and
                np.array_equal(rrecs, recs[:int(res["nrecs"][:cpu_gaps].sum())]))
        out["cpu_baseline"] = {"value": round(cpu_gaps / secs, 1), "unit": "gaps/s", "cores": 1,
                               "kind": "reference",
                               "sample": f"the first {cpu_gaps} gaps, Dynprog_single_gap of oracle/_ref, "
                                         f"{secs:.2f} s on 1 thread",
                               "same_results": bool(same)}
    return out


def per_pair_vs_batched(lib, ctx, seed, npairs=20000, nsample=500):
    """The same mixed-length pairs (70/25/5 short/long/cDNA) aligned as one
    batch and as one plan per pair (every pair its own kernel launches),
    both device-resident, timed with CUDA events on the context's stream."""
    import torch
    genome, blocks = gdp.make_genome(lib, 777, 1 << 24)
    pairs, arena = gdp.make_pairs(lib, gdp.WL_MIX, seed, genome, npairs)
    ctx.set_genome(blocks, None, genome.size)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    d_arena = torch.from_numpy(arena).cuda()
    d_res = torch.empty(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / reps

    plan = ctypes.c_void_p()
    assert lib.gdp_plan_create(ctx.h, gdp._ptr(pairs), pairs.size, ctypes.byref(plan)) == 0, ctx.error()
    d_recs = torch.empty(max(int(lib.gdp_plan_total_recs(plan)), 1) * gdp.REC_DTYPE.itemsize, dtype=torch.uint8,
                         device="cuda")
    batch_ms = timed(lambda: lib.gdp_plan_execute(ctx.h, plan, ctypes.c_void_p(d_pairs.data_ptr()),
                                                  ctypes.c_void_p(d_arena.data_ptr()),
                                                  ctypes.c_void_p(d_res.data_ptr()),
                                                  ctypes.c_void_p(d_recs.data_ptr())), 2)
    batch_res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE).copy()
    lib.gdp_plan_destroy(plan)
    cells = gdp.band_cells(pairs)

    sample = np.arange(min(nsample, pairs.size))
    plans, offs, tot = [], [], 0
    for i in sample:
        pl = ctypes.c_void_p()
        assert lib.gdp_plan_create(ctx.h, gdp._ptr(pairs[i:i + 1]), 1, ctypes.byref(pl)) == 0, ctx.error()
        plans.append(pl)
        offs.append(tot)
        tot += max(int(lib.gdp_plan_total_recs(pl)), 1)
    d_recs1 = torch.empty(tot * gdp.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    pb, ab, rb, cb = d_pairs.data_ptr(), d_arena.data_ptr(), d_res.data_ptr(), d_recs1.data_ptr()

    def one_by_one():
        for k, i in enumerate(sample):
            lib.gdp_plan_execute(ctx.h, plans[k], ctypes.c_void_p(pb + int(i) * gdp.PAIR_DTYPE.itemsize),
                                 ctypes.c_void_p(ab), ctypes.c_void_p(rb + int(i) * gdp.RESULT_DTYPE.itemsize),
                                 ctypes.c_void_p(cb + offs[k] * gdp.REC_DTYPE.itemsize))

    pair_ms = timed(one_by_one, 1)
    one_res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
    for pl in plans:
        lib.gdp_plan_destroy(pl)
    same = all(np.array_equal(one_res[k][sample], batch_res[k][sample])
               for k in ("status", "score", "tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs"))
    batched = float(cells.sum()) / (batch_ms * 1e-3) / 1e9
    per_pair = float(cells[sample].sum()) / (pair_ms * 1e-3) / 1e9
    return {"workload": f"mix 70/25/5 short/long/cDNA, {pairs.size} pairs ({int(cells.sum())} cells)",
            "batched_gcups": round(batched, 3), "per_pair_gcups": round(per_pair, 3),
            "per_pair_sample": f"first {sample.size} of the same pairs, one plan (own launches) per pair",
            "ratio": round(batched / per_pair, 2),
            "batched_alignments_per_s": round(pairs.size / (batch_ms * 1e-3), 1),
            "per_pair_alignments_per_s": round(sample.size / (pair_ms * 1e-3), 1),
            "results_identical": bool(same)}


def serving_sweep(lib, device, seed, rates, seconds_per_rate=1.0, max_requests=400_000, pool_size=20_000,
                  workers=4):
    """The serving loop under Poisson load: single-pair requests of the
    mixed distribution, genome windows extracted on the device from a
    resident 100 Mbp genome, admission by a 40 GB direction budget."""
    genome, blocks = gdp.make_genome(lib, 4242, 100_000_000)
    pool, arena = gdp.make_resident_pairs(lib, gdp.WL_MIX, seed, genome, pool_size)
    cells = gdp.band_cells(pool)
    srv = gdp.Server(lib, device=device, workers=workers, budget=40 << 30, blocks=blocks, length=genome.size)
    srv.drive(pool, arena, 300_000, rate=1e6, seed=1)       # warm-up: every worker's buffers reach working size
    rows = []
    for k, rate in enumerate(rates):
        n = int(min(max_requests, max(200, rate * seconds_per_rate)))
        lat, elapsed, _ = srv.drive(pool, arena, n, rate=rate, seed=100 + k)
        served = cells[np.arange(n) % pool.size].sum()
        rows.append({"offered_per_s": rate, "requests": n,
                     "sustained_per_s": round(n / elapsed, 1),
                     "p50_ms": round(float(np.percentile(lat, 50)), 3),
                     "p99_ms": round(float(np.percentile(lat, 99)), 3),
                     "gcups": round(float(served) / elapsed / 1e9, 2)})
    st = srv.stats()
    srv.close()
    knee = max((r["offered_per_s"] for r in rows if r["sustained_per_s"] >= 0.95 * r["offered_per_s"]),
               default=None)
    return {"genome": "100 Mbp seeded random, resident (genomecomp, 2-bit + N flags)",
            "requests": "single pairs of the 70/25/5 short/long/cDNA mix, device-extracted windows",
            "workers": workers, "dir_budget_gb": 40, "sweep": rows, "knee_offered_per_s": knee,
            "batches": st["batches"], "max_batch_pairs": st["max_batch_pairs"],
            "peak_admitted_dir_gb": round(st["peak_reserved_bytes"] / 2**30, 3)}


def run_reference_arm(args):
    # host cores only: rank 0 runs the sample, the other ranks exit at once
    # (no process group, so nothing waits on rank 0's minutes of CPU work)
    if int(os.environ.get("RANK", "0")) != 0:
        return
    lib = gdp.load()
    name = args.workload
    import oracle
    kind = "reference" if oracle.reference_available() else "port"
    ref = oracle.reference() if kind == "reference" else oracle.restatement()
    ref.init(0)
    threads = os.cpu_count() or 1
    genome, blocks = gdp.make_genome(lib, 777, 1 << 24)
    ref.set_genome(blocks, None, genome.size)
    cal = cpu_baseline(lib, name, args.seed, args.cpu_seconds / max(args.steps, 1), threads, (genome, blocks))
    pairs, arena = cal["data"]
    kept = cal["kept"]
    cells = int(gdp.band_cells(pairs).sum())
    for _ in range(args.warmup):
        m = max(1, pairs.size // 20)
        ref.bench(pairs[:m], arena, threads, kept[:m])
    times = []
    for _ in range(args.steps):
        secs, _ = ref.bench(pairs, arena, threads, kept)
        times.append(secs)
    t = sum(times)
    value = cells * args.steps / t / 1e9
    line = {"metric": "GCUPS (in-band cells, fill + traceback), batched", "value": round(value, 4),
            "unit": "GCUPS", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16/int8",
            "data": "synthetic", "config": {"workload": name, "pairs_per_step": int(pairs.size),
                                            "description": WORKLOADS[name][2]},
            "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": f"{pairs.size} pairs of '{name}' per step, fill + traceback at the "
                                       f"kept precision, on {threads} threads"},
            "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "alignments_per_s": round(pairs.size * args.steps / t, 1)}
    print(json.dumps(line), flush=True)


def run_gdp(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    lib = gdp.load()
    name = args.workload
    npairs = args.npairs or WORKLOADS[name][1]
    genome, blocks, pairs, arena = make_workload(lib, name, npairs, args.seed + 1000 * rank)
    cells = int(gdp.band_cells(pairs).sum())
    ctx = gdp.Context(lib, device=local)
    ctx.set_genome(blocks, None, genome.size)

    # resident inputs and outputs
    plan = ctypes.c_void_p()
    rc = lib.gdp_plan_create(ctx.h, gdp._ptr(pairs), pairs.size, ctypes.byref(plan))
    assert rc == 0, ctx.error()
    total_recs = int(lib.gdp_plan_total_recs(plan))
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    d_arena = torch.from_numpy(arena).cuda()
    d_res = torch.empty(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_recs = torch.empty(max(total_recs, 1) * gdp.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    def step():
        rc = lib.gdp_plan_execute(ctx.h, plan, ctypes.c_void_p(d_pairs.data_ptr()),
                                  ctypes.c_void_p(d_arena.data_ptr()), ctypes.c_void_p(d_res.data_ptr()),
                                  ctypes.c_void_p(d_recs.data_ptr()))
        assert rc == 0, ctx.error()

    for _ in range(args.warmup):
        step()
    lib.gdp_sync(ctx.h)
    res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
    bad = int((res["status"] != 0).sum())

    sampler = ClockSampler(local)
    ctx.profile(True)
    ctx.profile_reset()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = ctx.launches()
    sampler.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step()
    t1.record(stream)
    t1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = ctx.launches() - launches0
    barrier(world)
    ms = t0.elapsed_time(t1)
    prof = ctx.profile_read()
    ctx.profile(False)
    ms_max = max_over_ranks(world, ms)
    total_cells = sum_over_ranks(world, float(cells))
    total_pairs = sum_over_ranks(world, float(pairs.size))
    value = total_cells * args.steps / (ms_max * 1e-3) / 1e9

    # dominant kernel and its roofline (integer issue bound)
    top = max(prof.items(), key=lambda kv: kv[1][0])
    top_name, (top_ms, top_n) = top
    avg_launch_ms = top_ms / top_n
    int_peak = ctx.int_peak()
    achieved_ops = cells * OPS_PER_CELL / (avg_launch_ms * 1e-3)
    dir_bytes = int(lib.gdp_plan_dir_bytes(plan))

    # end to end through the host-buffer C ABI call, inputs and outputs in pinned host memory
    e2e_steps = max(1, min(args.e2e_steps, args.steps))

    def pinned_like(arr):
        t = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
        a = t.numpy().view(arr.dtype).reshape(arr.shape)
        a[...] = arr
        return t, a

    _tp, h_pairs = pinned_like(pairs)
    _ta, h_arena = pinned_like(arena)
    _tr, results = pinned_like(np.zeros(pairs.size, dtype=gdp.RESULT_DTYPE))
    _tc, recs = pinned_like(np.zeros(max(total_recs, 1), dtype=gdp.REC_DTYPE))
    used = ctypes.c_int64(0)

    def e2e_step():
        rc = lib.gdp_align_batch(ctx.h, gdp._ptr(h_pairs), h_pairs.size, gdp._ptr(h_arena), h_arena.size,
                                 gdp._ptr(results), gdp._ptr(recs), recs.size, ctypes.byref(used))
        assert rc == 0, ctx.error()

    e2e_step()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1) / e2e_steps)
    e2e_value = total_cells / (e2e_ms * 1e-3) / 1e9
    h2d = pairs.nbytes + arena.nbytes
    d2h = results.nbytes + int(used.value) * gdp.REC_DTYPE.itemsize
    e2e_bad = int((results["status"] != 0).sum())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(lib, name, args.seed, args.cpu_seconds)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    lib.gdp_plan_destroy(plan)
    extra = {}
    if rank == 0 and world == 1 and not args.no_per_pair:
        extra["per_pair_vs_batched"] = per_pair_vs_batched(lib, ctx, args.seed + 7)
        extra["endpoint_search"] = endpoint_search(lib, ctx, args.seed + 9)
        extra["single_gap"] = single_gap_batch(lib, ctx, args.seed + 10)
    if rank == 0 and world == 1 and not args.no_serving:
        extra["serving"] = serving_sweep(lib, local, args.seed + 8,
                                         [1e3, 1e4, 5e4, 1e5, 2e5, 3e5, 5e5, 1e6])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm = None
    if os.path.exists(peaks_path):
        hbm = json.load(open(peaks_path)).get("hbm_gbs")
    # DRAM bytes of the dominant kernel per launch: one ncu capture of the same
    # kernel on 50,000 pairs of this workload (dram__bytes_read.sum +
    # dram__bytes_write.sum = 123.70 + 266.46 MB over 300,657,762 in-band
    # cells), scaled to this launch by its in-band cells; the kernel's bytes
    # grow with the cells (directions and carries per swept cell)
    traffic, traffic_src = None, None
    if name == "short" and top_name.startswith("fill_thread<W16,full"):
        traffic = int(round((123.696896e6 + 266.455296e6) / 300657762 * cells))
        traffic_src = ("ncu capture of this kernel on 50,000 pairs (390.2 MB), scaled by in-band cells "
                       "to this launch")
    if rank == 0:
        line = {
            "metric": "GCUPS (in-band cells, fill + traceback), batched",
            "value": round(value, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16/int8", "data": "synthetic",
            "config": {"workload": name, "pairs_per_gpu": int(pairs.size), "description": WORKLOADS[name][2],
                       "cells_per_gpu": cells, "l2": "inputs larger than L2 (sequence arena %.0f MB, "
                       "direction words %.0f MB per step)" % (arena.nbytes / 1e6, dir_bytes / 1e6),
                       "parallelism": f"pairs sharded, {world} independent rank(s)"},
            "alignments_per_s": round(total_pairs * args.steps / (ms_max * 1e-3), 1),
            "e2e": {"value": round(e2e_value, 3), "unit": "GCUPS", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3),
                    "host_buffers": "pinned", "bad_status_pairs": e2e_bad},
            "roofline": {"bound": "int", "kernel": top_name,
                         "achieved": round(achieved_ops / 1e12, 3), "peak": round(int_peak / 1e12, 3),
                         "unit": "Tops/s (int32 lane-ops)", "frac": round(achieved_ops / int_peak, 4),
                         "peak_source": "measured int32 issue probe (gdp_measure_int_peak)",
                         "ops_per_cell": OPS_PER_CELL, "avg_launch_ms": round(avg_launch_ms, 3),
                         "traffic": traffic,
                         "traffic_source": traffic_src,
                         "dir_write_gbs": round(dir_bytes / (avg_launch_ms * 1e-3) / 1e9, 1),
                         "hbm_peak_gbs": hbm},
            "kernels": {k: {"ms_total": round(v[0], 3), "launches": v[1]} for k, v in prof.items()},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "bad_status_pairs": bad,
            "cpu_baseline": cpu,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gdp", "reference"], default="gdp")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="short")
    ap.add_argument("--npairs", type=int, default=0)
    ap.add_argument("--seed", type=int, default=1002)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-pair", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gdp(args)


if __name__ == "__main__":
    main()
