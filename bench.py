#!/usr/bin/env python
"""Benchmark of the batched banded affine-gap DP path (fills + tracebacks).

Default workload (one step = one batch): 1,000,000 short-read pairs,
rlength U{75..300}, lband/uband U{3..30}, 3% substitutions, 1% indels, 5%
random non-matching windows, 8-bit fills with the 16-bit rerun on overflow,
traceback of every pair.  Synthetic, seeded.  Metric: GCUPS over the
in-band cells of the reference's compare domain, whole job, fill +
traceback.  `value` is measured with pairs and sequences resident in HBM,
the plan replayed as a CUDA graph with the autotuner's routing in force;
`e2e` goes through the host-buffer C-ABI call gdp_align_batch (host->device
copies, planning, kernels, device->host copies of results and Pair records
all inside the timed region).  The CPU leg times the reference on a prefix
of the same pairs and checks the device's outputs on it pair by pair
(`parity`).  Configurations 1 (10,000 fixed 150 x 160 pairs), 3 (50,000
cDNA gaps, upper and lower fills) and 4 (2,000,000 mixed pairs) are
measured at their sizes beside it, each with its CPU figure and parity
sample on the same pairs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gdp|reference]

For N > 1 launch with torchrun; each rank aligns its own shard of the same
size (weak scaling, no data-path collective: pairs are independent).
`--impl reference` times the reference's own CPU code (oracle/_ref, built
from the reference sources) on the host cores over a prefix of the same
pairs; that process loads no CUDA library.
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
    "mix": (gdp.WL_MIX, 2_000_000, "70/25/5 short/long/cDNA draws (a cDNA draw is its upper and lower fill)"),
    "cdna": (gdp.WL_CDNA, 100_000, "cDNA gaps, r log-U[200,5000], g = r U(1,1.5): upper fill (uband g-r+14) "
                                    "with traceback plus lower fill (lband 14), 16-bit"),
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
    """The seeded workload `name` (libgdp.so or the standalone generator
    libgdpwl.so give the same pairs)."""
    kind = WORKLOADS[name][0]
    genome, blocks = gdp.make_genome(lib, 777, genome_len)
    pairs, arena = gdp.make_pairs(lib, kind, seed, genome, npairs)
    return genome, blocks, pairs, arena


def _final_cell_in_band(pairs):
    """Whether each pair's final cell (rlength, glength) lies in its band:
    outside it the reference leaves the cell unwritten (a cDNA gap's lower
    fill when glength > rlength), so no final score is compared there."""
    d = pairs["rlength"].astype(np.int64) - pairs["glength"].astype(np.int64)
    v = pairs["variant"]
    lo = np.where(v == gdp.FULL, -pairs["uband"].astype(np.int64),
                  np.where(v == gdp.UPPER, -pairs["uband"].astype(np.int64), 0))
    hi = np.where(v == gdp.UPPER, 0, pairs["lband"].astype(np.int64))
    return (d >= lo) & (d <= hi)


def parity_sample(sample, kept, ref_out, res, recs):
    """Per sampled pair, the device's outputs (results and records of the
    same pairs) against the reference's (ref_out from oracle outputs()):
    status, kept precision, final score, traceback score and counts,
    record count and record digest."""
    n = sample.size
    res = res[:n]
    tb = (sample["flags"] & gdp.FLAG_TRACEBACK) != 0
    want_prec = np.where((sample["precision"] == 8) & ((sample["flags"] & gdp.FLAG_RERUN16) != 0),
                         kept, sample["precision"])
    ok = (res["status"] == 0) & (res["precision"] == want_prec)
    ok &= ~_final_cell_in_band(sample) | (res["score"] == ref_out[:, 0])
    for j, k in enumerate(("tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs")):
        ok &= ~tb | (res[k] == ref_out[:, 1 + j])
    dig = gdp.record_digests(recs, np.where(tb, res["rec_offset"], 0), np.where(tb, res["nrecs"], 0))
    ok &= ~tb | (dig == ref_out[:, 7].view(np.uint32))
    bad = np.nonzero(~ok)[0]
    return {"pairs": int(n), "mismatches": int(bad.size), "first_mismatches": bad[:5].tolist(),
            "compared": "status, kept precision, final score, traceback score and counts, record count "
                        "and a digest of every Pair record, per pair"}


def cpu_leg(pairs, arena, blocks, genome_len, seconds, threads=None, res=None, recs=None, max_pairs=None):
    """The reference's own code (oracle/_ref; the restatement when the
    reference is absent) timed on the host cores over a prefix of the very
    pairs the device aligned, sized to about `seconds`: every pair once at
    the precision the rerun contract keeps (from the restatement, untimed).
    Beside it the same build with the per-column _mm_clflush compiled out
    (the "strong CPU" figure) on the same sample, and -- given the device's
    results and records of those pairs -- the per-pair parity of the
    sample (an untimed run with outputs)."""
    import oracle
    kind = "reference" if oracle.reference_available() else "port"
    ref = oracle.reference() if kind == "reference" else oracle.restatement()
    ref.init(0)
    ref.set_genome(blocks, None, genome_len)
    rest = oracle.restatement()
    rest.init(0)
    rest.set_genome(blocks, None, genome_len)
    threads = threads or os.cpu_count() or 1
    limit = min(pairs.size, max_pairs or pairs.size)
    n = min(limit, 256)
    while True:
        sample = pairs[:n]
        kept = rest.kept_precision(sample, arena, threads)
        secs, _ = ref.bench(sample, arena, threads, kept)
        if n >= limit or secs >= seconds * 0.7:
            break
        n = min(limit, int(n * min(16.0, max(1.3, seconds / max(secs, 1e-4)))))
    cells = int(gdp.band_cells(sample).sum())
    out = {"value": round(cells / secs / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
           "sample": f"the first {n} of the same pairs ({cells} in-band cells), fill + traceback at the "
                     f"kept precision ({int((kept == 8).sum())} 8-bit), {secs:.2f} s wall on {threads} threads",
           "seconds": round(secs, 3), "pairs": int(n), "cells": cells,
           "alignments_per_s": round(n / secs, 1)}
    if kind == "reference" and os.path.exists(oracle.REF_LIB_NOFLUSH):
        nf = oracle.reference(noflush=True)
        nf.init(0)
        nf.set_genome(blocks, None, genome_len)
        s2, _ = nf.bench(sample, arena, threads, kept)
        out["noflush"] = {"value": round(cells / s2 / 1e9, 4), "unit": "GCUPS", "cores": threads,
                          "seconds": round(s2, 3),
                          "build": "the same reference sources with the per-column _mm_clflush compiled out "
                                   "(oracle/_ref/libgdpref_noflush.so)"}
    if res is not None:
        _, ref_out = ref.outputs(sample, arena, threads, kept)
        out["parity"] = parity_sample(sample, kept, ref_out, res, recs)
    return out


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


def single_gap_batch(lib, ctx, seed, ngaps=200000, cpu_gaps=100000):
    """Dynprog_single_gap over a batch of stage-3 single gaps, end to end
    through gdp_single_gap_batch (host gaps and sequences in, host records
    out), against the reference's own Dynprog_single_gap on the host (all
    host threads, each with its own Dynprog_T and Pairpool_T, over a
    bounded prefix of the same gaps; its results are checked against the
    device's on that prefix, untimed)."""
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
        threads = os.cpu_count() or 1
        secs, _ = rs.bench(sample, arena, threads, 200, 40)
        secs1, _ = rs.bench(sample[:cpu_gaps // 8], arena, 1, 200, 40)
        st, off, rrecs = rs.run(sample, arena)
        same = (np.array_equal(st[:, 0], res["tb_score"][:cpu_gaps]) and
                np.array_equal(st[:, 5], res["nrecs"][:cpu_gaps]) and
                np.array_equal(rrecs, recs[:int(res["nrecs"][:cpu_gaps].sum())]))
        out["cpu_baseline"] = {"value": round(cpu_gaps / secs, 1), "unit": "gaps/s", "cores": threads,
                               "kind": "reference",
                               "sample": f"the first {cpu_gaps} gaps, Dynprog_single_gap of oracle/_ref, "
                                         f"{secs:.2f} s on {threads} threads",
                               "one_thread_gaps_per_s": round((cpu_gaps // 8) / secs1, 1),
                               "same_results": bool(same)}
    return out



def stage3_end_gaps(genome, seed, ngaps, max_rlength, max_glength):
    """End gaps as stage 3 sends them to Dynprog_end5_gap / Dynprog_end3_gap:
    the query beyond the first (end 5) or last (end 3) aligned block, 8..250
    nt (log-uniform), against the genome stretch next to the block, 0..32 nt
    longer; half end 5, half end 3; the query matches the genome next to the
    block with 1 % substitutions, and for 30 % of gaps only over a random
    part of its length (an unaligned tail: adapter, poly-A, a missed exon);
    75 % QUERYEND_GAP, 25 % QUERYEND_INDELS; extraband_end 6; plus strand."""
    rng = np.random.default_rng(seed)
    rl = np.exp(rng.uniform(np.log(8), np.log(251), ngaps)).astype(np.int64)
    gl = rl + rng.integers(0, 33, ngaps)
    end5 = rng.random(ngaps) < 0.5
    L = genome.size
    goff = np.where(end5, rng.integers(512, L - 512, ngaps), rng.integers(0, L - 512, ngaps))
    keep = np.where(rng.random(ngaps) < 0.3, (rng.random(ngaps) * rl).astype(np.int64), rl)
    tot = int(rl.sum())
    qoff = np.zeros(ngaps, np.int64)
    qoff[1:] = np.cumsum(rl)[:-1]
    k = np.arange(tot) - np.repeat(qoff, rl)               # position in the query
    rlr, keepr, goffr, e5 = (np.repeat(a, rl) for a in (rl, keep, goff, end5))
    # end 3: query k against genome goff + k; end 5: query k against genome goff - (rl - 1) + k
    idx = np.where(e5, goffr - (rlr - 1) + k, goffr + k)
    q = genome[idx].copy()
    tail = np.where(e5, k < rlr - keepr, k >= keepr)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    q[tail] = rng.choice(acgt, size=int(tail.sum()))
    sub = rng.random(tot) < 0.01
    q[sub] = rng.choice(acgt, size=int(sub.sum()))
    q[q == ord("N")] = ord("A")
    gaps = np.zeros(ngaps, dtype=gdp.END_GAP_DTYPE)
    gaps["rseq"] = gaps["rseq_uc"] = np.where(end5, qoff + rl - 1, qoff)
    gaps["rlength"], gaps["glength"] = rl, gl
    gaps["roffset"] = np.where(end5, rl - 1 + rng.integers(0, 1000, ngaps), rng.integers(0, 1000, ngaps))
    gaps["goffset"] = goff
    gaps["chroffset"], gaps["chrhigh"] = 0, L
    gaps["end"] = np.where(end5, 5, 3)
    gaps["endalign"] = np.where(rng.random(ngaps) < 0.75, gdp.QUERYEND_GAP, gdp.QUERYEND_INDELS)
    gaps["watsonp"] = 1
    gaps["jump_late_p"] = rng.random(ngaps) < 0.5
    gaps["extraband_end"] = 6
    gaps["max_rlength"], gaps["max_glength"] = max_rlength, max_glength
    gaps["dynprogindex"] = 1
    return gaps, q


def end_gap_cells(gaps):
    """In-band cells of the upper and the lower fill of each end gap (the
    reference computes both): upper rows max(1, c - uband)..min(r, c) per
    column c, lower columns max(1, r - lband)..min(g, r) per row r."""
    rl, gl = gaps["rlength"].astype(np.int64), gaps["glength"].astype(np.int64)
    xb = gaps["extraband_end"].astype(np.int64)
    wide = gaps["endalign"] != gdp.QUERYEND_INDELS
    ub = np.where(wide & (gl >= rl), gl - rl + xb, xb)
    lb = np.where(wide & (gl < rl), rl - gl + xb, xb)
    cells = 0
    for i in range(gaps.size):
        c = np.arange(1, gl[i] + 1)
        cells += int(np.maximum(0, np.minimum(rl[i], c) - np.maximum(1, c - ub[i]) + 1).sum())
        r = np.arange(1, rl[i] + 1)
        cells += int(np.maximum(0, np.minimum(gl[i], r) - np.maximum(1, r - lb[i]) + 1).sum())
    return cells


def end_gap_batch(lib, ctx, seed, ngaps=200000, cpu_gaps=50000):
    """Dynprog_end5_gap / Dynprog_end3_gap over a batch of stage-3 end gaps,
    end to end through gdp_end_gap_batch (host gaps and sequences in, host
    records out), against the reference's own end-gap solvers on the host
    (all host threads, each with its own Dynprog_T and Pairpool_T, over a
    bounded prefix of the same gaps; its results are checked against the
    device's on that prefix, untimed)."""
    import torch
    genome, blocks = gdp.make_genome(lib, 779, 1 << 24)
    ctx.set_genome(blocks, None, genome.size)
    gaps, arena = stage3_end_gaps(genome, seed, ngaps, 500, 2000)
    res, recs = ctx.end_gaps(gaps, arena)
    cells = end_gap_cells(gaps)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    def pinned(arr):
        t = torch.empty(max(arr.nbytes, 1), dtype=torch.uint8, pin_memory=True)
        a = t.numpy()[:arr.nbytes].view(arr.dtype).reshape(arr.shape)
        a[...] = arr
        return t, a

    keep = [pinned(gaps), pinned(arena), pinned(np.zeros(ngaps, dtype=gdp.RESULT_DTYPE)),
            pinned(np.zeros(max(recs.size, 1), dtype=gdp.REC_DTYPE))]
    h_gaps, h_arena, h_res, h_recs = (k[1] for k in keep)
    used = ctypes.c_int64(0)
    times = []
    for _ in range(4):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = lib.gdp_end_gap_batch(ctx.h, gdp._ptr(h_gaps), ngaps, gdp._ptr(h_arena), h_arena.size,
                                   gdp._ptr(h_res), gdp._ptr(h_recs), h_recs.size, ctypes.byref(used))
        b.record(stream)
        b.synchronize()
        assert rc == 0 and used.value == recs.size, ctx.error()
        times.append(a.elapsed_time(b))
    ms = statistics.median(times[1:])
    assert np.array_equal(h_res, res) and np.array_equal(h_recs[:recs.size], recs)
    out = {"gaps": ngaps, "end5": int((gaps["end"] == 5).sum()),
           "filled_8bit": int((res["precision"] == 8).sum()), "fill_cells": cells,
           "records": int(recs.size), "ms": round(ms, 3), "gaps_per_s": round(ngaps / (ms * 1e-3), 1),
           "fill_gcups": round(cells / (ms * 1e-3) / 1e9, 3), "bad_status": int((res["status"] != 0).sum()),
           "h2d_bytes": int(gaps.nbytes + arena.nbytes), "d2h_bytes": int(res.nbytes + recs.nbytes),
           "timing": "host gaps and sequences to host records (gdp_end_gap_batch, pinned host "
                     "buffers), median of 3 after one warm-up, CUDA events on the context stream"}
    import oracle
    if cpu_gaps > 0 and oracle.reference_available():
        ref = oracle.reference()
        ref.init(0)
        ref.set_genome(blocks, None, genome.size)
        re = oracle.ReferenceEndGap(ref, 200, 40)
        re.setup()
        sample = gaps[:cpu_gaps]
        threads = os.cpu_count() or 1
        secs, _ = re.bench(sample, arena, threads, 200, 40)
        secs1, _ = re.bench(sample[:cpu_gaps // 8], arena, 1, 200, 40)
        st, off, rrecs = re.run(sample, arena)
        same = (np.array_equal(st[:, 0], res["tb_score"][:cpu_gaps]) and
                np.array_equal(st[:, 5], res["nrecs"][:cpu_gaps]) and
                np.array_equal(rrecs, recs[:int(res["nrecs"][:cpu_gaps].sum())]))
        out["cpu_baseline"] = {"value": round(cpu_gaps / secs, 1), "unit": "gaps/s", "cores": threads,
                               "kind": "reference",
                               "sample": f"the first {cpu_gaps} gaps, Dynprog_end5_gap / Dynprog_end3_gap of "
                                         f"oracle/_ref, {secs:.2f} s on {threads} threads",
                               "one_thread_gaps_per_s": round((cpu_gaps // 8) / secs1, 1),
                               "same_results": bool(same)}
    return out


def stage3_cdna_gaps(genome, seed, ngaps, max_rlength, max_glength):
    """cDNA gaps as stage 3 sends them to Dynprog_cdna_gap (src/stage3.c:
    9313): a genome gap of 20..150 nt (log-uniform) between two aligned
    blocks, a query gap 10..60 nt longer (an insertion of unrelated bases at
    a random place, 1 % substitutions elsewhere), both query stretches
    glength + 10 long (extramaterial_paired), extraband_paired 6, plus
    strand, HIGHQ, both tie rules."""
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    gaps = np.zeros(ngaps, dtype=gdp.CDNA_GAP_DTYPE)
    gl = np.exp(rng.uniform(np.log(20), np.log(151), ngaps)).astype(np.int64)
    ins = rng.integers(10, 61, ngaps)
    goff = rng.integers(1000, genome.size - 1000, ngaps)
    chunks, off = [], 0
    for i in range(ngaps):
        g, k = int(gl[i]), int(ins[i])
        rl = g + 10
        seg = genome[goff[i]:goff[i] + g].copy()
        s = int(rng.integers(0, g + 1))
        mid = np.concatenate([seg[:s], rng.choice(acgt, size=k), seg[s:]])
        sub = rng.random(mid.size) < 0.01
        mid[sub] = rng.choice(acgt, size=int(sub.sum()))
        q = np.concatenate([rng.choice(acgt, size=rl + 4), mid, rng.choice(acgt, size=rl + 4)])
        q[q == ord("N")] = ord("A")
        gaps["rseq"][i] = gaps["rseq_uc"][i] = off + rl + 4
        gaps["rlengthL"][i] = gaps["rlengthR"][i] = rl
        gaps["glength"][i] = g
        gaps["roffsetL"][i] = 100
        gaps["rev_roffsetR"][i] = 100 + mid.size - 1
        gaps["goffset"][i] = goff[i]
        chunks.append(q)
        off += q.size
    gaps["chroffset"], gaps["chrhigh"] = 0, genome.size
    gaps["watsonp"] = 1
    gaps["jump_late_p"] = rng.random(ngaps) < 0.5
    gaps["extraband_paired"] = 6
    gaps["max_rlength"], gaps["max_glength"] = max_rlength, max_glength
    gaps["dynprogindex"] = 1
    return gaps, np.concatenate(chunks)


def cdna_gap_batch(lib, ctx, seed, ngaps=20000, cpu_gaps=5000):
    """Dynprog_cdna_gap over a batch of stage-3 cDNA gaps, end to end through
    gdp_cdna_gap_batch (host gaps and sequences in, host records out),
    against the reference's own Dynprog_cdna_gap on the host (all host
    threads over a bounded prefix of the same gaps; its results are checked
    against the device's on that prefix, untimed)."""
    import torch
    genome, blocks = gdp.make_genome(lib, 780, 1 << 24)
    ctx.set_genome(blocks, None, genome.size)
    gaps, arena = stage3_cdna_gaps(genome, seed, ngaps, 500, 2000)
    res, recs = ctx.cdna_gaps(gaps, arena)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    def pinned(arr):
        t = torch.empty(max(arr.nbytes, 1), dtype=torch.uint8, pin_memory=True)
        a = t.numpy()[:arr.nbytes].view(arr.dtype).reshape(arr.shape)
        a[...] = arr
        return t, a

    keep = [pinned(gaps), pinned(arena), pinned(np.zeros(ngaps, dtype=gdp.RESULT_DTYPE)),
            pinned(np.zeros(max(recs.size, 1), dtype=gdp.REC_DTYPE))]
    h_gaps, h_arena, h_res, h_recs = (k[1] for k in keep)
    used = ctypes.c_int64(0)
    times = []
    for _ in range(4):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rc = lib.gdp_cdna_gap_batch(ctx.h, gdp._ptr(h_gaps), ngaps, gdp._ptr(h_arena), h_arena.size,
                                    gdp._ptr(h_res), gdp._ptr(h_recs), h_recs.size, ctypes.byref(used))
        b.record(stream)
        b.synchronize()
        assert rc == 0 and used.value == recs.size, ctx.error()
        times.append(a.elapsed_time(b))
    ms = statistics.median(times[1:])
    assert np.array_equal(h_res, res) and np.array_equal(h_recs[:recs.size], recs)
    out = {"gaps": ngaps, "incomplete": int(res["end_found"].sum()), "filled_8bit": int((res["precision"] == 8).sum()),
           "records": int(recs.size), "ms": round(ms, 3), "gaps_per_s": round(ngaps / (ms * 1e-3), 1),
           "bad_status": int((res["status"] != 0).sum()),
           "h2d_bytes": int(gaps.nbytes + arena.nbytes), "d2h_bytes": int(res.nbytes + recs.nbytes),
           "timing": "host gaps and sequences to host records (gdp_cdna_gap_batch, pinned host "
                     "buffers), median of 3 after one warm-up, CUDA events on the context stream"}
    import oracle
    if cpu_gaps > 0 and oracle.reference_available():
        ref = oracle.reference()
        ref.init(0)
        ref.set_genome(blocks, None, genome.size)
        rc_ = oracle.ReferenceCdnaGap(ref, 200, 40)
        sample = gaps[:cpu_gaps]
        threads = os.cpu_count() or 1
        secs, _ = rc_.bench(sample, arena, threads, 200, 40)
        st, off, rrecs = rc_.run(sample, arena)
        same = (np.array_equal(st[:, 0], res["tb_score"][:cpu_gaps]) and
                np.array_equal(st[:, 5], res["nrecs"][:cpu_gaps]) and
                np.array_equal(rrecs, recs[:int(res["nrecs"][:cpu_gaps].sum())]))
        out["cpu_baseline"] = {"value": round(cpu_gaps / secs, 1), "unit": "gaps/s", "cores": threads,
                               "kind": "reference",
                               "sample": f"the first {cpu_gaps} gaps, Dynprog_cdna_gap of oracle/_ref, "
                                         f"{secs:.2f} s on {threads} threads",
                               "same_results": bool(same)}
    return out

def serving_sweep(lib, device, seed, rates, seconds_per_rate=2.0, max_requests=400_000, pool_size=20_000,
                  workers=4):
    """The serving loop under Poisson load: single-pair requests of the
    mixed distribution, genome windows extracted on the device from a
    resident 100 Mbp genome, admission by a 40 GB direction budget.  Each
    rate runs for `seconds_per_rate` of arrivals (at most max_requests
    requests); the sustained rate is the requests over the time from the
    first arrival to the last completion, so the last requests' latency
    (about 0.1 s for long reads) weighs less in a longer window."""
    genome, blocks = gdp.make_genome(lib, 4242, 100_000_000)
    pool, arena = gdp.make_resident_pairs(lib, gdp.WL_MIX, seed, genome, pool_size)
    cells = gdp.band_cells(pool)
    srv = gdp.Server(lib, device=device, workers=workers, budget=40 << 30, blocks=blocks, length=genome.size)
    cls = srv.classes(pool)                                  # 0 short, 1 long (longest stretch > 512)
    srv.drive(pool, arena, 300_000, rate=1e6, seed=1)       # warm-up: every worker's buffers reach working size
    rows = []
    for k, rate in enumerate(rates):
        n = int(min(max_requests, max(200, rate * seconds_per_rate)))
        lat, elapsed, _ = srv.drive(pool, arena, n, rate=rate, seed=100 + k)
        served = cells[np.arange(n) % pool.size].sum()
        c = cls[np.arange(n) % pool.size]
        row = {"offered_per_s": rate, "requests": n,
               "sustained_per_s": round(n / elapsed, 1),
               "p50_ms": round(float(np.percentile(lat, 50)), 3),
               "p99_ms": round(float(np.percentile(lat, 99)), 3),
               "gcups": round(float(served) / elapsed / 1e9, 2)}
        for k, label in ((0, "short"), (1, "long")):
            if (c == k).any():
                row[f"{label}_p50_ms"] = round(float(np.percentile(lat[c == k], 50)), 3)
                row[f"{label}_p99_ms"] = round(float(np.percentile(lat[c == k], 99)), 3)
        rows.append(row)
    st = srv.stats()
    srv.close()
    knee = max((r["offered_per_s"] for r in rows if r["sustained_per_s"] >= 0.95 * r["offered_per_s"]),
               default=None)
    return {"genome": "100 Mbp seeded random, resident (genomecomp, 2-bit + N flags)",
            "requests": "single pairs of the 70/25/5 short/long/cDNA mix, device-extracted windows",
            "workers": workers, "dir_budget_gb": 40, "sweep": rows, "knee_offered_per_s": knee,
            "classes": {"short": "longest stretch <= 512 nt, batched apart on the higher stream priority, "
                                 "served by three workers in four (and by the others when no long request waits)",
                        "short_share": round(float((cls == 0).mean()), 3),
                        "class_batches": st["class_batches"], "class_pairs": st["class_pairs"]},
            "batches": st["batches"], "max_batch_pairs": st["max_batch_pairs"],
            "peak_admitted_dir_gb": round(st["peak_reserved_bytes"] / 2**30, 3)}


def per_pair_concurrent(lib, pairs, arena, blocks, genome_len, sample, res0, params, nthreads=8):
    """The per-pair GPU path as a multi-threaded caller uses it (GMAP's
    worker threads each calling the reference-signature entry points): the
    sample split over `nthreads` host threads, each with its own context
    (own streams, the routing parameters `params`) executing one one-pair
    plan per pair back to back, all threads at once.  Wall clock from a
    device-wide synchronize before the first launch to one after the last."""
    import torch
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    d_arena = torch.from_numpy(arena).cuda()
    d_res = torch.empty(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    slices = np.array_split(sample, nthreads)
    ctxs, plans, offs, tot = [], [], [], 0
    for sl in slices:
        c = gdp.Context(lib, device=torch.cuda.current_device())
        c.set_genome(blocks, None, genome_len)
        for k, v in params.items():
            lib.gdp_ctx_set_param(c.h, k.encode(), int(v))
        pl_c, off_c = [], []
        for i in sl:
            pl = ctypes.c_void_p()
            assert lib.gdp_plan_create(c.h, gdp._ptr(pairs[i:i + 1]), 1, ctypes.byref(pl)) == 0, c.error()
            pl_c.append(pl)
            off_c.append(tot)
            tot += max(int(lib.gdp_plan_total_recs(pl)), 1)
        ctxs.append(c)
        plans.append(pl_c)
        offs.append(off_c)
    d_recs = torch.empty(tot * gdp.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    pb, ab, rb, cb = d_pairs.data_ptr(), d_arena.data_ptr(), d_res.data_ptr(), d_recs.data_ptr()

    def run(t):
        c = ctxs[t]
        for j, i in enumerate(slices[t]):
            lib.gdp_plan_execute(c.h, plans[t][j], ctypes.c_void_p(pb + int(i) * gdp.PAIR_DTYPE.itemsize),
                                 ctypes.c_void_p(ab), ctypes.c_void_p(rb + int(i) * gdp.RESULT_DTYPE.itemsize),
                                 ctypes.c_void_p(cb + offs[t][j] * gdp.REC_DTYPE.itemsize))
        lib.gdp_sync(c.h)

    def all_threads():
        th = [threading.Thread(target=run, args=(t,)) for t in range(nthreads)]
        for x in th:
            x.start()
        for x in th:
            x.join()

    all_threads()                      # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    all_threads()
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    one = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
    for t in range(nthreads):
        for pl in plans[t]:
            lib.gdp_plan_destroy(pl)
        ctxs[t].close()
    same = all(np.array_equal(one[k][sample], res0[k][sample])
               for k in ("status", "score", "precision", "tb_score", "nmatches", "nmismatches", "nopens",
                         "nindels", "nrecs"))
    pcells = float(gdp.band_cells(pairs[sample]).sum())
    return {"gcups": round(pcells / (wall_ms * 1e-3) / 1e9, 3), "pairs": int(sample.size),
            "threads": nthreads, "alignments_per_s": round(sample.size / (wall_ms * 1e-3), 1),
            "sample": f"the same {sample.size} pairs, one plan per pair, {nthreads} host threads each with its "
                      f"own context, concurrently; wall clock between device-wide synchronizes",
            "results_identical_to_batch": bool(same)}


def measure_config(lib, ctx, label, name, npairs, seed, chunk, cpu_seconds, genome=None, tune_pairs=0,
                   per_pair=0, cpu_max_pairs=None):
    """One workload at its stated size on the device, chunk by chunk (each
    chunk its own seeded draw of the distribution, generated outside every
    timed region):
      * device: each chunk as a device-resident plan executed as a CUDA
        graph (the first execution runs and captures the plan, the second,
        timed, launches the graph);
      * e2e: each chunk through gdp_align_batch from pinned host buffers to
        host results and Pair records (the internal waves stream the
        direction memory);
      * per_pair (optional): the first `per_pair` pairs, one plan each;
      * cpu_baseline: the reference on a prefix of chunk 0, with the
        per-pair parity of that prefix against chunk 0's e2e outputs.
    With tune_pairs, gdp_autotune first picks the routing parameters on a
    separate draw of the same distribution, and they stay in force."""
    import torch
    kind = WORKLOADS[name][0]
    if genome is None:
        genome, blocks = gdp.make_genome(lib, 777, 1 << 24)
    else:
        genome, blocks = genome
    ctx.set_genome(blocks, None, genome.size)
    out = {"workload": WORKLOADS[name][2], "pairs": int(npairs), "chunk_pairs": int(chunk)}
    if tune_pairs:
        tp, ta = gdp.make_pairs(lib, kind, seed + 4242, genome, tune_pairs)
        params, best = ctx.autotune(tp, ta)
        out["autotune"] = {"sample_pairs": int(tune_pairs), "params": params, "sample_ms": round(best, 3)}
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    nchunks = (npairs + chunk - 1) // chunk
    cells = dev_ms = e2e_ms = 0.0
    bad = e2e_bad = launches = h2d = d2h = 0
    first = None
    host = {}

    def pinned(key, nbytes):
        have = host.get(key)
        if have is None or have.numel() < nbytes:
            host[key] = torch.empty(max(nbytes, 16), dtype=torch.uint8, pin_memory=True)
        return host[key]

    for k in range(nchunks):
        m = min(chunk, npairs - k * chunk)
        pairs, arena = gdp.make_pairs(lib, kind, seed + k, genome, m)
        cells += float(gdp.band_cells(pairs).sum())
        plan = ctypes.c_void_p()
        assert lib.gdp_plan_create(ctx.h, gdp._ptr(pairs), pairs.size, ctypes.byref(plan)) == 0, ctx.error()
        lib.gdp_plan_use_graph(plan, 1)
        total_recs = int(lib.gdp_plan_total_recs(plan))
        d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
        d_arena = torch.from_numpy(arena).cuda()
        d_res = torch.empty(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        d_recs = torch.empty(max(total_recs, 1) * gdp.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        args4 = [ctypes.c_void_p(t.data_ptr()) for t in (d_pairs, d_arena, d_res, d_recs)]
        assert lib.gdp_plan_execute(ctx.h, plan, *args4) == 0, ctx.error()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launches()
        a.record(stream)
        assert lib.gdp_plan_execute(ctx.h, plan, *args4) == 0, ctx.error()
        b.record(stream)
        b.synchronize()
        launches += ctx.launches() - l0
        dev_ms += a.elapsed_time(b)
        res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
        bad += int((res["status"] != 0).sum())
        lib.gdp_plan_destroy(plan)
        del d_pairs, d_arena, d_res, d_recs
        torch.cuda.empty_cache()
        # end to end from pinned host buffers
        hp = pinned("pairs", pairs.nbytes).numpy()[:pairs.nbytes].view(gdp.PAIR_DTYPE)
        hp[...] = pairs
        ha = pinned("arena", arena.nbytes).numpy()[:arena.nbytes]
        ha[...] = arena
        hr = pinned("res", pairs.size * gdp.RESULT_DTYPE.itemsize).numpy()[
            :pairs.size * gdp.RESULT_DTYPE.itemsize].view(gdp.RESULT_DTYPE)
        cap = max(total_recs, 1)
        hc = pinned("recs", cap * gdp.REC_DTYPE.itemsize).numpy()[:cap * gdp.REC_DTYPE.itemsize].view(gdp.REC_DTYPE)
        used = ctypes.c_int64(0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.gdp_align_batch(ctx.h, gdp._ptr(hp), hp.size, gdp._ptr(ha), ha.size, gdp._ptr(hr), gdp._ptr(hc),
                                 cap, ctypes.byref(used))
        e1.record(stream)
        e1.synchronize()
        assert rc == 0, ctx.error()
        e2e_ms += e0.elapsed_time(e1)
        e2e_bad += int((hr["status"] != 0).sum())
        h2d += pairs.nbytes + arena.nbytes
        d2h += hr.nbytes + int(used.value) * gdp.REC_DTYPE.itemsize
        if k == 0:
            first = (pairs, arena, hr.copy(), hc[:int(used.value)].copy())
    out["device"] = {"gcups": round(cells / (dev_ms * 1e-3) / 1e9, 3), "ms": round(dev_ms, 3),
                     "alignments_per_s": round(npairs / (dev_ms * 1e-3), 1), "graph": True,
                     "gpu_launches": int(launches), "bad_status_pairs": bad,
                     "timing": "device-resident plans, one per chunk, each executed as a CUDA graph; "
                               "CUDA events on the context stream around each chunk's graph launch"}
    out["e2e"] = {"gcups": round(cells / (e2e_ms * 1e-3) / 1e9, 3), "ms": round(e2e_ms, 3),
                  "h2d_bytes": int(h2d), "d2h_bytes": int(d2h), "bad_status_pairs": e2e_bad,
                  "host_buffers": "pinned"}
    out["cells"] = int(cells)
    pairs, arena, res0, recs0 = first
    if per_pair:
        sample = np.arange(min(per_pair, pairs.size))
        d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
        d_arena = torch.from_numpy(arena).cuda()
        d_res = torch.empty(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        plans, offs, tot = [], [], 0
        for i in sample:
            pl = ctypes.c_void_p()
            assert lib.gdp_plan_create(ctx.h, gdp._ptr(pairs[i:i + 1]), 1, ctypes.byref(pl)) == 0, ctx.error()
            plans.append(pl)
            offs.append(tot)
            tot += max(int(lib.gdp_plan_total_recs(pl)), 1)
        d_recs = torch.empty(tot * gdp.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        pb, ab, rb, cb = d_pairs.data_ptr(), d_arena.data_ptr(), d_res.data_ptr(), d_recs.data_ptr()

        def one_by_one():
            for j, i in enumerate(sample):
                lib.gdp_plan_execute(ctx.h, plans[j], ctypes.c_void_p(pb + int(i) * gdp.PAIR_DTYPE.itemsize),
                                     ctypes.c_void_p(ab), ctypes.c_void_p(rb + int(i) * gdp.RESULT_DTYPE.itemsize),
                                     ctypes.c_void_p(cb + offs[j] * gdp.REC_DTYPE.itemsize))

        one_by_one()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        one_by_one()
        b.record(stream)
        b.synchronize()
        pair_ms = a.elapsed_time(b)
        one = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
        for pl in plans:
            lib.gdp_plan_destroy(pl)
        same = all(np.array_equal(one[k][sample], res0[k][sample])
                   for k in ("status", "score", "precision", "tb_score", "nmatches", "nmismatches", "nopens",
                             "nindels", "nrecs"))
        pcells = float(gdp.band_cells(pairs[sample]).sum())
        per = pcells / (pair_ms * 1e-3) / 1e9
        out["per_pair"] = {"gcups": round(per, 3), "pairs": int(sample.size),
                           "alignments_per_s": round(sample.size / (pair_ms * 1e-3), 1),
                           "sample": f"the first {sample.size} pairs of chunk 0, one plan (its own launches) "
                                     f"per pair, back to back on one stream",
                           "results_identical_to_batch": bool(same)}
        out["batched_vs_per_pair"] = round(out["device"]["gcups"] / per, 2)
        routing = {k: ctx.get_param(k) for k in ("warp_min_x", "warp_max_sweep", "group_slack", "tb_warp",
                                                  "check_groups", "check_min_x")}
        conc = per_pair_concurrent(lib, pairs, arena, blocks, genome.size, sample, res0, routing)
        out["per_pair_concurrent"] = conc
        out["batched_vs_per_pair_concurrent"] = round(out["device"]["gcups"] / conc["gcups"], 2)
    if cpu_seconds > 0:
        out["cpu_baseline"] = cpu_leg(pairs, arena, blocks, genome.size, cpu_seconds, res=res0, recs=recs0,
                                      max_pairs=cpu_max_pairs)
    return out


def run_reference_arm(args):
    """The reference's own CPU code (oracle/_ref, compiled from its sources)
    on the host cores, over a prefix of the same seeded pairs the device
    arm aligns.  This process loads no CUDA library: the pairs come from the
    standalone generator libgdpwl.so and the code timed from oracle/."""
    # host cores only: rank 0 runs the sample, the other ranks exit at once
    # (no process group, so nothing waits on rank 0's minutes of CPU work)
    if int(os.environ.get("RANK", "0")) != 0:
        return
    wl = gdp.load_workload()
    name = args.workload
    npairs = args.npairs or WORKLOADS[name][1]
    genome, blocks, pairs, arena = make_workload(wl, name, npairs, args.seed)
    import oracle
    kind = "reference" if oracle.reference_available() else "port"
    ref = oracle.reference() if kind == "reference" else oracle.restatement()
    ref.init(0)
    ref.set_genome(blocks, None, genome.size)
    rest = oracle.restatement()
    rest.init(0)
    rest.set_genome(blocks, None, genome.size)
    threads = os.cpu_count() or 1
    per_step = args.ref_seconds / max(args.steps + 0.25 * args.warmup, 1)
    n = min(pairs.size, 512)
    while True:
        sample = pairs[:n]
        kept = rest.kept_precision(sample, arena, threads)
        secs, _ = ref.bench(sample, arena, threads, kept)
        if n >= pairs.size or secs >= per_step * 0.7:
            break
        n = min(pairs.size, int(n * min(16.0, max(1.3, per_step / max(secs, 1e-4)))))
    cells = int(gdp.band_cells(sample).sum())
    for _ in range(args.warmup):
        m = max(1, n // 4)
        ref.bench(sample[:m], arena, threads, kept[:m])
    times = []
    for _ in range(args.steps):
        secs, _ = ref.bench(sample, arena, threads, kept)
        times.append(secs)
    t = sum(times)
    value = cells * args.steps / t / 1e9
    line = {"metric": "GCUPS (in-band cells, fill + traceback), batched", "value": round(value, 4),
            "unit": "GCUPS", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16/int8",
            "data": "synthetic", "config": {"workload": name, "pairs_per_step": int(sample.size),
                                            "pairs_of_workload": int(pairs.size),
                                            "description": WORKLOADS[name][2]},
            "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": f"the first {sample.size} of the {pairs.size} pairs of '{name}' "
                                       f"(seed {args.seed}, the device arm's pairs) per step, fill + traceback "
                                       f"at the kept precision, on {threads} threads"},
            "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "alignments_per_s": round(sample.size * args.steps / t, 1)}
    if kind == "reference" and os.path.exists(oracle.REF_LIB_NOFLUSH):
        nf = oracle.reference(noflush=True)
        nf.init(0)
        nf.set_genome(blocks, None, genome.size)
        s2, _ = nf.bench(sample, arena, threads, kept)
        line["strong_cpu"] = {"value": round(cells / s2 / 1e9, 4), "unit": "GCUPS", "cores": threads,
                              "build": "the reference with the per-column _mm_clflush compiled out, same sample"}
    print(json.dumps(line), flush=True)


def kernel_cells(pairs, kernel, ctx):
    """In-band cells of the pairs a fill kernel group fills in one step:
    the kernel's variant; its pass (16-bit kinds fill the 16-bit pairs and
    the 16-bit pass of every rerun pair); pairs with fewer lanes (query
    rows; lower: genome columns) than warp_min_x go one thread per pair
    (fill_thread), the others to lane groups or CTAs."""
    if "," not in kernel:
        return int(gdp.band_cells(pairs).sum())
    variant = {"full": gdp.FULL, "upper": gdp.UPPER, "lower": gdp.LOWER}[kernel.split(",")[1]]
    rerun = ((pairs["precision"] == 8) & ((pairs["flags"] & gdp.FLAG_RERUN16) != 0))
    if "W16" in kernel:
        sel = (pairs["precision"] == 16) | rerun
    elif "8bit-check" in kernel:
        sel = rerun   # at most: the pass runs only where the 16-bit pass left it open
    else:
        sel = (pairs["precision"] == 8) & ~rerun
    lanes = np.where(pairs["variant"] == gdp.LOWER, pairs["glength"], pairs["rlength"])
    thread = lanes < ctx.get_param("warp_min_x")
    sel &= (pairs["variant"] == variant) & (thread if kernel.startswith(("fill_thread", "fill_packed")) else ~thread)
    return int(gdp.band_cells(pairs[sel]).sum())


def run_gdp(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    lib = gdp.load()
    name = args.workload
    kind = WORKLOADS[name][0]
    npairs = args.npairs or WORKLOADS[name][1]
    genome, blocks, pairs, arena = make_workload(lib, name, npairs, args.seed + 1000 * rank)
    cells = int(gdp.band_cells(pairs).sum())
    ctx = gdp.Context(lib, device=local)
    ctx.set_genome(blocks, None, genome.size)

    # routing parameters from the autotuner, on a separate draw of the
    # workload of the batch's own size (which routing wins depends on how
    # many pairs each kind holds)
    tuned = None
    if not args.no_autotune:
        tp, ta = gdp.make_pairs(lib, kind, args.seed + 77 + 1000 * rank, genome, min(args.tune_pairs or npairs, npairs))
        params, best = ctx.autotune(tp, ta)
        tuned = {"sample_pairs": int(tp.size), "params": params, "sample_ms": round(best, 3)}
        del tp, ta

    # resident inputs and outputs; the plan runs as a CUDA graph
    plan = ctypes.c_void_p()
    rc = lib.gdp_plan_create(ctx.h, gdp._ptr(pairs), pairs.size, ctypes.byref(plan))
    assert rc == 0, ctx.error()
    lib.gdp_plan_use_graph(plan, 1)
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

    for _ in range(max(args.warmup, 2)):
        step()
    lib.gdp_sync(ctx.h)
    res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
    bad = int((res["status"] != 0).sum())

    sampler = ClockSampler(local)
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
    ms_max = max_over_ranks(world, ms)
    total_cells = sum_over_ranks(world, float(cells))
    total_pairs = sum_over_ranks(world, float(pairs.size))
    value = total_cells * args.steps / (ms_max * 1e-3) / 1e9

    # per-kernel device times: the same K steps once more with CUDA events
    # around every launch (the profiled launches run without the graph)
    ctx.profile(True)
    ctx.profile_reset()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(args.steps):
        step()
    p1.record(stream)
    p1.synchronize()
    prof_ms = p0.elapsed_time(p1)
    prof = ctx.profile_read()
    ctx.profile(False)
    # the dominant kernel: one fill body, instantiated once per tie rule
    # (jump late / early); its two instantiations fill disjoint halves of
    # the batch and are counted together
    groups = {}
    for k, (kms, kn) in prof.items():
        g = k.replace(",early,", ",*,").replace(",late,", ",*,")
        tot, n_launch, members = groups.get(g, (0.0, 0, []))
        groups[g] = (tot + kms, n_launch + kn, members + [k])
    # the dominant fill group (the roofline counts fill lane-ops; a profiler
    # that serialises launches can make the traceback look larger)
    fills = {g: v for g, v in groups.items() if g.startswith("fill_")} or groups
    top_name, (top_ms, top_n, top_members) = max(fills.items(), key=lambda kv: kv[1][0])
    avg_launch_ms = top_ms / args.steps          # the group's device time per step
    int_peak = ctx.int_peak()
    top_cells = kernel_cells(pairs, top_name, ctx)
    achieved_ops = top_cells * OPS_PER_CELL / (avg_launch_ms * 1e-3)
    dir_bytes = int(lib.gdp_plan_dir_bytes(plan))

    # end to end through the host-buffer C ABI call, inputs and outputs in pinned host memory
    e2e_steps = max(1, args.e2e_steps)

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
    # what the call copied device to host: the results and the records as
    # runs (the host rebuilds the 12-byte records from them)
    d2h = ctx.get_param("last_d2h_bytes")
    records_bytes = int(used.value) * gdp.REC_DTYPE.itemsize
    e2e_bad = int((results["status"] != 0).sum())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_leg(pairs, arena, blocks, genome.size, args.cpu_seconds, res=results,
                      recs=recs[:int(used.value)])

    lib.gdp_plan_destroy(plan)
    del d_pairs, d_arena, d_res, d_recs
    torch.cuda.empty_cache()
    extra = {}
    if rank == 0 and world == 1 and not args.no_configs:
        cfg_genome = (genome, blocks)
        extra["config1_fixed"] = measure_config(lib, ctx, "config1", "fixed", 10_000, args.seed + 11, 10_000,
                                                args.cpu_seconds / 3, cfg_genome, per_pair=500)
        extra["config3_cdna"] = measure_config(lib, ctx, "config3", "cdna", 100_000, args.seed + 13, 100_000,
                                               args.cpu_seconds, cfg_genome)
        extra["config4_mix"] = measure_config(lib, ctx, "config4", "mix", args.mix_pairs, args.seed + 14,
                                              100_000, args.cpu_seconds, cfg_genome, tune_pairs=100_000,
                                              per_pair=1000)
    if rank == 0 and world == 1 and not args.no_per_pair:
        extra["endpoint_search"] = endpoint_search(lib, ctx, args.seed + 9)
        extra["single_gap"] = single_gap_batch(lib, ctx, args.seed + 10)
        extra["end_gap"] = end_gap_batch(lib, ctx, args.seed + 11)
        extra["cdna_gap"] = cdna_gap_batch(lib, ctx, args.seed + 12)
    if rank == 0 and world == 1 and not args.no_serving:
        extra["serving"] = serving_sweep(lib, local, args.seed + 8,
                                         [1e3, 1e4, 5e4, 1e5, 2e5, 3e5, 5e5, 1e6])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm = None
    if os.path.exists(peaks_path):
        hbm = json.load(open(peaks_path)).get("hbm_gbs")
    # DRAM bytes of the dominant kernel per launch: one ncu capture of the same
    # kernel on 300,000 pairs of this workload (its first launch, the 150,000
    # jump-early pairs: dram__bytes_read.sum + dram__bytes_write.sum =
    # 359.54 + 829.68 MB over 902,385,535 in-band cells), scaled to this
    # step's launches by their in-band cells; the kernel's bytes grow with the
    # cells (directions and carries per swept cell)
    traffic, traffic_src = None, None
    if name == "short" and top_name.startswith("fill_packed<W16,full"):
        traffic = int(round((359.537920e6 + 829.679616e6) / 902385535 * top_cells))
        traffic_src = ("ncu capture of this kernel on 300,000 pairs (1,189.2 MB for 902,385,535 in-band cells), "
                       "scaled by in-band cells to one step's launches")
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
                       "parallelism": f"pairs sharded, {world} independent rank(s)",
                       "graph": True, "autotune": tuned},
            "alignments_per_s": round(total_pairs * args.steps / (ms_max * 1e-3), 1),
            "e2e": {"value": round(e2e_value, 3), "unit": "GCUPS", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "records_rebuilt_bytes": records_bytes,
                    "record_transport": "runs" if ctx.get_param("record_runs") else "records",
                    "ms_per_step": round(e2e_ms, 3), "steps": e2e_steps,
                    "host_buffers": "pinned", "bad_status_pairs": e2e_bad},
            "roofline": {"bound": "int", "kernel": top_name, "instantiations": top_members,
                         "cells_per_step": int(top_cells),
                         "achieved": round(achieved_ops / 1e12, 3), "peak": round(int_peak / 1e12, 3),
                         "unit": "Tops/s (int32 lane-ops)", "frac": round(achieved_ops / int_peak, 4),
                         "peak_source": "measured int32 issue probe (gdp_measure_int_peak)",
                         # the packed fill computes two 16-bit lanes per 32-bit
                         # instruction, so its lane-op ceiling is twice the
                         # int32 rate; the fraction against that ceiling
                         "frac_of_packed_16x2_peak": (round(achieved_ops / (2 * int_peak), 4)
                                                      if top_name.startswith("fill_packed") else None),
                         "ops_per_cell": OPS_PER_CELL, "ms_per_step": round(avg_launch_ms, 3),
                         "kernel_times": "a profiled pass of the same K steps right after the timed region "
                                         "(CUDA events around every launch, on the launching stream)",
                         "traffic": traffic,
                         "traffic_source": traffic_src,
                         "dir_write_gbs": round(dir_bytes / (avg_launch_ms * 1e-3) / 1e9, 1),
                         "hbm_peak_gbs": hbm},
            "kernels": {k: {"ms_total": round(v[0], 3), "launches": v[1]} for k, v in prof.items()},
            "profiled_ms_per_step": round(prof_ms / args.steps, 3),
            "gpu_launches": int(launches),
            "clocks": clocks,
            "bad_status_pairs": bad,
            "cpu_baseline": cpu,
        }
        if cpu is not None and "parity" in cpu:
            line["parity"] = cpu["parity"]
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
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=90.0,
                    help="reference arm: total CPU seconds of the timed steps")
    ap.add_argument("--tune-pairs", type=int, default=0, help="autotuner sample (0: the batch's size)")
    ap.add_argument("--mix-pairs", type=int, default=2_000_000)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--no-per-pair", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gdp(args)


if __name__ == "__main__":
    main()
