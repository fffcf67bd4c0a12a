"""ctypes binding of libgdp.so for tests and benchmarks.

The library itself is C/CUDA (include/gdp.h); this module only mirrors its
structs as numpy dtypes and loads the shared object.  It never computes an
alignment: every score, direction and traceback comes from the CUDA kernels
inside libgdp.so, and loading fails loudly when the library is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GDP_LIB") or os.path.join(HERE, "lib", "libgdp.so")

FULL, UPPER, LOWER = 0, 1, 2
FLAG_JUMP_LATE, FLAG_REVP, FLAG_TRACEBACK, FLAG_RERUN16, FLAG_GWINDOW = 1, 2, 4, 8, 16
FLAG_ENDPOINT, FLAG_ENDPOINT_QEND = 32, 64
HIGHQ, MEDQ, LOWQ, ENDQ = 0, 1, 2, 3
STATUS = {0: "GDP_OK", 1: "GDP_ERR_LEN", 2: "GDP_ERR_BAND", 3: "GDP_ERR_PARAM",
          4: "GDP_ERR_BUDGET", 5: "GDP_ERR_TIMEOUT", 6: "GDP_ERR_CUDA",
          7: "GDP_ERR_RECS", 8: "GDP_ERR_NOGENOME"}

# struct gdp_pair (include/gdp.h), 88 bytes
PAIR_DTYPE = np.dtype([
    ("rseq", "<i8"), ("rseq_uc", "<i8"), ("gseq", "<i8"), ("gseq_alt", "<i8"),
    ("rlength", "<i4"), ("glength", "<i4"), ("lband", "<i4"), ("uband", "<i4"),
    ("variant", "i1"), ("precision", "i1"), ("mismatchtype", "i1"), ("flags", "i1"),
    ("open", "<i2"), ("extend", "<i2"),
    ("tb_r", "<i4"), ("tb_c", "<i4"),
    ("queryoffset", "<i4"), ("genomeoffset", "<i4"),
    ("chroffset", "<u4"), ("chrhigh", "<u4"),
    ("watsonp", "i1"), ("genestrand", "i1"), ("xflags", "<i2"),
    ("dynprogindex", "<i4"),
])
assert PAIR_DTYPE.itemsize == 88

# struct gdp_rec, 12 bytes
REC_DTYPE = np.dtype([
    ("querypos", "<i4"), ("genomepos", "<i4"),
    ("cdna", "S1"), ("comp", "S1"), ("genome", "S1"), ("genomealt", "S1"),
])
assert REC_DTYPE.itemsize == 12

# struct gdp_result, 64 bytes
RESULT_DTYPE = np.dtype([
    ("status", "<i4"), ("score", "<i4"), ("precision", "<i4"), ("rerun", "<i4"),
    ("tb_score", "<i4"), ("nmatches", "<i4"), ("nmismatches", "<i4"),
    ("nopens", "<i4"), ("nindels", "<i4"), ("nrecs", "<i4"),
    ("rec_offset", "<i8"),
    ("end_score", "<i4"), ("end_r", "<i4"), ("end_c", "<i4"), ("end_found", "<i4"),
])
assert RESULT_DTYPE.itemsize == 64

XFLAG_SEGMENT = 1

# struct gdp_single_gap, 72 bytes: the arguments of Dynprog_single_gap
SINGLE_GAP_DTYPE = np.dtype([
    ("rseq", "<i8"), ("rseq_uc", "<i8"),
    ("rlength", "<i4"), ("glength", "<i4"), ("roffset", "<i4"), ("goffset", "<i4"),
    ("chroffset", "<u4"), ("chrhigh", "<u4"),
    ("watsonp", "i1"), ("genestrand", "i1"), ("jump_late_p", "i1"), ("widebandp", "i1"),
    ("extraband_single", "<i4"), ("defect_rate", "<f8"),
    ("max_rlength", "<i4"), ("max_glength", "<i4"), ("dynprogindex", "<i4"), ("pad", "<i4"),
])
assert SINGLE_GAP_DTYPE.itemsize == 72
SINGLE_NULL, SINGLE_SIMPLE, SINGLE_DP = 0, 1, 2
XFLAG_SEGMENT_REV = 2

# struct gdp_end_gap, 72 bytes: the arguments of Dynprog_end5_gap / _end3_gap
END_GAP_DTYPE = np.dtype([
    ("rseq", "<i8"), ("rseq_uc", "<i8"),
    ("rlength", "<i4"), ("glength", "<i4"), ("roffset", "<i4"), ("goffset", "<i4"),
    ("chroffset", "<u4"), ("chrhigh", "<u4"),
    ("end", "i1"), ("endalign", "i1"), ("watsonp", "i1"), ("genestrand", "i1"), ("jump_late_p", "i1"),
    ("require_pos_score_p", "i1"), ("pad", "<i2"),
    ("extraband_end", "<i4"), ("max_rlength", "<i4"), ("max_glength", "<i4"), ("dynprogindex", "<i4"),
    ("defect_rate", "<f8"),
])
assert END_GAP_DTYPE.itemsize == 72
QUERYEND_GAP, QUERYEND_INDELS, QUERYEND_NOGAPS, BEST_LOCAL = 0, 1, 2, 3

# struct gdp_cdna_gap, 80 bytes: the arguments of Dynprog_cdna_gap
CDNA_GAP_DTYPE = np.dtype([
    ("rseq", "<i8"), ("rseq_uc", "<i8"),
    ("rlengthL", "<i4"), ("rlengthR", "<i4"), ("glength", "<i4"),
    ("roffsetL", "<i4"), ("rev_roffsetR", "<i4"), ("goffset", "<i4"),
    ("chroffset", "<u4"), ("chrhigh", "<u4"),
    ("watsonp", "i1"), ("genestrand", "i1"), ("jump_late_p", "i1"), ("pad8", "i1"),
    ("extraband_paired", "<i4"), ("max_rlength", "<i4"), ("max_glength", "<i4"), ("dynprogindex", "<i4"),
    ("pad32", "<i4"), ("defect_rate", "<f8"),
])
assert CDNA_GAP_DTYPE.itemsize == 80

WL_FIXED, WL_SHORT, WL_CDNA, WL_MIX, WL_LONG = 1, 2, 3, 4, 5


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def load(path=LIB_PATH):
    """Loads libgdp.so and declares its entry points."""
    if not os.path.exists(path):
        raise RuntimeError(f"libgdp.so not built at {path}: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    lib.gdp_version.restype = ctypes.c_char_p
    lib.gdp_ctx_create.argtypes = [ctypes.POINTER(vp), i32, i32, i64]
    lib.gdp_ctx_destroy.argtypes = [vp]
    lib.gdp_set_genome.argtypes = [vp, vp, vp, ctypes.c_uint64]
    lib.gdp_align_batch.argtypes = [vp, vp, i64, vp, i64, vp, vp, i64, ctypes.POINTER(i64)]
    lib.gdp_align_batch_multi.argtypes = [ctypes.POINTER(vp), i32, vp, i64, vp, i64, vp, vp, i64,
                                          ctypes.POINTER(i64)]
    lib.gdp_plan_create.argtypes = [vp, vp, i64, ctypes.POINTER(vp)]
    lib.gdp_plan_execute.argtypes = [vp, vp, vp, vp, vp, vp]
    lib.gdp_plan_total_recs.argtypes = [vp]
    lib.gdp_plan_total_recs.restype = i64
    lib.gdp_plan_rec_offset.argtypes = [vp, i64]
    lib.gdp_plan_rec_offset.restype = i64
    lib.gdp_plan_dir_bytes.argtypes = [vp]
    lib.gdp_plan_dir_bytes.restype = i64
    lib.gdp_plan_destroy.argtypes = [vp]
    lib.gdp_plan_use_graph.argtypes = [vp, i32]
    lib.gdp_ctx_set_param.argtypes = [vp, ctypes.c_char_p, i64]
    lib.gdp_ctx_get_param.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i64)]
    lib.gdp_autotune.argtypes = [vp, vp, i64, vp, i64, ctypes.POINTER(ctypes.c_double)]
    lib.gdp_sync.argtypes = [vp]
    lib.gdp_debug_tables.argtypes = [i32, vp, vp, vp]
    lib.gdp_ctx_stream.argtypes = [vp]
    lib.gdp_ctx_stream.restype = vp
    lib.gdp_profile_enable.argtypes = [vp, i32]
    lib.gdp_profile_read.argtypes = [vp, i32, ctypes.c_char_p, i32, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(i64)]
    lib.gdp_profile_reset.argtypes = [vp]
    lib.gdp_measure_int_peak.argtypes = [vp]
    lib.gdp_measure_int_peak.restype = ctypes.c_double
    lib.gdp_fill16_noalloc.argtypes = [i32, i32, vp, i64, vp, i64, vp, i64, vp, vp]
    lib.gdp_fill_dump.argtypes = [vp, vp, i64, vp, i64, vp, vp, vp, vp, vp, vp]
    lib.gdp_launch_count.argtypes = [vp]
    lib.gdp_launch_count.restype = i64
    lib.gdp_last_error.argtypes = [vp]
    lib.gdp_last_error.restype = ctypes.c_char_p
    lib.gdp_workload_genome.argtypes = [ctypes.c_uint64, vp, i64]
    lib.gdp_workload_genomecomp.argtypes = [vp, i64, vp]
    lib.gdp_workload_pairs.argtypes = [i32, ctypes.c_uint64, vp, i64, i64, vp, vp, i64,
                                       ctypes.POINTER(i64)]
    lib.gdp_workload_pairs.restype = i64
    lib.gdp_pair_cells.argtypes = [vp]
    lib.gdp_pair_cells.restype = i64
    lib.gdp_workload_resident_pairs.argtypes = lib.gdp_workload_pairs.argtypes
    lib.gdp_workload_resident_pairs.restype = i64
    dp = ctypes.POINTER(ctypes.c_double)
    lib.gdp_server_create.argtypes = [i32, i32, i32, i64, i64, vp, vp, ctypes.c_uint64, ctypes.POINTER(vp)]
    lib.gdp_server_submit.argtypes = [vp, vp, i64, vp, i64]
    lib.gdp_server_submit.restype = i64
    lib.gdp_server_wait.argtypes = [vp, i64, vp, vp, i64, ctypes.POINTER(i64), dp]
    lib.gdp_server_drive.argtypes = [vp, vp, i64, vp, i64, ctypes.c_double, ctypes.c_uint64, vp, vp, dp]
    lib.gdp_server_stats.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64),
                                     ctypes.POINTER(i64), dp]
    lib.gdp_server_destroy.argtypes = [vp]
    lib.gdp_server_set_classes.argtypes = [vp, i64, i32]
    lib.gdp_server_class_of.argtypes = [vp, vp, i64]
    lib.gdp_server_class_stats.argtypes = [vp, vp, vp]
    ip = ctypes.POINTER(i32)
    lib.gdp_endpoint_combine.argtypes = [vp, vp, i32, i32, i32, i32, ip, ip, ip]
    lib.gdp_single_setup.argtypes = [vp, i32, i32, i32, i32]
    lib.gdp_single_gap_batch.argtypes = [vp, vp, i64, vp, i64, vp, vp, vp, i64, ctypes.POINTER(i64)]
    lib.gdp_runs_encode.argtypes = [vp, vp, vp, i32, vp]
    lib.gdp_runs_encode.restype = i64
    lib.gdp_runs_decode.argtypes = [vp, vp, vp, i64, vp, i32]
    lib.gdp_cdna_gap_batch.argtypes = [vp, vp, i64, vp, i64, vp, vp, i64, ctypes.POINTER(i64)]
    lib.gdp_end_setup.argtypes = [vp, i32, i32, i32]
    lib.gdp_end_gap_batch.argtypes = [vp, vp, i64, vp, i64, vp, vp, i64, ctypes.POINTER(i64)]
    lib.gdp_gap_queue_create.argtypes = [i32, i32, i64, i64, vp, vp, ctypes.c_uint64, ctypes.POINTER(vp)]
    lib.gdp_gap_queue_setup.argtypes = [vp, i32, i32, i32, i32]
    lib.gdp_gap_queue_align.argtypes = [vp, vp, vp, vp, vp, vp, vp, i64, ctypes.POINTER(i64)]
    lib.gdp_gap_queue_stats.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64)]
    lib.gdp_gap_queue_destroy.argtypes = [vp]
    lib.gdp_gap_queue_destroy.restype = None
    return lib


WORKLOAD_LIB_PATH = os.path.join(HERE, "lib", "libgdpwl.so")


def load_workload(path=WORKLOAD_LIB_PATH):
    """Loads libgdpwl.so, the seeded workload generator alone (no CUDA):
    make_genome / make_pairs / make_resident_pairs accept it in place of
    libgdp.so, so a process that only runs CPU code generates the same
    pairs without loading the CUDA library."""
    if not os.path.exists(path):
        raise RuntimeError(f"libgdpwl.so not built at {path}: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    lib.gdp_workload_genome.argtypes = [ctypes.c_uint64, vp, i64]
    lib.gdp_workload_genomecomp.argtypes = [vp, i64, vp]
    lib.gdp_workload_pairs.argtypes = [i32, ctypes.c_uint64, vp, i64, i64, vp, vp, i64, ctypes.POINTER(i64)]
    lib.gdp_workload_pairs.restype = i64
    lib.gdp_workload_resident_pairs.argtypes = lib.gdp_workload_pairs.argtypes
    lib.gdp_workload_resident_pairs.restype = i64
    lib.gdp_pair_cells.argtypes = [vp]
    lib.gdp_pair_cells.restype = i64
    return lib


def record_digests(recs, offsets, counts):
    """Per pair, a 32-bit digest of its Pair records in push order (the
    same digest oracle/ computes for the reference's records): the sum over
    records k of (w0 * 0x9E3779B1 + w1 * 0x85EBCA77 + w2 * 0xC2B2AE3D + 1) *
    (2k + 1) mod 2^32, w0..w2 the record's three little-endian words."""
    counts = np.asarray(counts, dtype=np.int64)
    offsets = np.asarray(offsets, dtype=np.int64)
    out = np.zeros(counts.size, dtype=np.uint32)
    tot = int(counts.sum())
    if tot == 0:
        return out
    seg = np.repeat(np.arange(counts.size), counts)
    first = np.repeat(np.cumsum(counts) - counts, counts)
    k = np.arange(tot, dtype=np.int64) - first
    idx = np.repeat(offsets, counts) + k
    w = np.ascontiguousarray(recs).view(np.uint32).reshape(-1, 3)[idx].astype(np.uint64)
    m = np.uint64(0xFFFFFFFF)
    h = (w[:, 0] * np.uint64(0x9E3779B1) + w[:, 1] * np.uint64(0x85EBCA77) +
         w[:, 2] * np.uint64(0xC2B2AE3D) + np.uint64(1)) & m
    h = (h * (2 * k.astype(np.uint64) + np.uint64(1))) & m
    np.add.at(out, seg, h.astype(np.uint32))
    return out


def endpoint_combine(lib, upper, lower, jump_late, qend, precision, rlength):
    """The reference's (finalscore, bestr, bestc) of one end gap from the
    results of its upper and lower halves (gdp_endpoint_combine)."""
    u = np.ascontiguousarray(upper, dtype=RESULT_DTYPE).reshape(1)
    lo = np.ascontiguousarray(lower, dtype=RESULT_DTYPE).reshape(1)
    fs, br, bc = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    rc = lib.gdp_endpoint_combine(_ptr(u), _ptr(lo), int(jump_late), int(qend), int(precision), int(rlength),
                                  ctypes.byref(fs), ctypes.byref(br), ctypes.byref(bc))
    if rc != 0:
        raise RuntimeError(f"gdp_endpoint_combine: {STATUS.get(rc, rc)}")
    return fs.value, br.value, bc.value


def runs_encode(lib, pair, arena, recs):
    """The record-run stream of one pair's records (gdp_runs_encode)."""
    p = np.ascontiguousarray(pair, dtype=PAIR_DTYPE).reshape(1)
    r = np.ascontiguousarray(recs, dtype=REC_DTYPE)
    n = lib.gdp_runs_encode(_ptr(p), _ptr(arena), _ptr(r), r.size, None)
    if n < 0:
        raise RuntimeError("gdp_runs_encode: bad arguments")
    out = np.zeros(max(n, 1), np.uint8)
    lib.gdp_runs_encode(_ptr(p), _ptr(arena), _ptr(r), r.size, _ptr(out))
    return out[:n]


def runs_decode(lib, pair, arena, stream, nrecs):
    """The records a run stream rebuilds (gdp_runs_decode), or None."""
    p = np.ascontiguousarray(pair, dtype=PAIR_DTYPE).reshape(1)
    out = np.zeros(max(nrecs, 1), dtype=REC_DTYPE)
    st = np.ascontiguousarray(stream, dtype=np.uint8)
    rc = lib.gdp_runs_decode(_ptr(p), _ptr(arena), _ptr(st), st.size, _ptr(out), nrecs)
    return out[:nrecs] if rc == 0 else None


def tables(lib, mode=0):
    """The substitution / consistency tables libgdp builds (host only)."""
    pd = np.zeros((4, 128, 128), np.int16)
    cons = np.zeros((3, 128, 128), np.uint8)
    nt = np.zeros(128, np.int8)
    rc = lib.gdp_debug_tables(mode, _ptr(pd), _ptr(cons), _ptr(nt))
    if rc != 0:
        raise RuntimeError(f"gdp_debug_tables: {STATUS.get(rc, rc)}")
    return pd, cons, nt


def make_genome(lib, seed, length):
    """Returns (char genome as uint8 array, genomecomp blocks as uint32 array)."""
    g = np.zeros(length, dtype=np.uint8)
    lib.gdp_workload_genome(seed, _ptr(g), length)
    nwords = (length + 31) // 32
    blocks = np.zeros(3 * nwords, dtype=np.uint32)
    lib.gdp_workload_genomecomp(_ptr(g), length, _ptr(blocks))
    return g, blocks


def make_pairs(lib, kind, seed, genome, npairs, arena_bytes=None):
    """Generates a seeded synthetic batch; returns (pairs, arena)."""
    if arena_bytes is None:
        per = {WL_FIXED: 600, WL_SHORT: 1200, WL_CDNA: 16000, WL_MIX: 12000, WL_LONG: 36000}[kind]
        arena_bytes = npairs * per + (1 << 16)
    pairs = np.zeros(npairs, dtype=PAIR_DTYPE)
    arena = np.zeros(arena_bytes, dtype=np.uint8)
    used = ctypes.c_int64(0)
    n = lib.gdp_workload_pairs(kind, seed, _ptr(genome), genome.size, npairs, _ptr(pairs),
                               _ptr(arena), arena_bytes, ctypes.byref(used))
    if n != npairs:
        raise RuntimeError(f"arena too small: generated {n} of {npairs} pairs")
    return pairs, arena[:max(used.value, 1)].copy()


def make_resident_pairs(lib, kind, seed, genome, npairs, arena_bytes=None):
    """Like make_pairs, but every genome window is a slice of `genome`
    flagged FLAG_GWINDOW (the device extracts it from the resident genome);
    the arena still holds the window bytes."""
    if arena_bytes is None:
        per = {WL_FIXED: 700, WL_SHORT: 1400, WL_CDNA: 16000, WL_MIX: 12000, WL_LONG: 36000}[kind]
        arena_bytes = npairs * per + (1 << 16)
    pairs = np.zeros(npairs, dtype=PAIR_DTYPE)
    arena = np.zeros(arena_bytes, dtype=np.uint8)
    used = ctypes.c_int64(0)
    n = lib.gdp_workload_resident_pairs(kind, seed, _ptr(genome), genome.size, npairs, _ptr(pairs),
                                        _ptr(arena), arena_bytes, ctypes.byref(used))
    if n != npairs:
        raise RuntimeError(f"arena too small: generated {n} of {npairs} pairs")
    return pairs, arena[:max(used.value, 1)].copy()


def pair_cells(lib, pairs):
    """In-band cells per pair over the reference's compare domain."""
    out = np.zeros(pairs.size, dtype=np.int64)
    base = pairs.ctypes.data
    for i in range(pairs.size):
        out[i] = lib.gdp_pair_cells(ctypes.c_void_p(base + i * PAIR_DTYPE.itemsize))
    return out


def shard_indices(pairs, world, rank):
    """Pair indices of `rank`'s shard when a batch is spread over `world`
    GPUs.  Pairs are independent, so a shard is any subset; to balance the
    work, pairs are ranked by in-band cells and dealt out in snake order
    (0, 1, .., world-1, world-1, .., 0, ...), which keeps the cell totals of
    the shards within one large pair of each other."""
    order = np.argsort(-band_cells(pairs), kind="stable")
    k = np.arange(order.size)
    turn = k % (2 * world)
    owner = np.where(turn < world, turn, 2 * world - 1 - turn)
    return np.sort(order[owner == rank])


def band_cells(pairs):
    """In-band cells per pair over the reference's compare domain (same as
    pair_cells), vectorised over the band's diagonals d = r - c."""
    r = pairs["rlength"].astype(np.int64)
    g = pairs["glength"].astype(np.int64)
    var = pairs["variant"]
    lb = np.where(var == UPPER, 0, pairs["lband"]).astype(np.int64)
    ub = np.where(var == LOWER, 0, pairs["uband"]).astype(np.int64)
    total = np.zeros(pairs.size, dtype=np.int64)
    if pairs.size == 0:
        return total
    for d in range(-int(ub.max()), int(lb.max()) + 1):
        on = (d >= -ub) & (d <= lb)
        cmin = np.maximum(1, 1 - d)
        cmax = np.minimum(g, r - d)
        total += np.where(on, np.maximum(0, cmax - cmin + 1), 0)
    return total


class Context:
    """One libgdp context (device, tables, resident genome)."""

    def __init__(self, lib, device=0, mode=0, budget=0):
        self.lib = lib
        h = ctypes.c_void_p()
        rc = lib.gdp_ctx_create(ctypes.byref(h), device, mode, budget)
        if rc != 0:
            raise RuntimeError(f"gdp_ctx_create failed: {STATUS.get(rc, rc)}")
        self.h = h

    def close(self):
        if self.h:
            self.lib.gdp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def error(self):
        return self.lib.gdp_last_error(self.h).decode()

    def launches(self):
        return int(self.lib.gdp_launch_count(self.h))

    def stream_handle(self):
        return int(self.lib.gdp_ctx_stream(self.h) or 0)

    def profile(self, on=True):
        self.lib.gdp_profile_enable(self.h, 1 if on else 0)

    def profile_reset(self):
        self.lib.gdp_profile_reset(self.h)

    def profile_read(self):
        """{kernel name: (total ms, launches)} since the last reset."""
        out = {}
        name = ctypes.create_string_buffer(64)
        for k in range(128):
            ms, n = ctypes.c_double(0), ctypes.c_int64(0)
            self.lib.gdp_profile_read(self.h, k, name, 64, ctypes.byref(ms), ctypes.byref(n))
            if n.value:
                out[name.value.decode()] = (ms.value, n.value)
        return out

    def set_param(self, name, value):
        rc = self.lib.gdp_ctx_set_param(self.h, name.encode(), int(value))
        if rc != 0:
            raise ValueError(f"gdp_ctx_set_param({name}, {value}): {STATUS.get(rc, rc)}")

    def get_param(self, name):
        v = ctypes.c_int64(0)
        rc = self.lib.gdp_ctx_get_param(self.h, name.encode(), ctypes.byref(v))
        if rc != 0:
            raise ValueError(f"gdp_ctx_get_param({name}): {STATUS.get(rc, rc)}")
        return v.value

    def autotune(self, pairs, arena):
        """Tunes the routing parameters on a sample batch; returns
        (parameters, best device ms of the sample)."""
        best = ctypes.c_double(0)
        rc = self.lib.gdp_autotune(self.h, _ptr(pairs), pairs.size, _ptr(arena), arena.size, ctypes.byref(best))
        if rc != 0:
            raise RuntimeError(f"gdp_autotune: {STATUS.get(rc, rc)} {self.error()}")
        names = ("warp_min_x", "warp_max_sweep", "group_slack", "tb_warp", "check_groups", "check_min_x")
        return {k: self.get_param(k) for k in names}, best.value

    def int_peak(self):
        return float(self.lib.gdp_measure_int_peak(self.h))

    def set_genome(self, blocks, altblocks=None, length=None):
        if length is None:
            length = blocks.size // 3 * 32
        rc = self.lib.gdp_set_genome(self.h, _ptr(blocks), _ptr(altblocks), length)
        if rc != 0:
            raise RuntimeError(f"gdp_set_genome: {STATUS.get(rc, rc)} {self.error()}")

    def align(self, pairs, arena, max_recs=None):
        n = pairs.size
        results = np.zeros(n, dtype=RESULT_DTYPE)
        if max_recs is None:
            max_recs = int((pairs["rlength"].astype(np.int64) + pairs["glength"] + 2).sum())
        recs = np.zeros(max(max_recs, 1), dtype=REC_DTYPE)
        used = ctypes.c_int64(0)
        rc = self.lib.gdp_align_batch(self.h, _ptr(pairs), n, _ptr(arena), arena.size,
                                      _ptr(results), _ptr(recs), max_recs, ctypes.byref(used))
        if rc != 0:
            raise RuntimeError(f"gdp_align_batch: {STATUS.get(rc, rc)} {self.error()}")
        return results, recs[:used.value]

    def single_setup(self, user_open=0, user_extend=0, user_dynprog_p=False, homopolymerp=False):
        return self.lib.gdp_single_setup(self.h, user_open, user_extend, int(user_dynprog_p), int(homopolymerp))

    def single_gaps(self, gaps, arena, max_recs=None):
        """Dynprog_single_gap over a batch: (results, path, records)."""
        n = gaps.size
        results = np.zeros(n, dtype=RESULT_DTYPE)
        path = np.zeros(n, dtype=np.int8)
        if max_recs is None:
            max_recs = int((np.maximum(gaps["rlength"], 0).astype(np.int64)
                            + np.maximum(gaps["glength"], 0) + 2).sum())
        recs = np.zeros(max(max_recs, 1), dtype=REC_DTYPE)
        used = ctypes.c_int64(0)
        rc = self.lib.gdp_single_gap_batch(self.h, _ptr(gaps), n, _ptr(arena), arena.size, _ptr(results),
                                           _ptr(path), _ptr(recs), max_recs, ctypes.byref(used))
        if rc != 0:
            raise RuntimeError(f"gdp_single_gap_batch: {STATUS.get(rc, rc)} {self.error()}")
        return results, path, recs[:used.value]

    def end_setup(self, user_open=0, user_extend=0, user_dynprog_p=False):
        return self.lib.gdp_end_setup(self.h, user_open, user_extend, int(user_dynprog_p))

    def end_gaps(self, gaps, arena, max_recs=None):
        """Dynprog_end5_gap / Dynprog_end3_gap over a batch: (results, records)."""
        n = gaps.size
        results = np.zeros(n, dtype=RESULT_DTYPE)
        if max_recs is None:
            max_recs = int((np.maximum(gaps["rlength"], 0).astype(np.int64)
                            + np.maximum(gaps["glength"], 0) + 2).sum())
        recs = np.zeros(max(max_recs, 1), dtype=REC_DTYPE)
        used = ctypes.c_int64(0)
        rc = self.lib.gdp_end_gap_batch(self.h, _ptr(gaps), n, _ptr(arena), arena.size, _ptr(results),
                                        _ptr(recs), max_recs, ctypes.byref(used))
        if rc != 0:
            raise RuntimeError(f"gdp_end_gap_batch: {STATUS.get(rc, rc)} {self.error()}")
        return results, recs[:used.value]

    def cdna_gaps(self, gaps, arena, max_recs=None):
        """Dynprog_cdna_gap over a batch: (results, records); results'
        end_found is the reference's incompletep."""
        n = gaps.size
        results = np.zeros(n, dtype=RESULT_DTYPE)
        if max_recs is None:
            max_recs = int((np.maximum(gaps["rlengthL"], 0).astype(np.int64) + np.maximum(gaps["rlengthR"], 0)
                            + 2 * np.maximum(gaps["glength"], 0) + 24).sum())
        recs = np.zeros(max(max_recs, 1), dtype=REC_DTYPE)
        used = ctypes.c_int64(0)
        rc = self.lib.gdp_cdna_gap_batch(self.h, _ptr(gaps), n, _ptr(arena), arena.size, _ptr(results),
                                         _ptr(recs), max_recs, ctypes.byref(used))
        if rc != 0:
            raise RuntimeError(f"gdp_cdna_gap_batch: {STATUS.get(rc, rc)} {self.error()}")
        return results, recs[:used.value]

    def fill_dump(self, pairs, arena, scores=True):
        """Dense in-band scores and directions of every pair.  With
        scores=False the fills run exactly as in production (no score
        dump), H comes back None and the directions are decoded from the
        production direction words."""
        n = pairs.size
        sizes = (pairs["glength"].astype(np.int64) + 1) * (pairs["rlength"].astype(np.int64) + 1)
        offs = np.zeros(n, dtype=np.int64)
        offs[1:] = np.cumsum(sizes)[:-1]
        total = int(sizes.sum())
        H = np.zeros(total, dtype=np.int16) if scores else None
        dN = np.zeros(total, dtype=np.int8)
        dE = np.zeros(total, dtype=np.int8)
        dF = np.zeros(total, dtype=np.int8)
        results = np.zeros(n, dtype=RESULT_DTYPE)
        rc = self.lib.gdp_fill_dump(self.h, _ptr(pairs), n, _ptr(arena), arena.size, _ptr(offs),
                                    _ptr(H), _ptr(dN), _ptr(dE), _ptr(dF), _ptr(results))
        if rc != 0:
            raise RuntimeError(f"gdp_fill_dump: {STATUS.get(rc, rc)} {self.error()}")
        return offs, H, dN, dE, dF, results


def align_multi(lib, contexts, pairs, arena, max_recs=None):
    """One batch over several contexts (gdp_align_batch_multi): (results,
    recs), pair i's records at results[i]["rec_offset"] in recs."""
    n = pairs.size
    results = np.zeros(n, dtype=RESULT_DTYPE)
    if max_recs is None:
        max_recs = int((pairs["rlength"].astype(np.int64) + pairs["glength"] + 2).sum())
    recs = np.zeros(max(max_recs, 1), dtype=REC_DTYPE)
    hs = (ctypes.c_void_p * len(contexts))(*[c.h.value if isinstance(c.h, ctypes.c_void_p) else c.h
                                             for c in contexts])
    used = ctypes.c_int64(0)
    rc = lib.gdp_align_batch_multi(hs, len(contexts), _ptr(pairs), n, _ptr(arena), arena.size, _ptr(results),
                                   _ptr(recs), max_recs, ctypes.byref(used))
    if rc != 0:
        raise RuntimeError(f"gdp_align_batch_multi: {STATUS.get(rc, rc)}")
    return results, recs[:used.value]


class Server:
    """The continuous-batching request loop (gdp_server_*)."""

    def __init__(self, lib, device=0, mode=0, workers=2, budget=0, max_batch=0, blocks=None, altblocks=None,
                 length=None):
        self.lib = lib
        if blocks is not None and length is None:
            length = blocks.size // 3 * 32
        h = ctypes.c_void_p()
        rc = lib.gdp_server_create(device, mode, workers, budget, max_batch, _ptr(blocks), _ptr(altblocks),
                                   length or 0, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"gdp_server_create failed: {STATUS.get(rc, rc)}")
        self.h = h
        self._keep = (blocks, altblocks)

    def close(self):
        if self.h:
            self.lib.gdp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, pairs, arena):
        rid = self.lib.gdp_server_submit(self.h, _ptr(pairs), pairs.size, _ptr(arena), arena.size)
        if rid < 0:
            raise RuntimeError(f"gdp_server_submit: {STATUS.get(-rid, rid)}")
        return rid, pairs.size, int((pairs["rlength"].astype(np.int64) + pairs["glength"] + 2).sum())

    def wait(self, ticket):
        rid, n, cap = ticket
        results = np.zeros(n, dtype=RESULT_DTYPE)
        recs = np.zeros(max(cap, 1), dtype=REC_DTYPE)
        nrecs, lat = ctypes.c_int64(0), ctypes.c_double(0)
        rc = self.lib.gdp_server_wait(self.h, rid, _ptr(results), _ptr(recs), cap, ctypes.byref(nrecs),
                                      ctypes.byref(lat))
        if rc not in (0, 4):     # GDP_ERR_BUDGET is a per-request outcome, in results["status"]
            raise RuntimeError(f"gdp_server_wait: {STATUS.get(rc, rc)}")
        return results, recs[:nrecs.value], lat.value

    def drive(self, pool, arena, nrequests, rate, seed=1, want_results=False):
        """Poisson load: returns (latencies ms, elapsed s, results or None)."""
        lat = np.zeros(nrequests, dtype=np.float64)
        res = np.zeros(nrequests, dtype=RESULT_DTYPE) if want_results else None
        el = ctypes.c_double(0)
        rc = self.lib.gdp_server_drive(self.h, _ptr(pool), pool.size, _ptr(arena), nrequests, rate, seed,
                                       _ptr(res), _ptr(lat), ctypes.byref(el))
        if rc != 0:
            raise RuntimeError(f"gdp_server_drive: {STATUS.get(rc, rc)}")
        return lat, el.value, res

    def stats(self):
        b, p, m, pk = (ctypes.c_int64(0) for _ in range(4))
        busy = ctypes.c_double(0)
        self.lib.gdp_server_stats(self.h, ctypes.byref(b), ctypes.byref(p), ctypes.byref(m), ctypes.byref(pk),
                                  ctypes.byref(busy))
        cb, cp = np.zeros(2, np.int64), np.zeros(2, np.int64)
        self.lib.gdp_server_class_stats(self.h, _ptr(cb), _ptr(cp))
        return {"batches": b.value, "pairs": p.value, "max_batch_pairs": m.value,
                "peak_reserved_bytes": pk.value, "busy_s": busy.value,
                "class_batches": cb.tolist(), "class_pairs": cp.tolist()}

    def set_classes(self, short_max_length=512, short_workers=1):
        return self.lib.gdp_server_set_classes(self.h, short_max_length, short_workers)

    def classes(self, pairs):
        """The size class (0 short, 1 long) of each pair as a one-pair request."""
        return np.array([self.lib.gdp_server_class_of(self.h, _ptr(pairs[i:i + 1]), 1) for i in range(pairs.size)],
                        dtype=np.int8)


class GapQueue:
    """gdp_gap_queue: Dynprog_single_gap calls from many threads, aligned together."""

    def __init__(self, lib, blocks, altblocks=None, length=None, device=0, mode=0, max_batch=0, max_wait_us=200):
        self.lib = lib
        self.h = ctypes.c_void_p()
        if length is None:
            length = blocks.size // 3 * 32
        self._keep = (blocks, altblocks)
        rc = lib.gdp_gap_queue_create(device, mode, max_batch, max_wait_us, _ptr(blocks), _ptr(altblocks), length,
                                      ctypes.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"gdp_gap_queue_create: {STATUS.get(rc, rc)}")

    def setup(self, user_open=0, user_extend=0, user_dynprog_p=False, homopolymerp=False):
        return self.lib.gdp_gap_queue_setup(self.h, user_open, user_extend, int(user_dynprog_p), int(homopolymerp))

    def align(self, gap, rsequence, rsequenceuc):
        """One gap (a SINGLE_GAP_DTYPE record; rseq offsets ignored) with its
        query strings (uint8 arrays); blocks until done."""
        g = np.array(gap, dtype=SINGLE_GAP_DTYPE).reshape(1)
        res = np.zeros(1, dtype=RESULT_DTYPE)
        path = np.zeros(1, dtype=np.int8)
        cap = max(int(g["rlength"][0]), 0) + max(int(g["glength"][0]), 0) + 2
        recs = np.zeros(cap, dtype=REC_DTYPE)
        n = ctypes.c_int64(0)
        rc = self.lib.gdp_gap_queue_align(self.h, _ptr(g), _ptr(rsequence), _ptr(rsequenceuc), _ptr(res),
                                          _ptr(path), _ptr(recs), cap, ctypes.byref(n))
        if rc != 0:
            raise RuntimeError(f"gdp_gap_queue_align: {STATUS.get(rc, rc)}")
        return res[0], int(path[0]), recs[:n.value]

    def stats(self):
        b, g, m = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        self.lib.gdp_gap_queue_stats(self.h, ctypes.byref(b), ctypes.byref(g), ctypes.byref(m))
        return {"batches": b.value, "gaps": g.value, "max_batch": m.value}

    def close(self):
        if self.h:
            self.lib.gdp_gap_queue_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
