"""Oracle loaders -- TEST INFRASTRUCTURE ONLY.

Two CPU oracles with one interface:
  * Reference: the reference's own AVX2 functions compiled from its sources
    into oracle/_ref/libgdpref.so (see oracle/Makefile).
  * Restatement: oracle/liboracle.so, this repository's plain-C restatement
    of the same algorithm (oracle/gdp_oracle.c), pinned against the first.

A third library with the same interface hosts the product instead of
checking it: oracle/_ref/libgmapenv.so is GMAP's own list / pairpool /
dynprog code with src/dynprog_simd.c removed, so its Dynprog_simd_* and
Dynprog_traceback_* calls land in the product's reference-signature entry
points (libgdp.so).  Tests compare it against the reference library.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
arm import this module, and only as the checker or the timed CPU baseline.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libgdpref.so")
REF_LIB_NOFLUSH = os.path.join(HERE, "_ref", "libgdpref_noflush.so")
GMAPENV_LIB = os.path.join(HERE, "_ref", "libgmapenv.so")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


# Genomes handed to a library, by library path.  Every CpuOracle of one path
# shares the library's single global genome pointer, so the arrays behind it
# must live as long as the last set_genome of any of those instances.
_GENOME_KEEP = {}


class CpuOracle:
    """Wraps libgdpref.so (prefix 'ref_') or liboracle.so (prefix 'orc_')."""

    def __init__(self, path, prefix, mode=ctypes.DEFAULT_MODE):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = ctypes.CDLL(path, mode=mode)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        self._init = getattr(self.lib, prefix + "init")
        self._init.argtypes = [i32]
        self._set_genome = getattr(self.lib, prefix + "set_genome")
        self._set_genome.argtypes = [vp, vp, ctypes.c_uint64]
        self._align = getattr(self.lib, prefix + "align")
        self._align.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, i32]
        self._align.restype = i32
        self._bench = getattr(self.lib, prefix + "bench")
        self._bench.argtypes = [vp, vp, i64, i32, ctypes.POINTER(i64), vp]
        self._bench.restype = ctypes.c_double
        self._outputs = getattr(self.lib, prefix + "outputs", None)
        if self._outputs is not None:
            self._outputs.argtypes = [vp, vp, i64, i32, vp, vp]
            self._outputs.restype = ctypes.c_double
        self._pd = getattr(self.lib, prefix + "pairdistance")
        self._pd.argtypes = [i32, i32, i32]
        self._cons = getattr(self.lib, prefix + "consistent")
        self._cons.argtypes = [i32, i32, i32]

    def init(self, mode=0):
        self._init(mode)

    def pairdistance(self, mt, c1, c2):
        return self._pd(mt, c1, c2)

    def consistent(self, gs, c1, c2):
        return self._cons(gs, c1, c2)

    def set_genome(self, blocks, altblocks=None, length=None):
        if length is None:
            length = blocks.size // 3 * 32
        _GENOME_KEEP[self.path] = (blocks, altblocks)
        self._set_genome(_ptr(blocks), _ptr(altblocks), length)

    def align(self, pair_arr, i, arena, want_matrix=True, max_recs=None):
        """Fills pair i (and traces back if its flags ask).  Returns a dict."""
        p = pair_arr[i:i + 1]
        rl, gl = int(p["rlength"][0]), int(p["glength"][0])
        n = (rl + 1) * (gl + 1)
        H = np.zeros(n, np.int16) if want_matrix else None
        dN = np.zeros(n, np.int8) if want_matrix else None
        dE = np.zeros(n, np.int8) if want_matrix else None
        dF = np.zeros(n, np.int8) if want_matrix else None
        final = np.zeros(1, np.int32)
        stats = np.zeros(6, np.int32)
        if max_recs is None:
            max_recs = rl + gl + 8
        recs = np.zeros(max_recs, dtype=_rec_dtype())
        nrec = self._align(_ptr(p), _ptr(arena), _ptr(H), _ptr(dN), _ptr(dE), _ptr(dF),
                           _ptr(final), _ptr(stats), _ptr(recs), max_recs)
        return {"score": int(final[0]), "H": H, "dN": dN, "dE": dE, "dF": dF,
                "stats": stats, "recs": recs[:min(nrec, max_recs)], "nrecs": nrec}

    def outputs(self, pairs, arena, nthreads, kept=None):
        """Every pair once on nthreads threads, as bench() runs them, with
        its outputs: an (n, 8) int32 array of the final score, traceback
        score, nmatches, nmismatches, nopens, nindels, record count and the
        records' 32-bit digest (gdp.record_digests computes the same digest
        of the device's records).  Returns (seconds, outputs)."""
        out = np.zeros((pairs.size, 8), dtype=np.int32)
        if kept is not None:
            kept = np.ascontiguousarray(kept, dtype=np.int8)
        secs = self._outputs(_ptr(pairs), _ptr(arena), pairs.size, nthreads, _ptr(kept), _ptr(out))
        return secs, out

    def bench(self, pairs, arena, nthreads, kept=None):
        """Wall seconds and a score checksum for every pair once on nthreads
        threads.  `kept` (int8 per pair, from kept_precision) says which
        precision an 8-bit pair flagged RERUN16 keeps; only that precision
        runs (the least work giving the contract's outputs).  Without it such
        pairs run in 16-bit."""
        cs = ctypes.c_int64(0)
        if kept is not None:
            kept = np.ascontiguousarray(kept, dtype=np.int8)
            assert kept.size == pairs.size
        secs = self._bench(_ptr(pairs), _ptr(arena), pairs.size, nthreads, ctypes.byref(cs), _ptr(kept))
        return secs, cs.value

    def kept_precision(self, pairs, arena, nthreads):
        """Per pair, the precision the rerun contract keeps (restatement only:
        it needs to know whether an 8-bit traceback reads unwritten cells)."""
        fn = self.lib.orc_kept_precision
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
        fn.restype = None
        kept = np.zeros(pairs.size, dtype=np.int8)
        fn(_ptr(pairs), _ptr(arena), pairs.size, nthreads, _ptr(kept))
        return kept


class ReferenceSingleGap:
    """The reference's own Dynprog_single_gap (oracle/ref_single.c) over a
    batch of gaps, in a reference library (shares its genome and tables)."""

    def __init__(self, ref, maxlookback, extraquerygap):
        lib = ref.lib
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        lib.ref_single_init.argtypes = [i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        lib.ref_single_setup.argtypes = [i32, i32, i32]
        lib.ref_single_gap_batch.argtypes = [vp, i32, vp, vp, vp, i64, vp]
        lib.ref_single_gap_batch.restype = i64
        mr, mg = ctypes.c_int(0), ctypes.c_int(0)
        lib.ref_single_init(maxlookback, extraquerygap, ctypes.byref(mr), ctypes.byref(mg))
        self.lib = lib
        self.max_rlength, self.max_glength = mr.value, mg.value

    def setup(self, user_open=0, user_extend=0, user_dynprog_p=False):
        self.lib.ref_single_setup(user_open, user_extend, int(user_dynprog_p))

    def bench(self, gaps, arena, nthreads, maxlookback, extraquerygap):
        """Wall seconds and a checksum of Dynprog_single_gap over every gap
        once on nthreads threads, each with its own Dynprog_T (sized by
        maxlookback / extraquerygap) and Pairpool_T."""
        lib = self.lib
        lib.ref_single_gap_bench.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
        lib.ref_single_gap_bench.restype = ctypes.c_double
        cs = ctypes.c_int64(0)
        secs = lib.ref_single_gap_bench(_ptr(gaps), gaps.size, _ptr(arena), nthreads, maxlookback, extraquerygap,
                                        ctypes.byref(cs))
        return secs, cs.value

    def run(self, gaps, arena):
        """Per gap: stats (traceback_score, nmatches, nmismatches, nopens,
        nindels, npairs, list is NULL, dynprogindex after), record offsets,
        and the records (the returned List, head first)."""
        n = gaps.size
        stats = np.zeros((n, 8), np.int32)
        off = np.zeros(n, np.int64)
        cap = int((np.maximum(gaps["rlength"], 0).astype(np.int64) + np.maximum(gaps["glength"], 0) + 2).sum()) + 1
        recs = np.zeros(cap, dtype=_rec_dtype())
        used = self.lib.ref_single_gap_batch(_ptr(gaps), n, _ptr(arena), _ptr(stats), _ptr(recs), cap, _ptr(off))
        assert used <= cap
        return stats, off, recs[:used]


def _segment(g, galt, chroffset, chrhigh, goffset, glength, watsonp):
    """Dynprog_single_gap's gsequence and gsequence_alt: Genome_get_segment_
    right (plus) or the reverse complement of Genome_get_segment_left
    (minus), src/genome.c:11022-11120; g and galt are uint8 genomes (ACGTN),
    galt's characters at g's N positions read N."""
    compl = {65: 84, 67: 71, 71: 67, 84: 65}
    seg = np.empty(glength, np.uint8)
    alt = np.empty(glength, np.uint8)
    for j in range(glength):
        pos = chroffset + goffset + j if watsonp else chrhigh - goffset - j
        if (watsonp and pos >= chrhigh) or (not watsonp and pos < chroffset):
            seg[j] = alt[j] = 42
            continue
        c = int(g[pos])
        a = c if c == 78 else int(galt[pos])
        seg[j], alt[j] = (c, a) if watsonp else (compl.get(c, c), compl.get(a, a))
    return seg, alt


def single_gap_restated(orc, gaps, arena, g, galt, user=None):
    """Dynprog_single_gap (src/dynprog_single.c:428-675) restated over a CPU
    oracle's fill and traceback (orc: restatement() or reference(), tables
    and genome set).  Returns the same (stats, offsets, records) as
    ReferenceSingleGap.run, without the dynprogindex column's update."""
    n = gaps.size
    stats = np.zeros((n, 8), np.int32)
    off = np.zeros(n, np.int64)
    out = []
    used = 0
    for i in range(n):
        x = gaps[i]
        rl, gl = int(x["rlength"]), int(x["glength"])
        off[i] = used
        stats[i, 7] = int(x["dynprogindex"])
        if rl <= 0 or gl <= 0 or rl > int(x["max_rlength"]) or gl > int(x["max_glength"]):
            stats[i, :7] = (-32768, 0, 0, 0, 0, 0, 1)
            continue
        seg, alt = _segment(g, galt, int(x["chroffset"]), int(x["chrhigh"]), int(x["goffset"]), gl,
                            bool(x["watsonp"]))
        rs = arena[int(x["rseq"]):int(x["rseq"]) + rl]
        ru = arena[int(x["rseq_uc"]):int(x["rseq_uc"]) + rl]
        q = 0 if x["defect_rate"] < 0.003 else 1 if x["defect_rate"] < 0.014 else 2
        if gl == rl:
            # single_gap_simple (:345-425): pushed left to right, so the List
            # starts at the last position
            score = nmatch = nmis = 0
            recs = []
            for k in range(rl):
                c1, cu, c2, ca = int(rs[k]), int(ru[k]), int(seg[k]), int(alt[k])
                if c2 == 42:
                    continue
                if cu == c2 or cu == ca:
                    comp = b"*"
                elif orc.consistent(int(x["genestrand"]), cu, c2) or orc.consistent(int(x["genestrand"]), cu, ca):
                    comp = b":"
                else:
                    comp = b" "
                if comp == b" ":
                    score -= 3
                    nmis += 1
                else:
                    score += 1
                    nmatch += 1
                qp, gp = int(x["roffset"]) + k, int(x["goffset"]) + k
                if qp >= 0 and gp >= 0:
                    recs.append((qp, gp, bytes([c1]), comp, bytes([c2]), bytes([ca])))
            if nmis <= 1 and recs:
                stats[i, :7] = (score, nmatch, nmis, 0, 0, len(recs), 0)
                out.extend(reversed(recs))
                used += len(recs)
                continue
        # the fill (:599-650): bands, precision by use8p_size, traceback from (rlength, glength)
        xb = int(x["extraband_single"])
        if not x["widebandp"]:
            lb = ub = xb
        elif gl >= rl:
            lb, ub = xb, gl - rl + xb
        else:
            lb, ub = rl - gl + xb, xb
        use8p = 128 // (3, 2, 1)[q] - 1
        p = np.zeros(1, dtype=_pair_dtype())
        local = np.concatenate([rs, ru, seg, alt])
        p["rseq"], p["rseq_uc"], p["gseq"], p["gseq_alt"] = 0, rl, 2 * rl, 2 * rl + gl
        p["rlength"], p["glength"], p["lband"], p["uband"] = rl, gl, lb, ub
        p["variant"] = 0
        p["precision"] = 8 if (rl < use8p and gl < use8p) else 16
        p["mismatchtype"] = q
        p["flags"] = 4 | (1 if x["jump_late_p"] else 0)
        if user is not None:
            p["open"], p["extend"] = user
        else:
            p["open"], p["extend"] = (-8, -7, -6)[q], (-3, -2, -1)[q]
        p["tb_r"], p["tb_c"] = rl, gl
        p["queryoffset"], p["genomeoffset"] = int(x["roffset"]), int(x["goffset"])
        p["chroffset"], p["chrhigh"] = int(x["chroffset"]), int(x["chrhigh"])
        p["watsonp"], p["genestrand"] = int(x["watsonp"]), int(x["genestrand"])
        p["dynprogindex"] = int(x["dynprogindex"])
        r = orc.align(p, 0, local, want_matrix=False)
        st = r["stats"]
        stats[i, :7] = (st[0], st[1], st[2], st[3], st[4], r["nrecs"], r["nrecs"] == 0)
        for rec in r["recs"]:
            out.append(tuple(rec))
        used += len(r["recs"])
    recs = np.array(out, dtype=_rec_dtype()) if out else np.zeros(0, dtype=_rec_dtype())
    return stats, off, recs



class ReferenceEndGap:
    """The reference's own Dynprog_end5_gap / Dynprog_end3_gap
    (oracle/ref_end.c) over a batch of end gaps, in a reference library
    (shares its genome and tables)."""

    def __init__(self, ref, maxlookback, extraquerygap):
        lib = ref.lib
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        lib.ref_end_init.argtypes = [i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        lib.ref_end_setup.argtypes = [i32, i32, i32]
        lib.ref_end_gap_batch.argtypes = [vp, i32, vp, vp, vp, i64, vp]
        lib.ref_end_gap_batch.restype = i64
        mr, mg = ctypes.c_int(0), ctypes.c_int(0)
        lib.ref_end_init(maxlookback, extraquerygap, ctypes.byref(mr), ctypes.byref(mg))
        self.lib = lib
        self.max_rlength, self.max_glength = mr.value, mg.value

    def setup(self, user_open=0, user_extend=0, user_dynprog_p=False):
        self.lib.ref_end_setup(user_open, user_extend, int(user_dynprog_p))

    def bench(self, gaps, arena, nthreads, maxlookback, extraquerygap):
        """Wall seconds and a checksum of the end-gap solvers over every gap
        once on nthreads threads, each with its own Dynprog_T (sized by
        maxlookback / extraquerygap) and Pairpool_T."""
        lib = self.lib
        lib.ref_end_gap_bench.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
        lib.ref_end_gap_bench.restype = ctypes.c_double
        cs = ctypes.c_int64(0)
        secs = lib.ref_end_gap_bench(_ptr(gaps), gaps.size, _ptr(arena), nthreads, maxlookback, extraquerygap,
                                     ctypes.byref(cs))
        return secs, cs.value

    def run(self, gaps, arena):
        """Per gap: stats (traceback_score, nmatches, nmismatches, nopens,
        nindels, npairs, list is NULL, dynprogindex after), record offsets,
        and the records (the returned List, head first)."""
        n = gaps.size
        stats = np.zeros((n, 8), np.int32)
        off = np.zeros(n, np.int64)
        cap = int((np.maximum(gaps["rlength"], 0).astype(np.int64) + np.maximum(gaps["glength"], 0) + 2).sum()) + 1
        recs = np.zeros(cap, dtype=_rec_dtype())
        used = self.lib.ref_end_gap_batch(_ptr(gaps), n, _ptr(arena), _ptr(stats), _ptr(recs), cap, _ptr(off))
        assert used <= cap
        return stats, off, recs[:used]


class ReferenceCdnaGap:
    """The reference's own Dynprog_cdna_gap (oracle/ref_cdna.c) over a batch
    of gaps, in a reference library (shares its genome and tables)."""

    def __init__(self, ref, maxlookback, extraquerygap):
        lib = ref.lib
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        lib.ref_cdna_init.argtypes = [i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        lib.ref_cdna_gap_batch.argtypes = [vp, i32, vp, vp, vp, i64, vp]
        lib.ref_cdna_gap_batch.restype = i64
        mr, mg = ctypes.c_int(0), ctypes.c_int(0)
        lib.ref_cdna_init(maxlookback, extraquerygap, ctypes.byref(mr), ctypes.byref(mg))
        self.lib = lib
        self.max_rlength, self.max_glength = mr.value, mg.value

    def bench(self, gaps, arena, nthreads, maxlookback, extraquerygap):
        """Wall seconds and a checksum of Dynprog_cdna_gap over every gap once
        on nthreads threads, each with its own Dynprog_T pair and Pairpool_T."""
        lib = self.lib
        lib.ref_cdna_gap_bench.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
        lib.ref_cdna_gap_bench.restype = ctypes.c_double
        cs = ctypes.c_int64(0)
        secs = lib.ref_cdna_gap_bench(_ptr(gaps), gaps.size, _ptr(arena), nthreads, maxlookback, extraquerygap,
                                      ctypes.byref(cs))
        return secs, cs.value

    def run(self, gaps, arena):
        """Per gap: stats (traceback_score, incompletep, 0, 0, 0, npairs, list
        is NULL, dynprogindex after), record offsets, and the records (the
        returned List, head first)."""
        n = gaps.size
        stats = np.zeros((n, 8), np.int32)
        off = np.zeros(n, np.int64)
        cap = int((np.maximum(gaps["rlengthL"], 0).astype(np.int64) + np.maximum(gaps["rlengthR"], 0)
                   + 2 * np.maximum(gaps["glength"], 0) + 24).sum()) + 1
        recs = np.zeros(cap, dtype=_rec_dtype())
        used = self.lib.ref_cdna_gap_batch(_ptr(gaps), n, _ptr(arena), _ptr(stats), _ptr(recs), cap, _ptr(off))
        assert used <= cap
        return stats, off, recs[:used]


def _segment_end(g, galt, chroffset, chrhigh, goffset, glength, watsonp, end):
    """The genome segment of an end gap, stored forward: end 3 is
    Dynprog_end3_gap's gsequence (Genome_get_segment_right from chroffset +
    goffset on the plus strand, the reverse complement of Genome_get_
    segment_left down from chrhigh - goffset on the minus strand; '*' at and
    above chrhigh, or below chroffset); end 5 is Dynprog_end5_gap's
    rev_gsequence (src/dynprog_end.c:1384-1390): Genome_get_segment_left
    ending at chroffset + goffset ('*' below chroffset) or the reverse
    complement of Genome_get_segment_right from chrhigh - goffset ('*' at
    and above chrhigh).  Character j is genomic coordinate goffset + j (end
    3) or goffset - (glength - 1) + j (end 5)."""
    compl = {65: 84, 67: 71, 71: 67, 84: 65}
    seg = np.empty(glength, np.uint8)
    alt = np.empty(glength, np.uint8)
    g0 = goffset - (glength - 1) if end == 5 else goffset
    for j in range(glength):
        pos = chroffset + g0 + j if watsonp else chrhigh - (g0 + j)
        if end == 5:
            star = pos < chroffset if watsonp else pos >= chrhigh
        else:
            star = pos >= chrhigh if watsonp else pos < chroffset
        if star:
            seg[j] = alt[j] = 42
            continue
        c = int(g[pos])
        a = c if c == 78 else int(galt[pos])
        seg[j], alt[j] = (c, a) if watsonp else (compl.get(c, c), compl.get(a, a))
    return seg, alt


def end_gap_restated(orc, gaps, arena, g, galt, user=None):
    """Dynprog_end5_gap / Dynprog_end3_gap (src/dynprog_end.c:1293-1650,
    :1923-2245) restated over a CPU oracle's fills and traceback (orc:
    restatement() or reference(), tables and genome set): ENDQ penalties by
    defect rate (:88-94), the length checks and cuts, Dynprog_compute_bands
    (src/dynprog.c:1246), 8-bit fills when either length is below 24
    (use8p_size[ENDQ], the || rule), the upper and lower fills (end 5 with
    revp and !jump_late_p), the endpoint scan (find_best_endpoint), the
    traceback from the best cell through the upper fill when bestc >= bestr,
    the nmatches + 1 < nmismatches rejection, and the List_reverse and
    indel trimming (end 5 reversed once more).  Returns the same (stats,
    offsets, records) as ReferenceEndGap.run, without the dynprogindex
    column's update.  NOGAPS gaps are not restated (stats all 0)."""
    n = gaps.size
    stats = np.zeros((n, 8), np.int32)
    off = np.zeros(n, np.int64)
    out = []
    used = 0
    for i in range(n):
        x = gaps[i]
        off[i] = used
        stats[i, 7] = int(x["dynprogindex"])
        stats[i, 6] = 1
        end, endalign = int(x["end"]), int(x["endalign"])
        rl, gl = int(x["rlength"]), int(x["glength"])
        if rl <= 0 or endalign == 2:
            continue
        rl = min(rl, int(x["max_rlength"]))
        if end == 5 and int(x["goffset"]) < 0:
            continue
        if gl <= 0:
            continue
        gl = min(gl, int(x["max_glength"]))
        if user is not None:
            op, ex = user
        else:
            d = float(x["defect_rate"])
            op, ex = (-10 if d < 0.003 else -8 if d < 0.014 else -6), -2
        xb = int(x["extraband_end"])
        qend = endalign == 1
        if qend:
            lb = ub = xb
        elif gl >= rl:
            lb, ub = xb, gl - rl + xb
        else:
            lb, ub = rl - gl + xb, xb
        prec = 8 if (rl < 24 or gl < 24) else 16
        seg, alt = _segment_end(g, galt, int(x["chroffset"]), int(x["chrhigh"]), int(x["goffset"]), gl,
                                bool(x["watsonp"]), end)
        r0 = int(x["rseq"]) - (rl - 1) if end == 5 else int(x["rseq"])
        u0 = int(x["rseq_uc"]) - (rl - 1) if end == 5 else int(x["rseq_uc"])
        rs, ru = arena[r0:r0 + rl], arena[u0:u0 + rl]
        late = (not x["jump_late_p"]) if end == 5 else bool(x["jump_late_p"])
        local = np.concatenate([rs, ru, seg, alt])
        p = np.zeros(1, dtype=_pair_dtype())
        p["rseq"], p["rseq_uc"], p["gseq"], p["gseq_alt"] = 0, rl, 2 * rl, 2 * rl + gl
        p["rlength"], p["glength"] = rl, gl
        p["precision"], p["mismatchtype"] = prec, 3
        p["open"], p["extend"] = op, ex
        p["flags"] = (1 if late else 0) | (2 if end == 5 else 0)
        p["queryoffset"], p["genomeoffset"] = int(x["roffset"]), int(x["goffset"])
        p["chroffset"], p["chrhigh"] = int(x["chroffset"]), int(x["chrhigh"])
        p["watsonp"], p["genestrand"] = int(x["watsonp"]), int(x["genestrand"])
        p["dynprogindex"] = int(x["dynprogindex"])
        up, lo = p.copy(), p.copy()
        up["variant"], up["uband"] = 1, ub
        lo["variant"], lo["lband"] = 2, lb
        if x["require_pos_score_p"]:
            continue
        Hu = orc.align(up, 0, local)["H"].reshape(gl + 1, rl + 1)
        Hl = orc.align(lo, 0, local)["H"].reshape(gl + 1, rl + 1)
        _, br, bc, _ = find_best_endpoint(Hu, Hl, rl, gl, lb, ub, late, qend, prec)
        t = (up if bc >= br else lo).copy()
        t["flags"] |= 4
        t["tb_r"], t["tb_c"] = br, bc
        r = orc.align(t, 0, local, want_matrix=False)
        st = r["stats"]
        score, nmatch, nmis, nopen, nindel = (int(v) for v in st[:5])
        if endalign in (0, 3) and nmatch + 1 < nmis:
            stats[i, :7] = (0, nmatch, nmis, nopen, nindel, 0, 1)
            continue
        recs = [tuple(rec) for rec in r["recs"]]
        k = 0
        while k < len(recs) and recs[k][3] == b"-":
            k += 1
        recs = recs[k:]
        if end == 5:
            recs.reverse()
        stats[i, :7] = (score, nmatch, nmis, nopen, nindel, len(recs), 0 if recs else 1)
        out.extend(recs)
        used += len(recs)
    recs = np.array(out, dtype=_rec_dtype()) if out else np.zeros(0, dtype=_rec_dtype())
    return stats, off, recs


def _pair_dtype():
    """struct gdp_pair (include/gdp.h), 88 bytes."""
    return np.dtype([
        ("rseq", "<i8"), ("rseq_uc", "<i8"), ("gseq", "<i8"), ("gseq_alt", "<i8"),
        ("rlength", "<i4"), ("glength", "<i4"), ("lband", "<i4"), ("uband", "<i4"),
        ("variant", "i1"), ("precision", "i1"), ("mismatchtype", "i1"), ("flags", "i1"),
        ("open", "<i2"), ("extend", "<i2"), ("tb_r", "<i4"), ("tb_c", "<i4"),
        ("queryoffset", "<i4"), ("genomeoffset", "<i4"), ("chroffset", "<u4"), ("chrhigh", "<u4"),
        ("watsonp", "i1"), ("genestrand", "i1"), ("xflags", "<i2"), ("dynprogindex", "<i4")])


def _rec_dtype():
    return np.dtype([("querypos", "<i4"), ("genomepos", "<i4"),
                     ("cdna", "S1"), ("comp", "S1"), ("genome", "S1"), ("genomealt", "S1")])


def reference(noflush=False):
    return CpuOracle(REF_LIB_NOFLUSH if noflush else REF_LIB, "ref_")


def restatement():
    return CpuOracle(ORACLE_LIB, "orc_")


def reference_available():
    return os.path.exists(REF_LIB)


def gmap_environment():
    """GMAP's host code around the product's reference-signature entry
    points.  Loaded into the global symbol scope, so that libgdp.so finds
    GMAP's Pairpool_push, Genome_get_char and tables there; load it before
    any other library that defines those names."""
    return CpuOracle(GMAPENV_LIB, "ref_", mode=ctypes.RTLD_GLOBAL)


def gmap_environment_available():
    return os.path.exists(GMAPENV_LIB)


def domain_mask(variant, rlength, glength, lband, uband):
    """Boolean (glength+1, rlength+1) mask of the reference's compare domain."""
    c = np.arange(glength + 1)[:, None]
    r = np.arange(rlength + 1)[None, :]
    if variant == 0:
        lo, hi = c - uband, c + lband
    elif variant == 1:
        lo, hi = c - uband, c
    else:
        lo, hi = c, c + lband
    m = (r >= np.maximum(lo, 1)) & (r <= np.minimum(hi, rlength)) & (c >= 1)
    return m


def find_best_endpoint(Hu, Hl, rlength, glength, lband, uband, jump_late, qend, precision, half=None):
    """The reference's end-gap endpoint scans over dense (c, r) score arrays
    of an upper fill (Hu) and a lower fill (Hl): find_best_endpoint_{8,16}
    (src/dynprog_end.c:143-294; rows 1..rlength, start score 0, bestr =
    bestc = 0) and, with `qend`, find_best_endpoint_to_queryend_indels_{8,16}
    (:358-508; row rlength only, start NEG_INFINITY_8/16, bestr = rlength,
    bestc = 0).  Each row scans the lower cells c < r, then the upper cells
    c >= r, keeping a cell with a score > (jump early) or >= (jump late) the
    best so far.  `half` ("upper" / "lower") restricts the scan to one
    matrix's cells.  Columns stop at glength: the reference's lower loop
    runs to c = r - 1 even past glength, outside the lower matrix, which
    only queries longer than glength + 1 reach.  Returns (finalscore,
    bestr, bestc, found)."""
    if qend:
        best, br, bc, rows = (-128 if precision == 8 else -32768), rlength, 0, [rlength]
    else:
        best, br, bc, rows = 0, 0, 0, range(1, rlength + 1)
    found = False
    for r in rows:
        clo, chigh = max(1, r - lband), min(glength, r + uband)
        for c in range(clo, chigh + 1):
            if c < r:
                if half == "upper":
                    continue
                v = int(Hl[c, r])
            else:
                if half == "lower":
                    continue
                v = int(Hu[c, r])
            if (v >= best) if jump_late else (v > best):
                best, br, bc, found = v, r, c, True
    return best, br, bc, found
