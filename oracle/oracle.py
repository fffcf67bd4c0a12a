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
