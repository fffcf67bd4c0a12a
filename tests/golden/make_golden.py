"""Records golden vectors from the reference's own compiled functions.

Run in a checkout where oracle/_ref/libgdpref.so has been built from the
reference sources (oracle/Makefile, `make ref`):

    python tests/golden/make_golden.py

It writes tests/golden/golden.npz: seeded random cases over all variants,
lane widths, tie rules, revp and mismatch types, plus samples of the
workload shapes, with for every case the reference's final score, its
traceback score and counts, its Pair records (push order), and a SHA-1
digest of its in-band scores and directions over the reference's compare
domain.  `defined` is False for the few tracebacks on which the reference
reads scratch its fill never wrote (their output is not defined).
"""
import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))

import cases  # noqa: E402
import gdp  # noqa: E402
import oracle  # noqa: E402


def fill_digest(out, pair):
    m = oracle.domain_mask(int(pair["variant"]), int(pair["rlength"]), int(pair["glength"]),
                           int(pair["lband"]), int(pair["uband"])).ravel()
    h = hashlib.sha1()
    for k in ("H", "dN", "dE", "dF"):
        h.update(np.ascontiguousarray(out[k][m]).tobytes())
    return np.frombuffer(h.digest(), np.uint8)


def concat(parts):
    arenas, off = [], 0
    out_pairs = []
    for p, a in parts:
        q = p.copy()
        for f in ("rseq", "rseq_uc", "gseq", "gseq_alt"):
            q[f] += off
        out_pairs.append(q)
        arenas.append(a)
        off += a.size
    return np.concatenate(out_pairs), np.concatenate(arenas)


def main():
    ref = oracle.reference()
    ref.init(0)
    rest = oracle.restatement()
    rest.init(0)
    rest.lib.orc_last_tb_stale.restype = ctypes.c_int
    g, blocks, altb = cases.genome(2024, length=1 << 17)
    ref.set_genome(blocks, altb, g.size)
    rest.set_genome(blocks, altb, g.size)
    lib = gdp.load()
    parts = [cases.random_cases(9001, 500), cases.random_cases(9002, 120, max_len=300)]
    parts.append(gdp.make_pairs(lib, gdp.WL_FIXED, 9003, g, 40))
    parts.append(gdp.make_pairs(lib, gdp.WL_SHORT, 9004, g, 40))
    pairs, arena = concat(parts)
    n = pairs.size
    score = np.zeros(n, np.int32)
    stats = np.zeros((n, 6), np.int32)
    digests = np.zeros((n, 20), np.uint8)
    defined = np.ones(n, np.uint8)
    recs = []
    for i in range(n):
        q = pairs[i:i + 1].copy()
        # the golden precision is the one the rerun contract keeps
        if q["flags"][0] & gdp.FLAG_RERUN16:
            o8 = ref.align(q.copy(), 0, arena)
            m = oracle.domain_mask(int(q["variant"][0]), int(q["rlength"][0]), int(q["glength"][0]),
                                   int(q["lband"][0]), int(q["uband"][0])).ravel()
            sat = bool((o8["H"][m] >= 127).any()) or o8["score"] <= -98
            if not sat and (q["flags"][0] & gdp.FLAG_TRACEBACK):
                rest.align(q.copy(), 0, arena, want_matrix=False)
                sat = bool(rest.lib.orc_last_tb_stale())   # undefined 8-bit traceback: rerun
            q["precision"] = 16 if sat else 8
        out = ref.align(q, 0, arena)
        rest.align(q, 0, arena, want_matrix=False)
        defined[i] = 0 if rest.lib.orc_last_tb_stale() else 1
        score[i] = out["score"]
        stats[i] = out["stats"]
        digests[i] = fill_digest(out, q[0])
        recs.append(out["recs"])
    recs = np.concatenate(recs)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), pairs=pairs, arena=arena,
                        genome_blocks=blocks, genome_alt=altb, genome_length=np.int64(g.size),
                        score=score, stats=stats, fill_digest=digests, defined=defined, recs=recs)
    print(f"{n} cases, {recs.size} records, {int((1 - defined).sum())} undefined tracebacks")


if __name__ == "__main__":
    main()
