"""Child process of tests/test_dropin.py: GMAP's own host code calling the
product's reference-signature entry points, compared with the reference.

The process first loads oracle/_ref/libgmapenv.so into the global symbol
scope.  That library is the reference's dynprog.c / pairpool.c / list.c /
mem.c / except.c without src/dynprog_simd.c, plus the oracle harness; its
Dynprog_simd_* and Dynprog_traceback_* calls therefore resolve to
libgdp.so, which fills on the GPU into the harness's Dynprog_T spaces and
pushes the traceback's Pairs through GMAP's own Pairpool_push.  The same
harness linked with the reference's dynprog_simd.o (libgdpref.so) gives the
expected results.  For every case the in-band scores and directions, the
final score, the traceback counters and the Pair list must be equal.

Cases whose reference traceback reads cells its fill never wrote (undefined
in the reference; flagged by the restatement) are only fill-checked.

Runs in its own process because the drop-in aborts on misuse, as the
reference does, and because GMAP's symbols must be global before libgdp.so
resolves them.  Prints one summary line; exit status 0 when bit-exact.
"""
import argparse
import ctypes
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))

import oracle as orc  # noqa: E402

ENV = orc.gmap_environment()   # first: GMAP's symbols become global

import numpy as np  # noqa: E402

import cases  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--n", type=int, default=200)
    ap.add_argument("--max-len", type=int, default=90)
    ap.add_argument("--min-len", type=int, default=1)
    ap.add_argument("--mode", type=int, default=0)
    args = ap.parse_args()

    ref = orc.reference()
    rest = orc.restatement()
    for o in (ENV, ref, rest):
        o.init(args.mode)
    rest.lib.orc_last_tb_stale.restype = ctypes.c_int
    _, blocks, altblocks = cases.genome(args.seed + 1000, 1 << 16)
    for o in (ENV, ref, rest):
        o.set_genome(blocks, altblocks, 1 << 16)

    pairs, arena = cases.random_cases(args.seed, args.n, max_len=args.max_len, min_len=args.min_len)
    pairs["flags"] &= ~np.int8(8)   # GDP_FLAG_RERUN16: the drop-in keeps each call's own precision
    if args.mode in (2, 4, 6):
        # non-stranded modes build consistency tables for genestrands +1 and +2
        # only (src/dynprog.c:1035-1046); GMAP never passes 0 there
        pairs["genestrand"] = np.random.default_rng(args.seed).integers(1, 3, pairs.size)
    fails, nundef = [], 0
    for i in range(pairs.size):
        p = pairs[i]
        rl, gl = int(p["rlength"]), int(p["glength"])
        rest.align(pairs, i, arena, want_matrix=False)
        stale = rest.lib.orc_last_tb_stale()
        q = pairs[i:i + 1].copy()
        if stale:
            nundef += 1
            q["flags"] &= ~np.int8(4)   # fill only
        e = ENV.align(q, 0, arena)
        r = ref.align(q, 0, arena)
        m = orc.domain_mask(int(p["variant"]), rl, gl, int(p["lband"]), int(p["uband"])).ravel()
        bad = []
        for name in ("H", "dN", "dE", "dF"):
            if not np.array_equal(e[name][m], r[name][m]):
                k = np.nonzero((e[name] != r[name]) & m)[0][0]
                bad.append(f"{name}@(c={k // (rl + 1)},r={k % (rl + 1)}) {e[name][k]} vs {r[name][k]}")
        if e["score"] != r["score"]:
            bad.append(f"score {e['score']} vs {r['score']}")
        if not stale:
            if list(e["stats"]) != list(r["stats"]):
                bad.append(f"stats {list(e['stats'])} vs {list(r['stats'])}")
            elif e["recs"].tobytes() != r["recs"].tobytes():
                bad.append("Pair records differ")
        if bad:
            fails.append(f"case {i} var {p['variant']} prec {p['precision']} r {rl} g {gl} "
                         f"l {p['lband']} u {p['uband']} flags {p['flags']}: " + "; ".join(bad[:3]))
    print(f"dropin seed {args.seed}: {pairs.size} cases, {len(fails)} mismatches, "
          f"{nundef} fill-only (undefined reference traceback)")
    for f in fails[:8]:
        print("  " + f)
    return 1 if fails else 0


if __name__ == "__main__":
    sys.exit(main())
