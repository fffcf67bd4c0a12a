"""Records golden vectors of the reference's own Dynprog_end5_gap and
Dynprog_end3_gap (src/dynprog_end.c:1293-1650, :1923-2245, compiled into
oracle/_ref/libgdpref.so).

Run in a checkout where oracle/_ref has been built from the reference
sources (oracle/Makefile, `make ref`):

    python tests/golden/make_golden_end.py

It writes tests/golden/end_gap.npz: 300 seeded end gaps (tests/end_cases.py)
over a 64 kb genome with an alternate genome, and for every gap the
reference's traceback score and counts, the number of pairs, whether the
List is NULL, the dynprogindex after the call, and the List's records, head
first.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "gmap-gsnap_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import end_cases  # noqa: E402
import oracle  # noqa: E402
import single_cases  # noqa: E402

GENOME_LEN = 1 << 16


def main():
    ref = oracle.reference()
    ref.init(0)
    g, alt, blocks, altblocks = single_cases.genome_pair(2026, GENOME_LEN)
    ref.set_genome(blocks, altblocks, GENOME_LEN)
    re = oracle.ReferenceEndGap(ref, 200, 40)
    re.setup()
    gaps, arena = end_cases.end_gap_cases(9201, 300, g, re.max_rlength, re.max_glength)
    stats, off, recs = re.run(gaps, arena)
    np.savez_compressed(os.path.join(HERE, "end_gap.npz"), gaps=gaps, arena=arena, genome=g, genome_alt=alt,
                        genome_blocks=blocks, genome_alt_blocks=altblocks, stats=stats, rec_offset=off, recs=recs)
    print(f"{gaps.size} gaps, {recs.size} records, {int(stats[:, 6].sum())} NULL lists")


if __name__ == "__main__":
    main()
