"""Records golden vectors of the reference's own Dynprog_cdna_gap
(src/dynprog_cdna.c:786-1290, compiled into oracle/_ref/libgdpref.so).

Run in a checkout where oracle/_ref has been built from the reference
sources (oracle/Makefile, `make ref`):

    python tests/golden/make_golden_cdna.py

It writes tests/golden/cdna_gap.npz: 200 seeded cDNA gaps
(tests/cdna_cases.py) over a 64 kb genome with an alternate genome, and for
every gap the reference's traceback score, incompletep, the number of
pairs, whether the List is NULL, the dynprogindex after the call, and the
List's records, head first.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "gmap-gsnap_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import cdna_cases  # noqa: E402
import oracle  # noqa: E402
import single_cases  # noqa: E402

GENOME_LEN = 1 << 16


def main():
    ref = oracle.reference()
    ref.init(0)
    g, alt, blocks, altblocks = single_cases.genome_pair(2027, GENOME_LEN)
    ref.set_genome(blocks, altblocks, GENOME_LEN)
    rc = oracle.ReferenceCdnaGap(ref, 200, 40)
    gaps, arena = cdna_cases.cdna_gap_cases(9301, 200, g, rc.max_rlength, rc.max_glength)
    stats, off, recs = rc.run(gaps, arena)
    np.savez_compressed(os.path.join(HERE, "cdna_gap.npz"), gaps=gaps, arena=arena, genome=g, genome_alt=alt,
                        genome_blocks=blocks, genome_alt_blocks=altblocks, stats=stats, rec_offset=off, recs=recs)
    print(f"{gaps.size} gaps, {recs.size} records, {int(stats[:, 6].sum())} NULL lists")


if __name__ == "__main__":
    main()
