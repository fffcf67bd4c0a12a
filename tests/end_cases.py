"""Seeded end gaps (the arguments of Dynprog_end5_gap / Dynprog_end3_gap)
for the parity tests of gdp_end_gap_batch.

The gaps look like those GMAP's stage 3 sends (src/stage3.c, the 5' and 3'
end extensions): the query beyond the last aligned block against the genome
beyond it, the genome stretch a little longer than the query.  The query
starts (end 3) or ends (end 5) with a stretch that matches the genome next
to the block, with mismatches and an indel or two, and continues with
unrelated bases, so that the endpoint search stops inside the band.  The
mix covers both ends, both strands, the three built end alignments
(QUERYEND_GAP, QUERYEND_INDELS, BEST_LOCAL), 8-bit and 16-bit fills
(either length below 24), segments that run past either chromosome end
('*'), lengths at and beyond the Dynprog_T's maxima (cut), zero and
negative lengths and end-5 offsets (no pairs), require_pos_score_p,
lower-case and IUPAC query characters, both tie rules and the three
defect-rate penalty levels.

Queries stay at most one base longer than their genome stretch (after the
cuts): for longer queries the reference's endpoint scan reads lower-matrix
cells beyond glength, which its fills never wrote.
"""
import numpy as np

import cases

ACGT = np.frombuffer(b"ACGT", np.uint8)


def end_segment(g, chroffset, chrhigh, goffset, glength, watsonp, end):
    """The segment the gap's fills read, stored forward (see
    oracle._segment_end); '*' where it leaves the chromosome."""
    import oracle
    return oracle._segment_end(g, g, chroffset, chrhigh, goffset, glength, watsonp, end)[0]


def end_gap_cases(seed, n, g, max_rlength, max_glength, max_len=180, endaligns=(0, 1, 3)):
    """(gaps, arena) with n seeded end gaps over genome g (uint8, ACGTN)."""
    import gdp
    rng = np.random.default_rng(seed)
    gaps = np.zeros(n, dtype=gdp.END_GAP_DTYPE)
    chunks, off = [], 0
    L = g.size
    for i in range(n):
        end = 5 if rng.random() < 0.5 else 3
        rl = int(rng.choice([rng.integers(1, 24), rng.integers(24, 90), rng.integers(90, max_len + 1)],
                            p=[0.35, 0.4, 0.25]))
        u = rng.random()
        if u < 0.7:
            gl = rl + int(rng.integers(0, 40))     # the genome stretch reaches beyond the query
        elif u < 0.85:
            gl = max(1, rl - 1)
        else:
            gl = max(1, rl + int(rng.integers(-1, 3)))
        chroffset = int(rng.integers(0, L // 2))
        chrhigh = int(rng.integers(chroffset + 4 * max_len, L - 1))
        span = chrhigh - chroffset
        watsonp = int(rng.random() < 0.5)
        v = rng.random()
        if v < 0.1:
            # the segment leaves the chromosome
            goffset = int(rng.integers(max(0, gl - 12), gl)) if end == 5 else max(0, span - gl + int(rng.integers(1, 12)))
        else:
            goffset = int(rng.integers(gl, span - gl)) if end == 5 else int(rng.integers(0, span - gl))
        seg = end_segment(g, chroffset, chrhigh, goffset, gl, watsonp, end)
        base = seg.copy()
        stars = base == ord("*")
        base[stars] = rng.choice(ACGT, size=int(stars.sum()))
        # the matching stretch next to the aligned block, then unrelated bases
        keep = int(rng.integers(0, rl + 1)) if rng.random() < 0.8 else rl
        if end == 3:
            near = cases._mutate(rng, base[:keep + 8], float(rng.choice([0.0, 0.02, 0.06])), 0.01)[:keep]
            q = np.concatenate([near, rng.choice(ACGT, size=rl - near.size)])
        else:
            near = cases._mutate(rng, base[::-1][:keep + 8], float(rng.choice([0.0, 0.02, 0.06])), 0.01)[:keep]
            q = np.concatenate([near, rng.choice(ACGT, size=rl - near.size)])[::-1].copy()
        quc = q.copy()
        if rng.random() < 0.2:
            k = rng.random(rl) < 0.1
            q[k] = q[k] + 32                             # lower-case query, upper-case rsequenceuc
        if rng.random() < 0.1:
            k = int(rng.integers(0, rl))
            quc[k] = q[k] = ord(rng.choice(list("NRYX")))
        w = rng.random()
        if w < 0.03:
            rl_field = int(rng.choice([0, -3]))          # no pairs
        elif w < 0.06:
            rl_field = max_rlength + int(rng.integers(1, 30))   # cut to max_rlength
        else:
            rl_field = rl
        gl_field = gl
        if rng.random() < 0.03:
            gl_field = int(rng.choice([0, -2]))
        elif rl_field > max_rlength or rng.random() < 0.03:
            gl_field = max_glength + int(rng.integers(1, 30))   # cut to max_glength
        rl_store = max(rl, min(max(rl_field, 0), max_rlength))
        if rl_store > rl:
            q = np.concatenate([q, rng.choice(ACGT, size=rl_store - rl)]) if end == 3 else \
                np.concatenate([rng.choice(ACGT, size=rl_store - rl), q])
            quc = q.copy()
        gaps["end"][i] = end
        if end == 5:
            # rev_rsequence points at the query's last character
            gaps["rseq"][i] = off + rl_store - 1
            gaps["rseq_uc"][i] = off + rl_store + rl_store - 1
        else:
            gaps["rseq"][i] = off
            gaps["rseq_uc"][i] = off + rl_store
        chunks += [q, quc]
        off += 2 * rl_store
        gaps["rlength"][i] = rl_field
        gaps["glength"][i] = gl_field
        gaps["roffset"][i] = int(rng.integers(rl_store, 3000)) if end == 5 else int(rng.integers(0, 3000))
        gaps["goffset"][i] = -1 if (end == 5 and rng.random() < 0.02) else goffset
        gaps["chroffset"][i] = chroffset
        gaps["chrhigh"][i] = chrhigh
        gaps["endalign"][i] = int(rng.choice(endaligns))
        gaps["watsonp"][i] = watsonp
        gaps["genestrand"][i] = 0
        gaps["jump_late_p"][i] = int(rng.random() < 0.5)
        gaps["require_pos_score_p"][i] = int(rng.random() < 0.04)
        gaps["extraband_end"][i] = int(rng.integers(0, 12))
        gaps["defect_rate"][i] = float(rng.choice([0.0, 0.002, 0.01, 0.03]))
        gaps["max_rlength"][i] = max_rlength
        gaps["max_glength"][i] = max_glength
        gaps["dynprogindex"][i] = int(rng.integers(1, 50)) * (1 if rng.random() < 0.5 else -1)
    arena = np.concatenate(chunks) if chunks else np.zeros(1, np.uint8)
    return gaps, arena
