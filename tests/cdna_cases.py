"""Seeded cDNA gaps (the arguments of Dynprog_cdna_gap) for the parity tests
of gdp_cdna_gap_batch.

The gaps look like those GMAP's stage 3 sends (src/stage3.c:9313): the read
holds more bases than the genome between two aligned blocks -- at least
glength + 10, as stage 3 asks before it calls the cDNA gap -- and both
query stretches are glength + extramaterial long (the left one from the
left block, the right one back from the right block), so each reaches into
the other block.  The query between the blocks is the genome stretch with
an insertion of unrelated bases, or with 9 genome bases replaced by more
unrelated ones, or unrelated bases, with substitutions.  The mix covers both strands, both tie
rules, 8-bit and 16-bit fills, the three defect-rate levels, segments that
leave the chromosome, glength <= 1 and lengths above the Dynprog_T maxima
(no pairs).  Query stretches are never shorter than the genome stretch, as
GMAP makes them: shorter ones would make the reference's bridge read rows
its fills never wrote.
"""
import numpy as np

import cases

ACGT = np.frombuffer(b"ACGT", np.uint8)


def cdna_gap_cases(seed, n, g, max_rlength, max_glength, max_len=70):
    """(gaps, arena) with n seeded cDNA gaps over genome g (uint8, ACGTN)."""
    import gdp
    import oracle
    rng = np.random.default_rng(seed)
    gaps = np.zeros(n, dtype=gdp.CDNA_GAP_DTYPE)
    chunks, off = [], 0
    L = g.size
    for i in range(n):
        gl = int(rng.integers(2, max_len + 1))
        em = int(rng.integers(0, 12))
        rl = gl + em
        chroffset = int(rng.integers(0, L // 2))
        chrhigh = int(rng.integers(chroffset + 6 * max_len, L - 1))
        span = chrhigh - chroffset
        watsonp = int(rng.random() < 0.5)
        if rng.random() < 0.08:
            goffset = max(0, span - gl + int(rng.integers(1, 8)))      # the segment leaves the chromosome
        else:
            goffset = int(rng.integers(0, span - gl))
        seg = oracle._segment_end(g, g, chroffset, chrhigh, goffset, gl, watsonp, 3)[0].copy()
        seg[seg == ord("*")] = rng.choice(ACGT, size=int((seg == ord("*")).sum()))
        u = rng.random()
        s = int(rng.integers(0, gl + 1))
        if u < 0.6:
            mid = np.concatenate([seg[:s], rng.choice(ACGT, size=int(rng.integers(10, 40))), seg[s:]])
        elif u < 0.8 and gl >= 12:
            s = min(s, gl - 9)   # 9 genome bases skipped as well
            mid = np.concatenate([seg[:s], rng.choice(ACGT, size=int(rng.integers(19, 40))), seg[s + 9:]])
        else:
            mid = rng.choice(ACGT, size=gl + int(rng.integers(10, 30)))
        mid = cases._mutate(rng, mid, float(rng.choice([0.0, 0.02, 0.05])), 0.0)
        # stage 3 calls the cDNA gap only for query gaps longer than the
        # genome gap by more than MININTRONLEN (src/stage3.c:9293)
        if mid.size < gl + 10:
            mid = np.concatenate([mid, rng.choice(ACGT, size=gl + 10 - mid.size)])
        # the blocks either side, long enough for both stretches to read into them
        left = rng.choice(ACGT, size=rl + 4)
        right = rng.choice(ACGT, size=rl + 4)
        q = np.concatenate([left, mid, right])
        quc = q.copy()
        if rng.random() < 0.2:
            k = rng.random(q.size) < 0.1
            q[k] = q[k] + 32
        roffsetL = int(rng.integers(0, 500))
        qbase = roffsetL - left.size              # query position of q[0]
        rev_roffsetR = roffsetL + mid.size - 1
        gl_field, rl_field = gl, rl
        w = rng.random()
        if w < 0.05:
            gl_field = int(rng.choice([0, 1]))
        elif w < 0.08:
            gl_field = max_glength + int(rng.integers(1, 20))
        elif w < 0.1:
            rl_field = max_rlength + int(rng.integers(1, 20))
        gaps["rseq"][i] = off + (roffsetL - qbase)
        gaps["rseq_uc"][i] = off + q.size + (roffsetL - qbase)
        chunks += [q, quc]
        off += 2 * q.size
        gaps["rlengthL"][i] = rl_field
        gaps["rlengthR"][i] = rl_field
        gaps["glength"][i] = gl_field
        gaps["roffsetL"][i] = roffsetL
        gaps["rev_roffsetR"][i] = rev_roffsetR
        gaps["goffset"][i] = goffset
        gaps["chroffset"][i] = chroffset
        gaps["chrhigh"][i] = chrhigh
        gaps["watsonp"][i] = watsonp
        gaps["genestrand"][i] = 0
        gaps["jump_late_p"][i] = int(rng.random() < 0.5)
        gaps["extraband_paired"][i] = int(rng.integers(0, 12))
        gaps["max_rlength"][i] = max_rlength
        gaps["max_glength"][i] = max_glength
        gaps["dynprogindex"][i] = int(rng.integers(1, 50)) * (1 if rng.random() < 0.5 else -1)
        gaps["defect_rate"][i] = float(rng.choice([0.0, 0.002, 0.01, 0.03]))
    arena = np.concatenate(chunks) if chunks else np.zeros(1, np.uint8)
    return gaps, arena
