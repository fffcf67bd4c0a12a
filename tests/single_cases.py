"""Seeded single-gap cases (Dynprog_single_gap's arguments) for the parity
tests of gdp_single_gap_batch.

The gaps look like those stage 3 sends (src/stage3.c:9092-9123): a query
stretch between two aligned blocks against the genome stretch between them,
widebandp true and extraband_single at least the length difference.  The
mix covers the single gap's branches: out-of-range lengths (no pairs),
equal lengths whose diagonal has 0..3 mismatches (the simple path and its
fall-through to the fill), indels (the fill), the 8-bit and 16-bit sizes of
each mismatch type (use8p_size 41 / 63 / 127), both strands, segments that
run past either chromosome end ('*'), minus-strand gaps at genomic
coordinate 0, lower-case and IUPAC query characters, an alternate genome,
both tie rules, and user penalties.
"""
import numpy as np

import cases

ACGT = np.frombuffer(b"ACGT", np.uint8)
COMPL = {ord("A"): ord("T"), ord("C"): ord("G"), ord("G"): ord("C"), ord("T"): ord("A")}


def segment(g, chroffset, chrhigh, goffset, glength, watsonp):
    """The gsequence Dynprog_single_gap reads (Genome_get_segment_right /
    _left, src/genome.c:11022-11120), for building queries near it."""
    out = np.empty(glength, np.uint8)
    for j in range(glength):
        if watsonp:
            pos = chroffset + goffset + j
            out[j] = ord("*") if pos >= chrhigh else g[pos]
        else:
            pos = chrhigh - goffset - j
            out[j] = ord("*") if pos < chroffset else COMPL.get(int(g[pos]), int(g[pos]))
    return out


def single_gap_cases(seed, n, g, max_rlength, max_glength, max_len=160):
    """(gaps, arena) with n seeded gaps over genome g (uint8, ACGTN)."""
    import gdp
    rng = np.random.default_rng(seed)
    gaps = np.zeros(n, dtype=gdp.SINGLE_GAP_DTYPE)
    chunks, off = [], 0
    L = g.size
    for i in range(n):
        u = rng.random()
        # lengths: short (8-bit for every mismatch type), middle, long (16-bit)
        rl = int(rng.choice([rng.integers(1, 41), rng.integers(41, 127), rng.integers(127, max_len + 1)],
                            p=[0.5, 0.3, 0.2]))
        kind = rng.random()
        if kind < 0.45:
            gl = rl                                    # equal lengths: the simple path or its fall-through
        elif kind < 0.9:
            gl = max(1, rl + int(rng.integers(-8, 9)))  # an indel or two
        else:
            gl = max(1, rl + int(rng.integers(-30, 31)))
        chroffset = int(rng.integers(0, L // 2))
        chrhigh = int(rng.integers(chroffset + 64, L))
        watsonp = int(rng.random() < 0.6)
        span = chrhigh - chroffset
        v = rng.random()
        if v < 0.1:
            goffset = max(0, span - gl + int(rng.integers(1, 12)))   # runs past the chromosome end
        elif v < 0.15 and not watsonp:
            goffset = 0                                               # minus strand at coordinate 0
        else:
            goffset = int(rng.integers(0, max(1, span - gl)))
        seg = segment(g, chroffset, chrhigh, goffset, gl, watsonp)
        base = seg.copy()
        base[base == ord("*")] = rng.choice(ACGT, size=int((base == ord("*")).sum()))
        if gl == rl:
            q = base.copy()
            nm = int(rng.choice([0, 1, 2, 3], p=[0.35, 0.35, 0.2, 0.1]))
            for k in rng.choice(rl, size=min(nm, rl), replace=False):
                q[k] = rng.choice(ACGT[ACGT != q[k]])
        else:
            q = cases._mutate(rng, base, 0.02, 0.0)
            if q.size > rl:
                q = q[:rl]
            elif q.size < rl:
                q = np.concatenate([q, rng.choice(ACGT, size=rl - q.size)])
        quc = q.copy()
        if rng.random() < 0.2:
            k = rng.random(rl) < 0.1
            q[k] = np.where(q[k] >= 97, q[k], q[k] + 32)        # lower-case query, upper-case rsequenceuc
        if rng.random() < 0.1:
            k = int(rng.integers(0, rl))
            quc[k] = q[k] = ord(rng.choice(list("NRYX")))
        if rng.random() < 0.04:
            rl_field = int(rng.choice([0, max_rlength + 1]))      # out-of-range lengths
        else:
            rl_field = rl
        gl_field = max_glength + 1 if rng.random() < 0.02 else gl
        gaps["rseq"][i] = off
        gaps["rseq_uc"][i] = off + rl
        chunks += [q, quc]
        off += 2 * rl
        gaps["rlength"][i] = rl_field
        gaps["glength"][i] = gl_field
        gaps["roffset"][i] = int(rng.integers(0, 2000))
        gaps["goffset"][i] = goffset
        gaps["chroffset"][i] = chroffset
        gaps["chrhigh"][i] = chrhigh
        gaps["watsonp"][i] = watsonp
        gaps["genestrand"][i] = 0                   # STANDARD mode has genestrand 0 only
        gaps["jump_late_p"][i] = int(rng.random() < 0.5)
        gaps["widebandp"][i] = 1
        gaps["extraband_single"][i] = abs(gl - rl) + int(rng.integers(0, 12))
        gaps["defect_rate"][i] = float(rng.choice([0.0, 0.002, 0.01, 0.03]))
        gaps["max_rlength"][i] = max_rlength
        gaps["max_glength"][i] = max_glength
        gaps["dynprogindex"][i] = int(rng.integers(1, 50)) * (1 if rng.random() < 0.5 else -1)
    arena = np.concatenate(chunks) if chunks else np.zeros(1, np.uint8)
    return gaps, arena


def genome_pair(seed, length):
    """A synthetic genome with a few N and an alternate genome (2 % other
    bases): (g, alt, blocks, altblocks), g and alt as uint8 ACGTN."""
    rng = np.random.default_rng(seed)
    g = rng.choice(ACGT, size=length)
    g[rng.random(length) < 0.01] = ord("N")
    alt = g.copy()
    m = rng.random(length) < 0.02
    alt[m] = rng.choice(ACGT, size=int(m.sum()))
    return g, alt, cases.encode_genomecomp(g), cases.encode_genomecomp(alt)
