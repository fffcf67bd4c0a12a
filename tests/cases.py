"""Seeded random alignment cases for the parity tests.

Covers the reference's parameter space: all three variants, 8- and 16-bit
lanes, both tie rules (jump_late_p), revp, all mismatch types, gap
penalties in [-127, 0], IUPAC / lower-case / N / '*' characters, bands from
0 up to the full rectangle, and lengths around the 16- and 32-row block
boundaries.  Every case keeps the traceback start inside the filled band,
which is the precondition the reference's callers establish
(Dynprog_compute_bands, src/dynprog.c:1246-1261).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))
import gdp  # noqa: E402

ACGT = b"ACGT"
IUPAC = b"ACGTNRYWSMKHBVDXacgtnU"


def _seq(rng, n, alphabet_mix):
    """Random sequence; alphabet_mix in {0: ACGT, 1: mostly ACGT with IUPAC/lower case}."""
    s = rng.choice(np.frombuffer(ACGT, np.uint8), size=n)
    if alphabet_mix:
        k = rng.random(n) < 0.08
        s[k] = rng.choice(np.frombuffer(IUPAC, np.uint8), size=int(k.sum()))
    return s


def _mutate(rng, src, sub, indel):
    out = []
    i = 0
    while i < len(src):
        u = rng.random()
        if u < indel:
            L = int(rng.integers(1, 4))
            if rng.random() < 0.5:
                out.extend(rng.choice(np.frombuffer(ACGT, np.uint8), size=L).tolist())
            else:
                i += L
        elif u < indel + sub:
            out.append(int(rng.choice(np.frombuffer(ACGT, np.uint8))))
            i += 1
        else:
            out.append(int(src[i]))
            i += 1
    return np.array(out if out else [65], dtype=np.uint8)


def random_cases(seed, n, variants=(0, 1, 2), precisions=(8, 16), max_len=90,
                 genome_len=1 << 16, exotic=True, min_len=1, extras=(0, 1, 2, 3, 5, 8, 13, 20, 31, 40)):
    """Returns (pairs, arena) with n random cases."""
    rng = np.random.default_rng(seed)
    pairs = np.zeros(n, dtype=gdp.PAIR_DTYPE)
    chunks = []
    off = 0
    for i in range(n):
        variant = int(rng.choice(variants))
        prec = int(rng.choice(precisions))
        rl = int(rng.integers(min_len, max_len + 1))
        kind = rng.random()
        base = _seq(rng, rl, exotic and rng.random() < 0.3)
        if kind < 0.15:
            gseq = _seq(rng, max(1, rl + int(rng.integers(-rl // 8 - 1, rl // 8 + 2))),
                        exotic and rng.random() < 0.3)  # unrelated
        else:
            gseq = _mutate(rng, base, rng.choice([0.0, 0.02, 0.1, 0.3]), rng.choice([0.0, 0.02, 0.08]))
        gl = len(gseq)
        if variant == 1 and gl < rl:
            gseq = np.concatenate([gseq, _seq(rng, rl - gl, 0)])
            gl = rl
        if variant == 2 and gl > rl:
            gseq = gseq[:rl]
            gl = rl
        if exotic and rng.random() < 0.1:
            k = int(rng.integers(0, gl))
            gseq[k:k + int(rng.integers(1, 4))] = ord("*")
        galt = gseq.copy()
        if exotic and rng.random() < 0.3:
            m = rng.random(gl) < 0.1
            galt[m] = rng.choice(np.frombuffer(ACGT, np.uint8), size=int(m.sum()))
        ruc = np.array([c - 32 if 97 <= c <= 122 else c for c in base], dtype=np.uint8)
        # bands: keep (rl, gl) inside the band, as Dynprog_compute_bands does
        extra = int(rng.choice(list(extras)))
        if variant == 0:
            lb = max(0, rl - gl) + int(rng.integers(0, extra + 1))
            ub = max(0, gl - rl) + int(rng.integers(0, extra + 1))
        elif variant == 1:
            lb, ub = 0, (gl - rl) + int(rng.integers(0, extra + 1))
        else:
            lb, ub = (rl - gl) + int(rng.integers(0, extra + 1)), 0
        p = pairs[i]
        for arr in (base, ruc, gseq, galt):
            chunks.append(arr)
        p["rseq"] = off
        p["rseq_uc"] = off + rl
        p["gseq"] = off + 2 * rl
        p["gseq_alt"] = off + 2 * rl + gl
        off += 2 * rl + 2 * gl
        p["rlength"], p["glength"], p["lband"], p["uband"] = rl, gl, lb, ub
        p["variant"], p["precision"] = variant, prec
        p["mismatchtype"] = int(rng.integers(0, 4))
        flags = gdp.FLAG_TRACEBACK
        if rng.random() < 0.5:
            flags |= gdp.FLAG_JUMP_LATE
        if rng.random() < 0.3:
            flags |= gdp.FLAG_REVP
        p["flags"] = flags
        if rng.random() < 0.7:
            p["open"], p["extend"] = int(rng.choice([-8, -7, -6, -10])), int(rng.choice([-3, -2, -1]))
        else:
            p["open"], p["extend"] = int(rng.integers(-127, 1)), int(rng.integers(-127, 1))
        p["tb_r"], p["tb_c"] = rl, gl
        p["queryoffset"] = int(rng.integers(0, 1000))
        p["genomeoffset"] = int(rng.integers(0, genome_len - 2 * (gl + 64)))
        p["chroffset"] = int(rng.integers(0, 64))
        p["chrhigh"] = int(genome_len - rng.integers(0, 64))
        p["watsonp"] = int(rng.random() < 0.7)
        p["genestrand"] = 0
        p["dynprogindex"] = int(rng.integers(-5, 6))
    arena = np.concatenate(chunks).astype(np.uint8) if chunks else np.zeros(1, np.uint8)
    return pairs, arena


def genome(seed, length=1 << 16, n_frac=0.01):
    """Synthetic genome (with a few N) in genomecomp blocks, plus an alternate."""
    rng = np.random.default_rng(seed)
    g = rng.choice(np.frombuffer(ACGT, np.uint8), size=length)
    g[rng.random(length) < n_frac] = ord("N")
    alt = g.copy()
    m = rng.random(length) < 0.02
    alt[m] = rng.choice(np.frombuffer(ACGT, np.uint8), size=int(m.sum()))
    return g, encode_genomecomp(g), encode_genomecomp(alt)


def encode_genomecomp(g):
    """Genomecomp blocks (src/genome.c:9723): {high, low, flags} per 32 nt."""
    n = g.size
    nw = (n + 31) // 32
    pad = np.full(nw * 32, ord("A"), dtype=np.uint8)
    pad[:n] = g
    code = np.zeros(nw * 32, dtype=np.uint32)
    for ch, v in ((b"A", 0), (b"C", 1), (b"G", 2), (b"T", 3)):
        code[pad == ch[0]] = v
        code[pad == ch[0] + 32] = v
    isn = ~np.isin(pad, np.frombuffer(b"ACGTacgt", np.uint8))
    code[isn] = 0
    code = code.reshape(nw, 32)
    isn = isn.reshape(nw, 32)
    sh = (2 * np.arange(16)).astype(np.uint32)
    low = (code[:, :16] << sh).sum(axis=1).astype(np.uint32)
    high = (code[:, 16:] << sh).sum(axis=1).astype(np.uint32)
    flags = (isn.astype(np.uint32) << np.arange(32, dtype=np.uint32)).sum(axis=1).astype(np.uint32)
    out = np.zeros(3 * nw, dtype=np.uint32)
    out[0::3], out[1::3], out[2::3] = high, low, flags
    return out
