"""Parity checks of the CUDA path (through libgdp.so's C ABI) against a CPU
oracle (the compiled reference or the restatement, oracle/)."""
import ctypes

import numpy as np

import gdp
import oracle as orc


def _as_precision(pairs, i, prec):
    p = pairs[i:i + 1].copy()
    p["precision"] = prec
    p["flags"] = p["flags"] & ~gdp.FLAG_RERUN16
    return p


def expected_precision(oracle, pairs, i, arena, restatement=None):
    """The rerun contract for an 8-bit pair flagged RERUN16: keep the 8-bit
    outputs unless the 8-bit fill reaches 127 inside the band or ends at or
    below -98, or (when it traces back) its 8-bit traceback would read cells
    the 8-bit fill never wrote; then keep the 16-bit outputs."""
    p = pairs[i]
    if p["precision"] == 16:
        return 16
    if not (p["flags"] & gdp.FLAG_RERUN16):
        return 8
    q = _as_precision(pairs, i, 8)
    # the fill decides the overflow; the reference's 8-bit traceback is not
    # run here, since for some pairs it reads scratch its fill never wrote
    # (undefined: stale data from earlier calls, even out-of-range reads)
    q["flags"] = q["flags"] & ~gdp.FLAG_TRACEBACK
    o = oracle.align(q, 0, arena)
    m = orc.domain_mask(int(p["variant"]), int(p["rlength"]), int(p["glength"]),
                        int(p["lband"]), int(p["uband"])).ravel()
    sat = (o["H"][m] >= 127).any() if m.any() else False
    if sat or o["score"] <= -98:
        return 16
    if restatement is not None and (p["flags"] & gdp.FLAG_TRACEBACK):
        restatement.lib.orc_last_tb_stale.restype = ctypes.c_int
        restatement.align(_as_precision(pairs, i, 8), 0, arena, want_matrix=False)
        if restatement.lib.orc_last_tb_stale():
            return 16
    return 8


def final_cell_in_band(p):
    """Whether pair p's final cell (rlength, glength) lies in its band.
    Outside it the reference leaves the cell unwritten (the lower fill of a
    gap with glength > rlength), so its "score" is whatever the scratch
    held; the device reports NEG_INFINITY there."""
    d = int(p["rlength"]) - int(p["glength"])
    v = int(p["variant"])
    lo = 0 if v == gdp.LOWER else -int(p["uband"])
    hi = 0 if v == gdp.UPPER else int(p["lband"])
    return lo <= d <= hi


def check_fill(ctx, oracle, pairs, arena, max_report=5, production=False):
    """Fills every pair on the GPU and compares scores and directions over
    the reference's compare domain and the final score.  With
    production=True the fills run exactly as a production batch (no score
    dump, so every column takes the body a production run gives it) and
    the directions are decoded from the production direction words; the
    in-band scores are then not available and only the final score is
    compared.  Returns a list of failure strings (empty when bit-exact)."""
    offs, H, dN, dE, dF, res = ctx.fill_dump(pairs, arena, scores=not production)
    fails = []
    for i in range(pairs.size):
        p = pairs[i]
        if res["status"][i] != 0:
            fails.append(f"pair {i}: status {gdp.STATUS.get(int(res['status'][i]))}")
            continue
        prec = expected_precision(oracle, pairs, i, arena)
        if int(res["precision"][i]) != prec:
            fails.append(f"pair {i}: kept precision {res['precision'][i]} expected {prec}")
            continue
        q = _as_precision(pairs, i, prec)
        q["flags"] = q["flags"] & ~gdp.FLAG_TRACEBACK
        o = oracle.align(q, 0, arena)
        rl, gl = int(p["rlength"]), int(p["glength"])
        n = (rl + 1) * (gl + 1)
        m = orc.domain_mask(int(p["variant"]), rl, gl, int(p["lband"]), int(p["uband"])).ravel()
        a0 = int(offs[i])
        bad = []
        for name, got in (("H", H), ("dN", dN), ("dE", dE), ("dF", dF)):
            if got is None:
                continue
            g = got[a0:a0 + n]
            if not np.array_equal(g[m], o[name][m]):
                k = np.nonzero((g != o[name]) & m)[0][0]
                bad.append(f"{name}@(c={k // (rl + 1)},r={k % (rl + 1)}) gpu {g[k]} cpu {o[name][k]}")
        if final_cell_in_band(p):
            if int(res["score"][i]) != o["score"]:
                bad.append(f"score gpu {res['score'][i]} cpu {o['score']}")
        elif int(res["score"][i]) != (-128 if prec == 8 else -32768):
            bad.append(f"final cell outside the band: score gpu {res['score'][i]}, want NEG_INFINITY")
        if bad:
            fails.append(f"pair {i} var {p['variant']} prec {prec} r {rl} g {gl} l {p['lband']} "
                         f"u {p['uband']} flags {p['flags']}: " + "; ".join(bad[:3]))
            if len(fails) >= max_report:
                break
    return fails


def check_traceback(ctx, oracle, restatement, pairs, arena, max_report=5):
    """Aligns the batch end to end (fill + traceback) and compares the final
    score, traceback score and counts, and every Pair record.  Tracebacks
    for which the reference reads scratch the fill never wrote (undefined
    in the reference) must come back as GDP_ERR_BAND."""
    res, recs = ctx.align(pairs, arena)
    fails = []
    restatement.lib.orc_last_tb_stale.restype = ctypes.c_int
    nundef = 0
    for i in range(pairs.size):
        p = pairs[i]
        prec = int(res["precision"][i])
        want = expected_precision(oracle, pairs, i, arena, restatement)
        if prec != want:
            fails.append(f"pair {i}: kept precision {prec}, contract says {want}")
            continue
        q = _as_precision(pairs, i, prec)
        # the restatement first: where it says the reference's traceback
        # reads scratch its fill never wrote, the reference is not run (its
        # result is undefined and its reads may leave the scratch)
        restatement.align(q, 0, arena, want_matrix=False)
        stale = restatement.lib.orc_last_tb_stale()
        st = int(res["status"][i])
        if stale:
            nundef += 1
            if st != 2:
                fails.append(f"pair {i}: undefined traceback but status {gdp.STATUS.get(st)}")
            continue
        o = oracle.align(q, 0, arena, want_matrix=False)
        if st != 0:
            fails.append(f"pair {i}: status {gdp.STATUS.get(st)}")
            continue
        bad = []
        if final_cell_in_band(p) and int(res["score"][i]) != o["score"]:
            bad.append(f"score {res['score'][i]} vs {o['score']}")
        got = [int(res[k][i]) for k in ("tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs")]
        if got != [int(v) for v in o["stats"]]:
            bad.append(f"stats {got} vs {list(o['stats'])}")
        r0 = int(res["rec_offset"][i])
        g = recs[r0:r0 + int(res["nrecs"][i])]
        if g.tobytes() != o["recs"].tobytes():
            bad.append("records differ")
        if bad:
            fails.append(f"pair {i} var {p['variant']} prec {prec} r {p['rlength']} g {p['glength']}: "
                         + "; ".join(bad))
            if len(fails) >= max_report:
                break
    return fails, nundef
