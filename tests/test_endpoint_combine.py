"""gdp_endpoint_combine on the host (no GPU): merging the upper and lower
halves of an end-gap endpoint search gives the cell the reference's
row-then-column scan would keep (src/dynprog_end.c:143-294, :358-508).

The halves are built from small random score grids by the same scan
restricted to each half (upper: c >= r, lower: c < r); the merged answer
must equal the scan over the whole grid."""
import numpy as np

import gdp


def _scan(H, rl, gl, lband, uband, late, qend, prec, half=None):
    if qend:
        best, br, bc, rows = (-128 if prec == 8 else -32768), rl, 0, [rl]
    else:
        best, br, bc, rows = 0, 0, 0, range(1, rl + 1)
    found = False
    for r in rows:
        for c in range(max(1, r - lband), min(gl, r + uband) + 1):
            if half == "upper" and c < r:
                continue
            if half == "lower" and c >= r:
                continue
            v = int(H[r, c])
            if (v >= best) if late else (v > best):
                best, br, bc, found = v, r, c, True
    return best, br, bc, found


def test_combine_matches_whole_scan(gdplib):
    rng = np.random.default_rng(11)
    for trial in range(400):
        rl, gl = int(rng.integers(1, 12)), int(rng.integers(1, 12))
        lband, uband = int(rng.integers(0, 8)), int(rng.integers(0, 8))
        late, qend = bool(rng.random() < 0.5), bool(rng.random() < 0.4)
        prec = 8 if rng.random() < 0.5 else 16
        H = rng.integers(-6, 5, size=(rl + 1, gl + 1))   # many ties
        halves = []
        for half in ("upper", "lower"):
            s, r, c, f = _scan(H, rl, gl, lband, uband, late, qend, prec, half)
            res = np.zeros(1, dtype=gdp.RESULT_DTYPE)
            res["end_score"], res["end_r"], res["end_c"], res["end_found"] = s, r, c, int(f)
            halves.append(res)
        got = gdp.endpoint_combine(gdplib, halves[0], halves[1], late, qend, prec, rl)
        want = _scan(H, rl, gl, lband, uband, late, qend, prec)[:3]
        assert got == want, (trial, rl, gl, lband, uband, late, qend, got, want)
