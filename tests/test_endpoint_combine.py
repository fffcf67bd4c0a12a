"""gdp_endpoint_combine on the host (no GPU): merging the upper and lower
halves of an end-gap endpoint search gives the cell the reference's
row-then-column scan would keep (src/dynprog_end.c:143-294, :358-508).

The halves are built from small random score grids by the oracle's scan
(oracle.find_best_endpoint) restricted to each half (upper: c >= r, lower:
c < r); the merged answer must equal the scan over the whole grid."""
import numpy as np

import gdp
import oracle as orc


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
            s, r, c, f = orc.find_best_endpoint(H.T, H.T, rl, gl, lband, uband, late, qend, prec, half)
            res = np.zeros(1, dtype=gdp.RESULT_DTYPE)
            res["end_score"], res["end_r"], res["end_c"], res["end_found"] = s, r, c, int(f)
            halves.append(res)
        got = gdp.endpoint_combine(gdplib, halves[0], halves[1], late, qend, prec, rl)
        want = orc.find_best_endpoint(H.T, H.T, rl, gl, lband, uband, late, qend, prec)[:3]
        assert got == want, (trial, rl, gl, lband, uband, late, qend, got, want)
