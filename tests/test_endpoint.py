"""End-gap endpoint search on the device (GDP_FLAG_ENDPOINT,
GDP_FLAG_ENDPOINT_QEND).

Dynprog_end5_gap / Dynprog_end3_gap fill the upper and the lower matrix of
one gap and scan both for the endpoint of the alignment
(src/dynprog_end.c:1415-1534): find_best_endpoint_{8,16} (:143-294) over
the band, find_best_endpoint_to_queryend_indels_{8,16} (:358-508) over the
last query row.  Here each fill runs its half of the scan over the scores
it computes, and gdp_endpoint_combine merges the halves.  The expected
answer is that scan (oracle.find_best_endpoint) over the reference's own
score matrices (oracle/_ref, or the pinned restatement): finalscore, bestr
and bestc must be identical.

Cases keep rlength <= glength + 1: for longer queries the reference's
lower-half scan (c < r) reads columns beyond glength, outside the lower
matrix it filled.
"""
import numpy as np
import pytest

import cases
import gdp
import oracle as orc

pytestmark = pytest.mark.gpu


def _gap_cases(seed, n):
    """n end gaps as (upper, lower) pair couples over the same sequences."""
    rng = np.random.default_rng(seed)
    base, arena = cases.random_cases(seed, n, variants=(1,), precisions=(8, 16), min_len=1, max_len=90)
    pairs = np.zeros(2 * n, dtype=gdp.PAIR_DTYPE)
    for i in range(n):
        p = base[i].copy()
        rl, gl = int(p["rlength"]), int(p["glength"])
        if rl > gl + 1:
            p["rlength"] = rl = gl + 1
        extra = int(rng.integers(0, 20))
        qend = rng.random() < 0.4
        flags = int(p["flags"]) & (gdp.FLAG_JUMP_LATE | gdp.FLAG_REVP)
        flags |= gdp.FLAG_ENDPOINT_QEND if qend else gdp.FLAG_ENDPOINT
        up, lo = p.copy(), p.copy()
        up["variant"], up["uband"], up["lband"] = gdp.UPPER, max(0, gl - rl) + extra, 0
        lo["variant"], lo["lband"], lo["uband"] = gdp.LOWER, max(0, rl - gl) + extra, 0
        for q in (up, lo):
            q["flags"] = flags
            q["tb_r"], q["tb_c"] = rl, gl
        pairs[2 * i], pairs[2 * i + 1] = up, lo
    return pairs, arena


@pytest.fixture(scope="module")
def env(gdplib, restatement):
    ref = orc.reference() if orc.reference_available() else restatement
    ref.init(0)
    g, blocks, altb = cases.genome(17, length=1 << 17)
    ref.set_genome(blocks, altb, g.size)
    ctx = gdp.Context(gdplib)
    ctx.set_genome(blocks, altb, g.size)
    yield ctx, ref
    ctx.close()


@pytest.mark.parametrize("seed", [501, 502])
def test_endpoint_search_matches_reference_scan(env, gdplib, seed):
    ctx, ref = env
    pairs, arena = _gap_cases(seed, 120)
    res, _ = ctx.align(pairs, arena)
    assert (res["status"] == 0).all(), res["status"]
    fails = []
    for i in range(0, pairs.size, 2):
        up, lo = pairs[i], pairs[i + 1]
        rl, gl = int(up["rlength"]), int(up["glength"])
        late = bool(up["flags"] & gdp.FLAG_JUMP_LATE)
        qend = bool(up["flags"] & gdp.FLAG_ENDPOINT_QEND)
        prec = int(up["precision"])
        ou, ol = ref.align(pairs, i, arena), ref.align(pairs, i + 1, arena)
        Hu = ou["H"].reshape(gl + 1, rl + 1)
        Hl = ol["H"].reshape(gl + 1, rl + 1)
        want = orc.find_best_endpoint(Hu, Hl, rl, gl, int(lo["lband"]), int(up["uband"]), late, qend, prec)[:3]
        got = gdp.endpoint_combine(gdplib, res[i], res[i + 1], late, qend, prec, rl)
        if got != want:
            fails.append(f"gap {i // 2} r {rl} g {gl} late {late} qend {qend} prec {prec}: got {got} want {want}")
    assert not fails, "\n".join(fails[:8])


def test_endpoint_flags_rejected_where_undefined(env):
    """Full-band fills and 8-bit rerun pairs do not take the search."""
    ctx, _ = env
    pairs, arena = _gap_cases(503, 4)
    pairs["variant"][0] = gdp.FULL
    pairs["flags"][2] |= gdp.FLAG_RERUN16
    pairs["precision"][2] = 8
    pairs["flags"][4] |= gdp.FLAG_ENDPOINT | gdp.FLAG_ENDPOINT_QEND
    res, _ = ctx.align(pairs, arena)
    assert res["status"][0] == 3 and res["status"][2] == 3 and res["status"][4] == 3
    assert (res["status"][[1, 3, 5, 6, 7]] == 0).all()
