"""Bit-exact parity of the CUDA fills and tracebacks (called through
libgdp.so's C ABI) with the reference's AVX2 functions.

The oracle is the reference itself compiled from its sources
(oracle/_ref/libgdpref.so) when that library is present, else the C
restatement (oracle/liboracle.so) that tests/test_oracle.py pins against
it.  Bar: identical integers -- every in-band score and E/F/nogap
direction over the reference's compare domain, the final score, the
traceback score and counts, and every Pair record.
"""
import os

import numpy as np
import pytest

import cases
import gdp
import oracle as orc
import parity

pytestmark = pytest.mark.gpu

GENOME = {}


@pytest.fixture(scope="module")
def env(gdplib, restatement):
    ref = orc.reference() if orc.reference_available() else restatement
    ref.init(0)
    g, blocks, altb = cases.genome(5, length=1 << 17)
    ctx = gdp.Context(gdplib)
    ctx.set_genome(blocks, altb, g.size)
    ref.set_genome(blocks, altb, g.size)
    restatement.set_genome(blocks, altb, g.size)
    GENOME['g'] = g
    yield ctx, ref, restatement
    ctx.close()


@pytest.mark.parametrize("seed,variants,precs", [
    (101, (0,), (16,)), (102, (0,), (8,)), (103, (1,), (16,)), (104, (1,), (8,)),
    (105, (2,), (16,)), (106, (2,), (8,)), (107, (0, 1, 2), (8, 16)),
])
def test_fill_random(env, seed, variants, precs):
    ctx, ref, _ = env
    pairs, arena = cases.random_cases(seed, 300, variants=variants, precisions=precs)
    fails = parity.check_fill(ctx, ref, pairs, arena)
    assert not fails, "\n".join(fails)


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("prec,rerun", [(16, False), (8, False), (8, True)])
def test_production_bodies_cell_by_cell(env, variant, prec, rerun):
    """The column bodies a production batch runs -- the steady-column and
    half-width bodies, and for rerun pairs the 16-bit pass that tracks the
    in-band maximum and the 8-bit pass -- compared cell by cell: every
    in-band E/F/nogap direction decoded from the production direction
    words, and the final score, for both tie rules.  Bands are wide enough
    for most columns of a block to be steady."""
    ctx, ref, _ = env
    seed = 500 + 10 * variant + prec + (1 if rerun else 0)
    pairs, arena = cases.random_cases(seed, 240, variants=(variant,), precisions=(prec,), min_len=8,
                                      max_len=220, extras=(4, 9, 16, 20, 31, 40, 64))
    if rerun:
        pairs["flags"] |= gdp.FLAG_RERUN16
    assert set(np.unique(pairs["flags"] & gdp.FLAG_JUMP_LATE).tolist()) == {0, gdp.FLAG_JUMP_LATE}
    fails = parity.check_fill(ctx, ref, pairs, arena, production=True)
    assert not fails, "\n".join(fails)


def test_rerun_bound_counts_the_corner(env):
    """The upper and lower fills score the corner cell (0, 0) with one table
    entry, so an exact match of 42 x 42 reaches 3 + 42 * 3 = 129 in 16 bits
    and saturates the 8-bit fill at (42, 42).  Rerun pairs of 40-44 rows
    around that bound, exact and with one mismatch, in every variant, must
    keep the precision the rerun contract gives, with every output
    bit-exact."""
    ctx, ref, rest = env
    rng = np.random.default_rng(4242)
    rows, chunks, off = [], [], 0
    for variant in (0, 1, 2):
        for n in (40, 41, 42, 43, 44):
            for mism in (0, 1):
                for late in (0, 1):
                    q = rng.choice(np.frombuffer(b"ACGT", np.uint8), size=n)
                    g = q.copy()
                    if mism:
                        k = int(rng.integers(0, n))
                        g[k] = ord("A") if g[k] != ord("A") else ord("C")
                    rows.append((variant, n, late, off))
                    chunks += [q, q, g, g]
                    off += 4 * n
    pairs = np.zeros(len(rows), dtype=gdp.PAIR_DTYPE)
    for j, (variant, n, late, o) in enumerate(rows):
        p = pairs[j]
        p["rseq"], p["rseq_uc"], p["gseq"], p["gseq_alt"] = o, o + n, o + 2 * n, o + 3 * n
        p["rlength"] = p["glength"] = n
        p["lband"], p["uband"] = (3, 3) if variant == 0 else ((0, 4) if variant == 1 else (4, 0))
        p["variant"], p["precision"], p["mismatchtype"] = variant, 8, 1
        p["open"], p["extend"] = -30, -56
        p["flags"] = gdp.FLAG_TRACEBACK | gdp.FLAG_RERUN16 | (gdp.FLAG_JUMP_LATE if late else 0)
        p["tb_r"], p["tb_c"] = n, n
        p["genomeoffset"], p["chrhigh"], p["watsonp"], p["dynprogindex"] = 100, 60000, 1, 1
    arena = np.concatenate(chunks).astype(np.uint8)
    fails = parity.check_fill(ctx, ref, pairs, arena, production=True)
    assert not fails, "\n".join(fails)
    fails = parity.check_fill(ctx, ref, pairs, arena)
    assert not fails, "\n".join(fails)
    fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
    assert not fails, "\n".join(fails)


@pytest.mark.parametrize("kind,n", [(gdp.WL_SHORT, 400), (gdp.WL_CDNA, 6), (gdp.WL_LONG, 3)])
def test_production_bodies_on_workload_pairs(env, gdplib, kind, n):
    """The bench's own workload distributions through the production column
    bodies: every in-band direction and the final score against the
    reference, at the precision the rerun contract keeps."""
    ctx, ref, _ = env
    pairs, arena = gdp.make_pairs(gdplib, kind, 90 + kind, GENOME['g'], n)
    fails = parity.check_fill(ctx, ref, pairs, arena, production=True)
    assert not fails, "\n".join(fails)


@pytest.mark.parametrize("seed", [201, 202, 203])
def test_traceback_random(env, seed):
    ctx, ref, rest = env
    pairs, arena = cases.random_cases(seed, 400)
    fails, nundef = parity.check_traceback(ctx, ref, rest, pairs, arena)
    assert not fails, "\n".join(fails)


@pytest.mark.parametrize("seed,variants", [(301, (0,)), (302, (1,)), (303, (2,))])
def test_long_pairs_one_warp_per_pair(env, seed, variants):
    """Pairs with at least 512 lanes run on lane groups (lane l of a group
    owns blocks l, l + K, ...); they must be bit-exact like the
    one-thread-per-pair fills."""
    ctx, ref, rest = env
    pairs, arena = cases.random_cases(seed, 10, variants=variants, precisions=(16,), min_len=530,
                                      max_len=1400, extras=(0, 3, 10, 40, 90))
    ctx.profile(True)
    ctx.profile_reset()
    fails = parity.check_fill(ctx, ref, pairs, arena)
    assert not fails, "\n".join(fails)
    fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
    assert not fails, "\n".join(fails)
    kernels = ctx.profile_read()
    ctx.profile(False)
    assert any(k.startswith("fill_warp") for k in kernels), kernels


@pytest.mark.parametrize("seed,variants", [(311, (0,)), (312, (1,)), (313, (2,))])
def test_wide_bands_one_cta_per_pair(env, seed, variants):
    """Long pairs whose blocks sweep more columns than one warp can pipeline
    run one CTA per pair (2 to 16 warps, shared-memory hand-off between
    warps); bit-exact like the other fills."""
    ctx, ref, rest = env
    pairs, arena = cases.random_cases(seed, 5, variants=variants, precisions=(16,), min_len=520,
                                      max_len=900, extras=(0, 40))
    # widen the band past what one warp can pipeline (sweep > 496 columns per block)
    if variants[0] == 0:
        pairs["lband"] += 260
        pairs["uband"] += 300
    elif variants[0] == 1:
        pairs["uband"] += 560
    else:
        pairs["lband"] += 560
    ctx.profile(True)
    ctx.profile_reset()
    fails = parity.check_fill(ctx, ref, pairs, arena)
    assert not fails, "\n".join(fails)
    fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
    assert not fails, "\n".join(fails)
    kernels = ctx.profile_read()
    ctx.profile(False)
    assert any(k.startswith("fill_cta") for k in kernels), kernels


@pytest.mark.parametrize("check_groups", [0, 1])
def test_rerun_contract(env, gdplib, check_groups):
    """8-bit pairs with the 16-bit rerun: the kept precision follows the
    overflow rule, and the kept outputs are bit-exact with that precision,
    whether the 8-bit pass runs one thread per pair or on lane groups."""
    ctx, ref, rest = env
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_SHORT, 31, GENOME['g'], 200)
    keep = ctx.get_param("check_groups"), ctx.get_param("check_min_x")
    ctx.set_param("check_groups", check_groups)
    ctx.set_param("check_min_x", 1 << 30)
    try:
        ctx.profile(True)
        ctx.profile_reset()
        fails = parity.check_fill(ctx, ref, pairs, arena)
        assert not fails, "\n".join(fails)
        res, _ = ctx.align(pairs, arena)
        assert (res["status"] == 0).all()
        assert (res["precision"] == 16).sum() > 0
        fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
        assert not fails, "\n".join(fails)
        kernels = ctx.profile_read()
        ctx.profile(False)
    finally:
        ctx.set_param("check_groups", keep[0])
        ctx.set_param("check_min_x", keep[1])
    assert any("8bit-check" in k and k.startswith("fill_warp" if check_groups else "fill_thread")
               for k in kernels), kernels


@pytest.mark.parametrize("kind,n", [(gdp.WL_FIXED, 300), (gdp.WL_CDNA, 12), (gdp.WL_LONG, 4)])
def test_workload_shapes(env, gdplib, kind, n):
    ctx, ref, rest = env
    pairs, arena = gdp.make_pairs(gdplib, kind, 40 + kind, GENOME['g'], n)
    if kind != gdp.WL_FIXED:
        fails = parity.check_fill(ctx, ref, pairs[:3], arena)
        assert not fails, "\n".join(fails)
    fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
    assert not fails, "\n".join(fails)


def test_edge_shapes(env):
    """Lengths 1, block boundaries (15/16/17, 31/32/33), zero bands, bands
    wider than the matrix."""
    ctx, ref, rest = env
    rng = np.random.default_rng(7)
    rows = []
    for rl in (1, 2, 15, 16, 17, 31, 32, 33, 47, 48, 64, 65):
        for dg in (0, 1, -1, 5):
            gl = max(1, rl + dg)
            for variant in (0, 1, 2):
                if variant == 1 and gl < rl:
                    continue
                if variant == 2 and gl > rl:
                    continue
                for lb_extra, ub_extra in ((0, 0), (1, 2), (40, 40)):
                    rows.append((rl, gl, variant, lb_extra, ub_extra))
    pairs, arena = cases.random_cases(0, 1)
    out = np.zeros(len(rows) * 2, dtype=gdp.PAIR_DTYPE)
    chunks, off = [], 0
    for j, (rl, gl, variant, le, ue) in enumerate(rows):
        for prec_i, prec in enumerate((8, 16)):
            q = rng.choice(np.frombuffer(b"ACGT", np.uint8), size=rl)
            gq = rng.choice(np.frombuffer(b"ACGT", np.uint8), size=gl)
            gq[:min(rl, gl)] = q[:min(rl, gl)]
            p = out[2 * j + prec_i]
            chunks += [q, q, gq, gq]
            p["rseq"], p["rseq_uc"], p["gseq"], p["gseq_alt"] = off, off + rl, off + 2 * rl, off + 2 * rl + gl
            off += 2 * rl + 2 * gl
            p["rlength"], p["glength"], p["variant"], p["precision"] = rl, gl, variant, prec
            if variant == 0:
                p["lband"], p["uband"] = max(0, rl - gl) + le, max(0, gl - rl) + ue
            elif variant == 1:
                p["uband"] = gl - rl + ue
            else:
                p["lband"] = rl - gl + le
            p["open"], p["extend"], p["mismatchtype"] = -8, -3, 0
            p["flags"] = gdp.FLAG_TRACEBACK | (gdp.FLAG_JUMP_LATE if j % 2 else 0)
            p["tb_r"], p["tb_c"] = rl, gl
            p["genomeoffset"], p["chrhigh"], p["watsonp"], p["dynprogindex"] = 100, 60000, 1, 1
    arena = np.concatenate(chunks).astype(np.uint8)
    fails = parity.check_fill(ctx, ref, out, arena)
    assert not fails, "\n".join(fails)
    fails, _ = parity.check_traceback(ctx, ref, rest, out, arena)
    assert not fails, "\n".join(fails)


def test_golden_vectors(env, gdplib):
    """The committed golden vectors (recorded from the reference's compiled
    functions) reproduce on the GPU: final scores, traceback stats, and a
    digest of every record."""
    ctx, _, _ = env
    path = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
    z = np.load(path)
    pairs, arena = z["pairs"], z["arena"]
    gctx = gdp.Context(gdplib)
    gctx.set_genome(z["genome_blocks"], z["genome_alt"], int(z["genome_length"]))
    res, recs = gctx.align(pairs, arena)
    defined = z["defined"].astype(bool)
    assert np.array_equal(res["score"], z["score"])
    assert (res["status"][defined] == 0).all()
    stats = np.stack([res[k] for k in ("tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs")], 1)
    assert np.array_equal(stats[defined], z["stats"][defined])
    offs = np.concatenate([[0], np.cumsum(z["stats"][:, 5])])
    for i in np.nonzero(defined)[0]:
        r0 = int(res["rec_offset"][i])
        g = recs[r0:r0 + int(res["nrecs"][i])]
        assert g.tobytes() == z["recs"][offs[i]:offs[i + 1]].tobytes(), f"pair {i}"
    gctx.close()


def test_batch_determinism_and_launches(env, gdplib):
    """Two runs of the same batch give identical bytes, and every run launches
    this library's kernels (no host fallback exists)."""
    ctx, _, _ = env
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_SHORT, 77, GENOME['g'], 2000)
    before = ctx.launches()
    r1, c1 = ctx.align(pairs, arena)
    mid = ctx.launches()
    r2, c2 = ctx.align(pairs, arena)
    assert mid > before
    assert r1.tobytes() == r2.tobytes() and c1.tobytes() == c2.tobytes()


def test_rerun_long_pairs_on_lane_groups(env, gdplib):
    """With check_min_x, the 8-bit pass of long rerun pairs runs on lane
    groups and that of short ones one thread per pair, in one plan; both are
    bit-exact under the rerun contract."""
    ctx, ref, rest = env
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_SHORT, 33, GENOME['g'], 300)
    keep = ctx.get_param("check_min_x")
    ctx.set_param("check_min_x", 160)
    try:
        ctx.profile(True)
        ctx.profile_reset()
        fails = parity.check_fill(ctx, ref, pairs, arena)
        assert not fails, "\n".join(fails)
        fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
        assert not fails, "\n".join(fails)
        kernels = ctx.profile_read()
        ctx.profile(False)
    finally:
        ctx.set_param("check_min_x", keep)
    assert any("8bit-check" in k and k.startswith("fill_warp") for k in kernels), kernels
    assert any("8bit-check" in k and k.startswith("fill_thread") for k in kernels), kernels


def test_rerun_short_pairs_beside_16bit_pass(env):
    """Rerun pairs too short for any score to reach 127 run their 8-bit pass
    beside the 16-bit pass (no wait for the 16-bit maximum); the kept
    precision and every output follow the rerun contract bit for bit."""
    ctx, ref, rest = env
    pairs, arena = cases.random_cases(341, 300, precisions=(8,), min_len=1, max_len=42)
    pairs["flags"] |= gdp.FLAG_RERUN16
    ctx.profile(True)
    ctx.profile_reset()
    fails = parity.check_fill(ctx, ref, pairs, arena)
    assert not fails, "\n".join(fails)
    fails, _ = parity.check_traceback(ctx, ref, rest, pairs, arena)
    assert not fails, "\n".join(fails)
    kernels = ctx.profile_read()
    ctx.profile(False)
    assert any(k.endswith("8bit-check-early>") for k in kernels), kernels
