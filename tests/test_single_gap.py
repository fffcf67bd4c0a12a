"""Dynprog_single_gap over a batch (gdp_single_gap_batch).

* CPU: the committed golden vectors of the reference's Dynprog_single_gap
  (tests/golden/single_gap.npz) are reproduced by the restatement, and by
  the reference library itself.
* CPU: the restated single gap (oracle.single_gap_restated: the host
  decisions and single_gap_simple in Python, the fill and traceback of the
  C restatement) equals the reference's own Dynprog_single_gap
  (src/dynprog_single.c:428-675, compiled into oracle/_ref) on every gap:
  traceback score and counts, NULL lists, and the returned List record by
  record.
* GPU: gdp_single_gap_batch equals the reference's Dynprog_single_gap on
  the same gaps, with and without an alternate genome and with user
  penalties (Dynprog_single_setup).
* GPU: the stage-3 batching adapter (gdp_gap_queue) called one gap at a
  time from eight threads gives each gap the result and records of the
  batch call, and batches the threads' gaps together.
"""
import os
import threading

import numpy as np
import pytest

import gdp
import oracle
import single_cases

GENOME_LEN = 1 << 16
MAXLOOKBACK, EXTRAQUERYGAP = 200, 40


@pytest.fixture(scope="module")
def genome():
    return single_cases.genome_pair(77, GENOME_LEN)


@pytest.fixture(scope="module")
def ref_single(reference):
    return oracle.ReferenceSingleGap(reference, MAXLOOKBACK, EXTRAQUERYGAP)


def _gaps(seed, n, ref_single, genome):
    return single_cases.single_gap_cases(seed, n, genome[0], ref_single.max_rlength, ref_single.max_glength)


def _check_same(stats_a, off_a, recs_a, stats_b, off_b, recs_b, what):
    bad = np.nonzero((stats_a[:, :7] != stats_b[:, :7]).any(axis=1))[0]
    assert bad.size == 0, f"{what}: stats differ at gaps {bad[:8].tolist()}: {stats_a[bad[:3]]} vs {stats_b[bad[:3]]}"
    for i in range(stats_a.shape[0]):
        k = int(stats_a[i, 5])
        a = recs_a[int(off_a[i]):int(off_a[i]) + k]
        b = recs_b[int(off_b[i]):int(off_b[i]) + k]
        assert np.array_equal(a, b), f"{what}: records of gap {i} differ"


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "single_gap.npz")


def _golden():
    z = np.load(GOLDEN)
    return {k: z[k] for k in z.files}


def test_restatement_matches_golden(restatement):
    """The restated single gap reproduces the committed golden vectors of the
    reference's Dynprog_single_gap (tests/golden/make_golden_single.py)."""
    z = _golden()
    restatement.set_genome(z["genome_blocks"], z["genome_alt_blocks"], z["genome"].size)
    st, off, recs = oracle.single_gap_restated(restatement, z["gaps"], z["arena"], z["genome"], z["genome_alt"])
    _check_same(z["stats"], z["rec_offset"], z["recs"], st, off, recs, "golden")


def test_reference_matches_golden(reference, ref_single):
    z = _golden()
    reference.set_genome(z["genome_blocks"], z["genome_alt_blocks"], z["genome"].size)
    ref_single.setup()
    st, off, recs = ref_single.run(z["gaps"], z["arena"])
    _check_same(z["stats"], z["rec_offset"], z["recs"], st, off, recs, "reference vs golden")
    assert np.array_equal(st[:, 7], z["stats"][:, 7])


def test_restatement_matches_reference(reference, restatement, ref_single, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks, GENOME_LEN)
    restatement.set_genome(blocks, altblocks, GENOME_LEN)
    ref_single.setup()
    gaps, arena = _gaps(3, 400, ref_single, genome)
    st_r, off_r, rec_r = ref_single.run(gaps, arena)
    st_o, off_o, rec_o = oracle.single_gap_restated(restatement, gaps, arena, g, alt)
    _check_same(st_r, off_r, rec_r, st_o, off_o, rec_o, "restatement")
    # every branch of the single gap was taken
    nulls = st_r[:, 6] == 1
    simple = (gaps["rlength"] == gaps["glength"]) & ~nulls & (st_r[:, 3] == 0) & (st_r[:, 2] <= 1)
    assert nulls.sum() >= 5 and simple.sum() >= 50 and (~nulls & ~simple).sum() >= 100
    badlen = ((gaps["rlength"] <= 0) | (gaps["glength"] <= 0) | (gaps["rlength"] > ref_single.max_rlength)
              | (gaps["glength"] > ref_single.max_glength))
    assert badlen.sum() >= 5 and (st_r[badlen, 0] == -32768).all() and (st_r[badlen, 6] == 1).all()
    # the reference advances dynprogindex away from zero by one per gap
    dpi = gaps["dynprogindex"]
    assert np.array_equal(st_r[:, 7], dpi + np.sign(dpi))


def test_restatement_user_penalties(reference, restatement, ref_single, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, None, GENOME_LEN)
    restatement.set_genome(blocks, None, GENOME_LEN)
    ref_single.setup(-11, -1, True)
    try:
        gaps, arena = _gaps(4, 150, ref_single, genome)
        st_r, off_r, rec_r = ref_single.run(gaps, arena)
        st_o, off_o, rec_o = oracle.single_gap_restated(restatement, gaps, arena, g, g, user=(-11, -1))
        _check_same(st_r, off_r, rec_r, st_o, off_o, rec_o, "user penalties")
    finally:
        ref_single.setup()


@pytest.mark.gpu
@pytest.mark.parametrize("alt_genome", [True, False])
def test_single_gap_batch_matches_reference(gdplib, reference, ref_single, genome, alt_genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks if alt_genome else None, GENOME_LEN)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altblocks if alt_genome else None, GENOME_LEN)
        gaps, arena = _gaps(11 + alt_genome, 3000, ref_single, genome)
        res, path, recs = ctx.single_gaps(gaps, arena)
        assert ctx.launches() > 0
    finally:
        ctx.close()
    st_r, off_r, rec_r = ref_single.run(gaps, arena)
    assert (res["status"] == 0).all(), np.unique(res["status"])
    st_d = np.stack([res["tb_score"], res["nmatches"], res["nmismatches"], res["nopens"], res["nindels"],
                     res["nrecs"], (res["nrecs"] == 0).astype(np.int32), st_r[:, 7]], axis=1)
    _check_same(st_r, off_r, rec_r, st_d, res["rec_offset"], recs, "device")
    assert (path == gdp.SINGLE_SIMPLE).sum() > 300 and (path == gdp.SINGLE_DP).sum() > 1000
    dp = path == gdp.SINGLE_DP
    assert set(np.unique(res["precision"][dp]).tolist()) == {8, 16}


@pytest.mark.gpu
def test_single_gap_batch_user_penalties(gdplib, reference, ref_single, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks, GENOME_LEN)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altblocks, GENOME_LEN)
        assert ctx.single_setup(-11, -1, True) == 0
        assert ctx.single_setup(0, 0, False, homopolymerp=True) == 3   # GDP_ERR_PARAM
        gaps, arena = _gaps(21, 800, ref_single, genome)
        res, path, recs = ctx.single_gaps(gaps, arena)
    finally:
        ctx.close()
    ref_single.setup(-11, -1, True)
    try:
        st_r, off_r, rec_r = ref_single.run(gaps, arena)
    finally:
        ref_single.setup()
    st_d = np.stack([res["tb_score"], res["nmatches"], res["nmismatches"], res["nopens"], res["nindels"],
                     res["nrecs"], (res["nrecs"] == 0).astype(np.int32), st_r[:, 7]], axis=1)
    _check_same(st_r, off_r, rec_r, st_d, res["rec_offset"], recs, "device, user penalties")


@pytest.mark.gpu
def test_gap_queue_from_threads_equals_batch(gdplib, genome):
    g, alt, blocks, altblocks = genome
    gaps, arena = single_cases.single_gap_cases(31, 1600, g, 500, 2000)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altblocks, GENOME_LEN)
        res_b, path_b, recs_b = ctx.single_gaps(gaps, arena)
    finally:
        ctx.close()
    q = gdp.GapQueue(gdplib, blocks, altblocks, GENOME_LEN, max_batch=256, max_wait_us=500)
    out = [None] * gaps.size
    errors = []

    def worker(t):
        try:
            for i in range(t, gaps.size, 8):
                x = gaps[i]
                rl = max(int(x["rlength"]), 0)
                rs = np.ascontiguousarray(arena[int(x["rseq"]):int(x["rseq"]) + rl])
                ru = np.ascontiguousarray(arena[int(x["rseq_uc"]):int(x["rseq_uc"]) + rl])
                out[i] = q.align(x, rs, ru)
        except Exception as e:   # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    stats = q.stats()
    q.close()
    assert not errors, errors
    keys = ("status", "score", "precision", "tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs")
    for i in range(gaps.size):
        r, p, recs = out[i]
        assert all(r[k] == res_b[i][k] for k in keys), (i, r, res_b[i])
        assert p == path_b[i]
        o = int(res_b["rec_offset"][i])
        assert np.array_equal(recs, recs_b[o:o + int(res_b["nrecs"][i])]), i
    assert stats["gaps"] == gaps.size and stats["batches"] < gaps.size and stats["max_batch"] > 1


@pytest.mark.gpu
def test_single_gap_record_cut_and_empty_batch(gdplib, genome):
    g, alt, blocks, altblocks = genome
    gaps, arena = single_cases.single_gap_cases(41, 300, g, 500, 2000)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, None, GENOME_LEN)
        full, path, recs = ctx.single_gaps(gaps, arena)
        cut = int(recs.size // 2)
        part, path2, recs2 = ctx.single_gaps(gaps, arena, max_recs=cut)
        empty = ctx.single_gaps(gaps[:0], arena)
    finally:
        ctx.close()
    assert np.array_equal(path, path2)
    ends = full["rec_offset"] + full["nrecs"]
    fits = ends <= cut
    first_out = int(np.argmin(fits)) if not fits.all() else gaps.size
    assert fits[:first_out].all() and not fits[first_out:].any()
    keys = ("status", "tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs", "rec_offset")
    assert all(np.array_equal(part[k][:first_out], full[k][:first_out]) for k in keys)
    late = np.arange(gaps.size) >= first_out
    had = late & (full["nrecs"] > 0)
    assert (part["status"][had] == 7).all() and (part["nrecs"][late] == 0).all()   # GDP_ERR_RECS
    assert np.array_equal(part["status"][late & ~had], full["status"][late & ~had])
    assert np.array_equal(recs2, recs[:recs2.size]) and recs2.size <= cut
    assert empty[0].size == 0 and empty[2].size == 0
