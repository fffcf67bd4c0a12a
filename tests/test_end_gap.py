"""Dynprog_end5_gap / Dynprog_end3_gap over a batch (gdp_end_gap_batch).

* CPU: the committed golden vectors of the reference's end-gap solvers
  (tests/golden/end_gap.npz) are reproduced by the restatement and by the
  reference library itself.
* CPU: the restated end gap (oracle.end_gap_restated: the host decisions,
  the endpoint scan and the post-processing in Python over the C
  restatement's fills and traceback) equals the reference's own
  Dynprog_end5_gap / Dynprog_end3_gap (compiled into oracle/_ref) on every
  gap: traceback score and counts, NULL lists, and the returned List
  record by record; with default and with user penalties.
* GPU: gdp_end_gap_batch equals the reference on the same gaps, with and
  without an alternate genome and with user penalties (Dynprog_end_setup);
  QUERYEND_NOGAPS and malformed gaps are rejected per gap; a record buffer
  that is too small cuts the batch at the first gap that does not fit.
"""
import os

import numpy as np
import pytest

import end_cases
import gdp
import oracle
import single_cases

GENOME_LEN = 1 << 16
MAXLOOKBACK, EXTRAQUERYGAP = 200, 40
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "end_gap.npz")


@pytest.fixture(scope="module")
def genome():
    return single_cases.genome_pair(78, GENOME_LEN)


@pytest.fixture(scope="module")
def ref_end(reference):
    r = oracle.ReferenceEndGap(reference, MAXLOOKBACK, EXTRAQUERYGAP)
    r.setup()
    return r


def _gaps(seed, n, ref_end, genome, **kw):
    return end_cases.end_gap_cases(seed, n, genome[0], ref_end.max_rlength, ref_end.max_glength, **kw)


def _check_same(stats_a, off_a, recs_a, stats_b, off_b, recs_b, what):
    bad = np.nonzero((stats_a[:, :7] != stats_b[:, :7]).any(axis=1))[0]
    assert bad.size == 0, f"{what}: stats differ at gaps {bad[:8].tolist()}: {stats_a[bad[:3]]} vs {stats_b[bad[:3]]}"
    for i in range(stats_a.shape[0]):
        k = int(stats_a[i, 5])
        a = recs_a[int(off_a[i]):int(off_a[i]) + k]
        b = recs_b[int(off_b[i]):int(off_b[i]) + k]
        assert np.array_equal(a, b), f"{what}: records of gap {i} differ"


def _golden():
    z = np.load(GOLDEN)
    return {k: z[k] for k in z.files}


def _device_stats(res, dpi):
    return np.stack([res["tb_score"], res["nmatches"], res["nmismatches"], res["nopens"], res["nindels"],
                     res["nrecs"], (res["nrecs"] == 0).astype(np.int32), dpi], axis=1)


def test_restatement_matches_golden(restatement):
    """The restated end gap reproduces the committed golden vectors of the
    reference's Dynprog_end5_gap / _end3_gap (tests/golden/make_golden_end.py)."""
    z = _golden()
    restatement.set_genome(z["genome_blocks"], z["genome_alt_blocks"], z["genome"].size)
    st, off, recs = oracle.end_gap_restated(restatement, z["gaps"], z["arena"], z["genome"], z["genome_alt"])
    _check_same(z["stats"], z["rec_offset"], z["recs"], st, off, recs, "golden")


def test_reference_matches_golden(reference, ref_end):
    z = _golden()
    reference.set_genome(z["genome_blocks"], z["genome_alt_blocks"], z["genome"].size)
    st, off, recs = ref_end.run(z["gaps"], z["arena"])
    _check_same(z["stats"], z["rec_offset"], z["recs"], st, off, recs, "reference vs golden")
    assert np.array_equal(st[:, 7], z["stats"][:, 7])


def test_restatement_matches_reference(reference, restatement, ref_end, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks, GENOME_LEN)
    restatement.set_genome(blocks, altblocks, GENOME_LEN)
    gaps, arena = _gaps(3, 500, ref_end, genome)
    st_r, off_r, rec_r = ref_end.run(gaps, arena)
    st_o, off_o, rec_o = oracle.end_gap_restated(restatement, gaps, arena, g, alt)
    _check_same(st_r, off_r, rec_r, st_o, off_o, rec_o, "restatement")
    # the mix reaches every branch: both ends, the three end alignments, 8-
    # and 16-bit fills, NULL results, cut lengths and segments off the chromosome
    rl = np.minimum(gaps["rlength"], ref_end.max_rlength)
    gl = np.minimum(gaps["glength"], ref_end.max_glength)
    early = (gaps["rlength"] <= 0) | (gaps["glength"] <= 0) | ((gaps["end"] == 5) & (gaps["goffset"] < 0))
    assert early.sum() >= 10 and (st_r[early, :7] == (0, 0, 0, 0, 0, 0, 1)).all()
    live = ~early & (gaps["require_pos_score_p"] == 0)
    assert set(np.unique(gaps["end"][live]).tolist()) == {3, 5}
    assert set(np.unique(gaps["endalign"][live]).tolist()) == {gdp.QUERYEND_GAP, gdp.QUERYEND_INDELS, gdp.BEST_LOCAL}
    assert (live & ((rl < 24) | (gl < 24))).sum() >= 50 and (live & (rl >= 24) & (gl >= 24)).sum() >= 100
    assert (live & (gaps["rlength"] > ref_end.max_rlength)).sum() >= 3
    assert (st_r[live, 5] > 0).sum() >= 300
    starred = [i for i in np.nonzero(live)[0]
               if (end_cases.end_segment(g, int(gaps["chroffset"][i]), int(gaps["chrhigh"][i]), int(gaps["goffset"][i]),
                                         int(gl[i]), bool(gaps["watsonp"][i]), int(gaps["end"][i])) == 42).any()]
    assert len(starred) >= 10
    # the reference advances dynprogindex away from zero once per gap that
    # passes its length checks
    dpi = gaps["dynprogindex"]
    assert np.array_equal(st_r[:, 7], np.where(early, dpi, dpi + np.sign(dpi)))


def test_restatement_user_penalties(reference, restatement, ref_end, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, None, GENOME_LEN)
    restatement.set_genome(blocks, None, GENOME_LEN)
    ref_end.setup(-12, -1, True)
    try:
        gaps, arena = _gaps(4, 200, ref_end, genome)
        st_r, off_r, rec_r = ref_end.run(gaps, arena)
        st_o, off_o, rec_o = oracle.end_gap_restated(restatement, gaps, arena, g, g, user=(-12, -1))
        _check_same(st_r, off_r, rec_r, st_o, off_o, rec_o, "user penalties")
    finally:
        ref_end.setup()


@pytest.mark.gpu
@pytest.mark.parametrize("alt_genome", [True, False])
def test_end_gap_batch_matches_reference(gdplib, reference, ref_end, genome, alt_genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks if alt_genome else None, GENOME_LEN)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altblocks if alt_genome else None, GENOME_LEN)
        gaps, arena = _gaps(11 + alt_genome, 3000, ref_end, genome)
        res, recs = ctx.end_gaps(gaps, arena)
        assert ctx.launches() > 0
    finally:
        ctx.close()
    st_r, off_r, rec_r = ref_end.run(gaps, arena)
    assert (res["status"] == 0).all(), np.unique(res["status"])
    _check_same(st_r, off_r, rec_r, _device_stats(res, st_r[:, 7]), res["rec_offset"], recs, "device")
    live = res["end_found"] > 0
    assert set(np.unique(res["precision"][live]).tolist()) == {8, 16}


@pytest.mark.gpu
def test_end_gap_batch_user_penalties(gdplib, reference, ref_end, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks, GENOME_LEN)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altblocks, GENOME_LEN)
        assert ctx.end_setup(-12, -1, True) == 0
        assert ctx.end_setup(-200, -1, True) == 3   # GDP_ERR_PARAM, the earlier setting stays
        gaps, arena = _gaps(21, 800, ref_end, genome)
        res, recs = ctx.end_gaps(gaps, arena)
    finally:
        ctx.close()
    ref_end.setup(-12, -1, True)
    try:
        st_r, off_r, rec_r = ref_end.run(gaps, arena)
    finally:
        ref_end.setup()
    _check_same(st_r, off_r, rec_r, _device_stats(res, st_r[:, 7]), res["rec_offset"], recs, "device, user penalties")


@pytest.mark.gpu
def test_end_gap_rejections_cut_and_empty_batch(gdplib, ref_end, genome):
    g, alt, blocks, altblocks = genome
    gaps, arena = _gaps(41, 300, ref_end, genome)
    bad = gaps.copy()
    bad["endalign"][0] = gdp.QUERYEND_NOGAPS
    bad["end"][1] = 4
    bad["genestrand"][2] = 7
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, None, GENOME_LEN)
        full, recs = ctx.end_gaps(gaps, arena)
        cut = int(recs.size // 2)
        part, recs2 = ctx.end_gaps(gaps, arena, max_recs=cut)
        rej, _ = ctx.end_gaps(bad, arena)
        empty = ctx.end_gaps(gaps[:0], arena)
    finally:
        ctx.close()
    assert (full["status"] == 0).all()
    ends = full["rec_offset"] + full["nrecs"]
    fits = ends <= cut
    first_out = int(np.argmin(fits)) if not fits.all() else gaps.size
    keys = ("status", "tb_score", "nmatches", "nmismatches", "nopens", "nindels", "nrecs", "rec_offset")
    assert all(np.array_equal(part[k][:first_out], full[k][:first_out]) for k in keys)
    late = np.arange(gaps.size) >= first_out
    had = late & (full["nrecs"] > 0)
    assert had.any() and (part["status"][had] == 7).all() and (part["nrecs"][late] == 0).all()   # GDP_ERR_RECS
    assert np.array_equal(recs2, recs[:recs2.size]) and recs2.size <= cut
    assert rej["status"][0] == 3 and rej["status"][1] == 3 and rej["nrecs"][:2].sum() == 0
    assert rej["status"][2] == 3 or full["nrecs"][2] == 0
    same = np.arange(gaps.size) >= 3
    assert all(np.array_equal(rej[k][same], full[k][same]) for k in ("status", "tb_score", "nrecs"))
    assert empty[0].size == 0 and empty[1].size == 0
