"""Dynprog_cdna_gap over a batch (gdp_cdna_gap_batch).

* CPU: the reference library reproduces the committed golden vectors of its
  own Dynprog_cdna_gap (tests/golden/cdna_gap.npz), and the seeded mix
  reaches the reference's branches (no pairs by length, gap holders, 8-bit
  and 16-bit fills, both tie rules, both strands).
* GPU: gdp_cdna_gap_batch equals the reference's Dynprog_cdna_gap on the
  same gaps, with and without an alternate genome: traceback score,
  incompletep, NULL lists and the returned List record by record; a record
  buffer that is too small cuts the batch at the first gap that does not
  fit; an empty batch returns nothing.
"""
import os

import numpy as np
import pytest

import cdna_cases
import gdp
import oracle
import single_cases

GENOME_LEN = 1 << 16
MAXLOOKBACK, EXTRAQUERYGAP = 200, 40
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cdna_gap.npz")


@pytest.fixture(scope="module")
def genome():
    return single_cases.genome_pair(79, GENOME_LEN)


@pytest.fixture(scope="module")
def ref_cdna(reference):
    return oracle.ReferenceCdnaGap(reference, MAXLOOKBACK, EXTRAQUERYGAP)


def _gaps(seed, n, ref_cdna, genome):
    return cdna_cases.cdna_gap_cases(seed, n, genome[0], ref_cdna.max_rlength, ref_cdna.max_glength)


def _check_same(stats_a, off_a, recs_a, stats_b, off_b, recs_b, what):
    bad = np.nonzero((stats_a[:, :7] != stats_b[:, :7]).any(axis=1))[0]
    assert bad.size == 0, f"{what}: stats differ at gaps {bad[:8].tolist()}: {stats_a[bad[:3]]} vs {stats_b[bad[:3]]}"
    for i in range(stats_a.shape[0]):
        k = int(stats_a[i, 5])
        a = recs_a[int(off_a[i]):int(off_a[i]) + k]
        b = recs_b[int(off_b[i]):int(off_b[i]) + k]
        assert np.array_equal(a, b), f"{what}: records of gap {i} differ"


def _device_stats(res, dpi):
    z = np.zeros(res.size, np.int32)
    return np.stack([res["tb_score"], res["end_found"], z, z, z, res["nrecs"],
                     (res["nrecs"] == 0).astype(np.int32), dpi], axis=1)


def test_reference_matches_golden(reference, ref_cdna):
    z = np.load(GOLDEN)
    reference.set_genome(z["genome_blocks"], z["genome_alt_blocks"], z["genome"].size)
    st, off, recs = ref_cdna.run(z["gaps"], z["arena"])
    _check_same(z["stats"], z["rec_offset"], z["recs"], st, off, recs, "reference vs golden")
    assert np.array_equal(st[:, 7], z["stats"][:, 7])


def test_cases_reach_the_branches(reference, ref_cdna, genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks, GENOME_LEN)
    gaps, arena = _gaps(5, 400, ref_cdna, genome)
    st, off, recs = ref_cdna.run(gaps, arena)
    short = gaps["glength"] <= 1
    over = (gaps["glength"] > ref_cdna.max_glength) | (gaps["rlengthL"] > ref_cdna.max_rlength)
    assert short.sum() >= 5 and over.sum() >= 5
    assert (st[short | over, 6] == 1).all()
    dpi = gaps["dynprogindex"]
    # the reference advances dynprogindex except when glength <= 1
    assert np.array_equal(st[:, 7], np.where(short, dpi, dpi + np.sign(dpi)))
    live = ~short & ~over
    assert (st[live, 1] == 1).sum() >= 200 and (st[live, 5] > 0).sum() >= 200
    q = np.where(gaps["defect_rate"] < 0.003, 41, np.where(gaps["defect_rate"] < 0.014, 63, 127))
    eight = (gaps["glength"] < q) | ((gaps["rlengthL"] < q) & (gaps["rlengthR"] <= q))
    assert (live & eight).sum() >= 50 and (live & ~eight).sum() >= 50
    assert (recs["comp"] == b"").sum() >= 200       # gap holders


@pytest.mark.gpu
@pytest.mark.parametrize("alt_genome", [True, False])
def test_cdna_gap_batch_matches_reference(gdplib, reference, ref_cdna, genome, alt_genome):
    g, alt, blocks, altblocks = genome
    reference.set_genome(blocks, altblocks if alt_genome else None, GENOME_LEN)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altblocks if alt_genome else None, GENOME_LEN)
        gaps, arena = _gaps(11 + alt_genome, 1500, ref_cdna, genome)
        res, recs = ctx.cdna_gaps(gaps, arena)
        assert ctx.launches() > 0
    finally:
        ctx.close()
    st_r, off_r, rec_r = ref_cdna.run(gaps, arena)
    assert (res["status"] == 0).all(), np.unique(res["status"], return_counts=True)
    _check_same(st_r, off_r, rec_r, _device_stats(res, st_r[:, 7]), res["rec_offset"], recs, "device")


@pytest.mark.gpu
def test_cdna_gap_record_cut_and_empty_batch(gdplib, ref_cdna, genome):
    g, alt, blocks, altblocks = genome
    gaps, arena = _gaps(41, 300, ref_cdna, genome)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, None, GENOME_LEN)
        full, recs = ctx.cdna_gaps(gaps, arena)
        cut = int(recs.size // 2)
        part, recs2 = ctx.cdna_gaps(gaps, arena, max_recs=cut)
        empty = ctx.cdna_gaps(gaps[:0], arena)
    finally:
        ctx.close()
    assert (full["status"] == 0).all()
    ends = full["rec_offset"] + full["nrecs"]
    fits = ends <= cut
    first_out = int(np.argmin(fits)) if not fits.all() else gaps.size
    keys = ("status", "tb_score", "nrecs", "rec_offset", "end_found")
    assert all(np.array_equal(part[k][:first_out], full[k][:first_out]) for k in keys)
    late = np.arange(gaps.size) >= first_out
    had = late & (full["nrecs"] > 0)
    assert had.any() and (part["status"][had] == 7).all() and (part["nrecs"][late] == 0).all()
    assert np.array_equal(recs2, recs[:recs2.size]) and recs2.size <= cut
    assert empty[0].size == 0 and empty[1].size == 0
