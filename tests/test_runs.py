"""The record-run codec (gdp_runs_encode / gdp_runs_decode, rec_runs.h):
gdp_align_batch brings traceback records to the host as runs and rebuilds
them there, so the rebuilt bytes must equal the records the traceback
wrote, whatever the pair.

* CPU: records the C restatement's traceback writes for random pairs (every
  variant, both precisions, revp, both tie rules, '*' genome characters,
  alternate genomes, IUPAC and lower-case query characters) go through the
  codec and come back byte for byte; short-read records take about a byte
  each; GDP_FLAG_GWINDOW pairs travel whole; a cut or altered stream is
  rejected or rebuilds other bytes, never reads past its end.
* GPU: gdp_align_batch gives the same records with the run transport on
  and off, and copies far fewer bytes to the host with it on.
"""
import numpy as np
import pytest

import cases
import gdp


def _traced(restatement, seed, n, **kw):
    pairs, arena = cases.random_cases(seed, n, **kw)
    pairs["flags"] |= gdp.FLAG_TRACEBACK
    pairs["flags"] &= ~np.int8(gdp.FLAG_RERUN16)
    pairs["tb_r"], pairs["tb_c"] = pairs["rlength"], pairs["glength"]
    out = []
    for i in range(n):
        r = restatement.align(pairs, i, arena, want_matrix=False)
        out.append(np.frombuffer(r["recs"].tobytes(), dtype=gdp.REC_DTYPE).copy())
    return pairs, arena, out


@pytest.fixture(scope="module")
def traced(restatement):
    g, blocks, altb = cases.genome(23, length=1 << 16)
    restatement.set_genome(blocks, altb, g.size)
    return _traced(restatement, 611, 400)


def test_runs_round_trip_every_pair(gdplib, traced):
    pairs, arena, recs = traced
    total_recs = total_bytes = 0
    for i, r in enumerate(recs):
        s = gdp.runs_encode(gdplib, pairs[i], arena, r)
        back = gdp.runs_decode(gdplib, pairs[i], arena, s, r.size)
        assert back is not None, i
        assert back.tobytes() == r.tobytes(), i
        total_recs += r.size
        total_bytes += s.size
    assert total_recs > 10000
    assert total_bytes < 0.45 * total_recs * gdp.REC_DTYPE.itemsize


def test_runs_short_reads_take_about_a_byte_per_record(gdplib, restatement):
    g, blocks, altb = cases.genome(29, length=1 << 16)
    restatement.set_genome(blocks, None, g.size)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_SHORT, 7, g, 300)
    pairs["flags"] &= ~np.int8(gdp.FLAG_RERUN16)
    pairs["precision"] = 16
    nrec = nbytes = 0
    for i in range(pairs.size):
        r = restatement.align(pairs, i, arena, want_matrix=False)
        rec = np.frombuffer(r["recs"].tobytes(), dtype=gdp.REC_DTYPE).copy()
        s = gdp.runs_encode(gdplib, pairs[i], arena, rec)
        assert gdp.runs_decode(gdplib, pairs[i], arena, s, rec.size).tobytes() == rec.tobytes()
        nrec += rec.size
        nbytes += s.size
    assert nrec > 30000 and nbytes < 0.2 * nrec * gdp.REC_DTYPE.itemsize


def test_runs_window_pairs_travel_whole(gdplib, traced):
    pairs, arena, recs = traced
    i = next(k for k, r in enumerate(recs) if r.size > 5)
    p = pairs[i].copy()
    p["flags"] |= gdp.FLAG_GWINDOW
    s = gdp.runs_encode(gdplib, p, arena, recs[i])
    assert s.size == 13 * recs[i].size
    assert gdp.runs_decode(gdplib, p, arena, s, recs[i].size).tobytes() == recs[i].tobytes()


def test_runs_reject_cut_and_altered_streams(gdplib, traced):
    pairs, arena, recs = traced
    checked = 0
    for i, r in enumerate(recs):
        if r.size < 20:
            continue
        s = gdp.runs_encode(gdplib, pairs[i], arena, r)
        assert gdp.runs_decode(gdplib, pairs[i], arena, s[:-1], r.size) is None      # cut
        assert gdp.runs_decode(gdplib, pairs[i], arena, s, r.size + 1) is None       # records missing
        longer = np.concatenate([s, np.zeros(1, np.uint8)])
        assert gdp.runs_decode(gdplib, pairs[i], arena, longer, r.size) is None      # bytes left over
        checked += 1
    assert checked > 50


@pytest.mark.gpu
def test_align_batch_records_same_with_and_without_runs(gdplib):
    g, blocks, altb = cases.genome(31, length=1 << 18)
    pairs, arena = cases.random_cases(31, 3000, genome_len=1 << 18)
    short, sarena = gdp.make_pairs(gdplib, gdp.WL_SHORT, 8, g, 20000)
    ctx = gdp.Context(gdplib)
    try:
        ctx.set_genome(blocks, altb, g.size)
        out = {}
        for runs in (1, 2, 0):
            ctx.set_param("record_runs", runs)
            ra, reca = ctx.align(pairs, arena)
            rb, recb = ctx.align(short, sarena)
            out[runs] = (ra, reca, rb, recb, ctx.get_param("last_d2h_bytes"))
    finally:
        ctx.close()
    off = out[0]
    for mode in (1, 2):
        on = out[mode]
        assert np.array_equal(on[0], off[0]) and on[1].tobytes() == off[1].tobytes(), mode
        assert np.array_equal(on[2], off[2]) and on[3].tobytes() == off[3].tobytes(), mode
    assert off[3].size > 1_000_000
    # the short batch (the last call) copied far fewer bytes with runs
    assert out[1][4] < 0.35 * off[4]
