"""One batch over several contexts (gdp_align_batch_multi).

The batch splits into contiguous shards, one per context (one per GPU in a
multi-GPU node; here several contexts share the one GPU, which exercises the
same sharding, rebased arenas and record placement).  Every pair's results
and Pair records must equal those of the same batch through one context, and
a sample of them the reference's.
"""
import ctypes

import numpy as np
import pytest

import gdp
import parity

FIELDS = ("status", "score", "precision", "rerun", "tb_score", "nmatches", "nmismatches", "nopens", "nindels",
          "nrecs")


def _batch(lib, genome):
    """Mixed pairs (short reads, long reads, cDNA gaps) followed by a second
    arena-ordered draw of short reads: shards then cut through both."""
    a, arena_a = gdp.make_pairs(lib, gdp.WL_MIX, 71, genome, 1500)
    b, arena_b = gdp.make_pairs(lib, gdp.WL_SHORT, 72, genome, 3000)
    b = b.copy()
    for f in ("rseq", "rseq_uc", "gseq", "gseq_alt"):
        b[f] += arena_a.size
    return np.concatenate([a, b]), np.concatenate([arena_a, arena_b])


@pytest.mark.gpu
@pytest.mark.parametrize("nctx", [1, 2, 3])
def test_multi_equals_one_context(gdplib, reference, restatement, nctx):
    genome, blocks = gdp.make_genome(gdplib, 2027, 1 << 22)
    pairs, arena = _batch(gdplib, genome)
    one = gdp.Context(gdplib, device=0)
    one.set_genome(blocks, None, genome.size)
    res1, recs1 = one.align(pairs, arena)
    one.close()
    ctxs = []
    for _ in range(nctx):
        c = gdp.Context(gdplib, device=0)
        c.set_genome(blocks, None, genome.size)
        ctxs.append(c)
    try:
        resm, recsm = gdp.align_multi(gdplib, ctxs, pairs, arena)
    finally:
        for c in ctxs:
            c.close()
    assert (res1["status"] == 0).all()
    for f in FIELDS:
        assert np.array_equal(res1[f], resm[f]), f
    for i in range(pairs.size):
        n = int(res1["nrecs"][i])
        o1, om = int(res1["rec_offset"][i]), int(resm["rec_offset"][i])
        assert recs1[o1:o1 + n].tobytes() == recsm[om:om + n].tobytes(), i
    # a sample against the reference's own fill and traceback, at the
    # precision the rerun contract keeps
    reference.set_genome(blocks, None, genome.size)
    restatement.set_genome(blocks, None, genome.size)
    for i in range(0, pairs.size, 97):
        prec = parity.expected_precision(reference, pairs, i, arena, restatement)
        assert int(resm["precision"][i]) == prec, i
        o = reference.align(parity._as_precision(pairs, i, prec), 0, arena, want_matrix=False)
        assert int(resm["score"][i]) == o["score"], i
        om, n = int(resm["rec_offset"][i]), int(resm["nrecs"][i])
        assert recsm[om:om + n].tobytes() == o["recs"].tobytes(), i


@pytest.mark.gpu
def test_multi_rejects_a_short_record_buffer(gdplib):
    genome, blocks = gdp.make_genome(gdplib, 2028, 1 << 20)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_FIXED, 73, genome, 64)
    ctxs = [gdp.Context(gdplib, device=0) for _ in range(2)]
    try:
        for c in ctxs:
            c.set_genome(blocks, None, genome.size)
        with pytest.raises(RuntimeError, match="ERR_RECS"):
            gdp.align_multi(gdplib, ctxs, pairs, arena, max_recs=100)
    finally:
        for c in ctxs:
            c.close()


def test_multi_rejects_bad_arguments(gdplib):
    """Argument checks come before any CUDA call (no GPU needed)."""
    used = ctypes.c_int64(5)
    assert gdplib.gdp_align_batch_multi(None, 0, None, 0, None, 0, None, None, 0, ctypes.byref(used)) == 3
    assert used.value == 0
    hs = (ctypes.c_void_p * 2)(None, None)
    assert gdplib.gdp_align_batch_multi(hs, 2, None, 0, None, 0, None, None, 0, ctypes.byref(used)) == 3
