"""The oracle is pinned before it is trusted (CPU only).

* The restatement (oracle/gdp_oracle.c) reproduces the committed golden
  vectors, which were recorded from the reference's own compiled functions
  (tests/golden/make_golden.py): final scores, traceback scores and counts,
  every Pair record, and a digest of the in-band scores and directions.
* Where the reference library (oracle/_ref, built from the reference
  sources) is present, the restatement also matches it live on fresh
  seeded cases, and both build identical substitution tables.
* libgdp's own host-built tables equal the reference's for every mode.
"""
import ctypes
import hashlib
import os

import numpy as np
import pytest

import cases
import gdp
import oracle as orc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def _digest(out, p):
    m = orc.domain_mask(int(p["variant"]), int(p["rlength"]), int(p["glength"]),
                        int(p["lband"]), int(p["uband"])).ravel()
    h = hashlib.sha1()
    for k in ("H", "dN", "dE", "dF"):
        h.update(np.ascontiguousarray(out[k][m]).tobytes())
    return np.frombuffer(h.digest(), np.uint8)


def _golden_precision(pairs, i, o8, restatement, arena):
    p = pairs[i]
    if not (p["flags"] & gdp.FLAG_RERUN16):
        return int(p["precision"])
    m = orc.domain_mask(int(p["variant"]), int(p["rlength"]), int(p["glength"]),
                        int(p["lband"]), int(p["uband"])).ravel()
    if (o8["H"][m] >= 127).any() or o8["score"] <= -98:
        return 16
    q = pairs[i:i + 1].copy()
    q["precision"] = 8
    restatement.lib.orc_last_tb_stale.restype = ctypes.c_int
    restatement.align(q, 0, arena, want_matrix=False)
    return 16 if restatement.lib.orc_last_tb_stale() else 8


def test_restatement_matches_golden(restatement):
    z = np.load(GOLDEN)
    pairs, arena = z["pairs"], z["arena"]
    restatement.set_genome(z["genome_blocks"], z["genome_alt"], int(z["genome_length"]))
    offs = np.concatenate([[0], np.cumsum(z["stats"][:, 5])])
    for i in range(pairs.size):
        q = pairs[i:i + 1].copy()
        if q["flags"][0] & gdp.FLAG_RERUN16:
            q["precision"] = _golden_precision(pairs, i, restatement.align(q.copy(), 0, arena),
                                               restatement, arena)
        out = restatement.align(q, 0, arena)
        assert out["score"] == z["score"][i], i
        assert np.array_equal(_digest(out, q[0]), z["fill_digest"][i]), i
        if z["defined"][i]:
            assert np.array_equal(out["stats"], z["stats"][i]), i
            assert out["recs"].tobytes() == z["recs"][offs[i]:offs[i + 1]].tobytes(), i


@pytest.mark.parametrize("seed", [31, 32])
def test_restatement_matches_reference_live(reference, restatement, seed):
    restatement.lib.orc_last_tb_stale.restype = ctypes.c_int
    g, blocks, altb = cases.genome(seed, length=1 << 17)
    reference.set_genome(blocks, altb, g.size)
    restatement.set_genome(blocks, altb, g.size)
    pairs, arena = cases.random_cases(seed, 300)
    for i in range(pairs.size):
        a = reference.align(pairs, i, arena)
        b = restatement.align(pairs, i, arena)
        p = pairs[i]
        m = orc.domain_mask(int(p["variant"]), int(p["rlength"]), int(p["glength"]),
                            int(p["lband"]), int(p["uband"])).ravel()
        for k in ("H", "dN", "dE", "dF"):
            assert np.array_equal(a[k][m], b[k][m]), (i, k)
        assert a["score"] == b["score"], i
        if not restatement.lib.orc_last_tb_stale():
            assert np.array_equal(a["stats"], b["stats"]), i
            assert a["recs"].tobytes() == b["recs"].tobytes(), i


@pytest.mark.parametrize("mode", range(7))
def test_tables_match_reference(reference, restatement, gdplib, mode):
    reference.init(mode)
    restatement.init(mode)
    pd, cons, nt = gdp.tables(gdplib, mode)
    probe = list(range(128))
    rng = np.random.default_rng(mode)
    for mt in range(4):
        for c1 in probe:
            for c2 in rng.choice(128, 24, replace=False).tolist() + [ord("A"), ord("N"), ord("z"), 4]:
                v = reference.pairdistance(mt, c1, c2)
                assert pd[mt, c1, c2] == v, (mode, mt, c1, c2)
                assert restatement.pairdistance(mt, c1, c2) == v
    strands = [0] if mode in (0, 1, 3, 5) else [1, 2]
    for gs in strands:
        for c1 in probe:
            for c2 in probe:
                v = reference.consistent(gs, c1, c2)
                assert cons[gs, c1, c2] == v, (mode, gs, c1, c2)
    reference.init(0)
    restatement.init(0)


def test_product_tables_standard_shape(gdplib):
    """Spot values of Dynprog_init's tables (src/dynprog.c:1069-1140) in
    libgdp's own tables, checkable without the reference sources."""
    pd, cons, nt = gdp.tables(gdplib, 0)
    A, C, G, T, N = (ord(c) for c in "ACGTN")
    assert pd[0, A, A] == 3 and pd[0, A, C] == -3 and pd[1, A, C] == -2
    assert pd[2, A, C] == -1 and pd[3, A, C] == -5
    assert pd[0, ord("R"), A] == 1 and pd[0, N, N] == 3 and pd[0, ord("a"), A] == 3
    assert pd[0, A, ord("z")] == 0 and pd[0, ord("*"), A] == 0
    assert nt[A] == 0 and nt[ord("t")] == 3 and nt[N] == 4 and nt[ord("*")] == 4
    assert cons[0, ord("R"), G] == 1 and cons[0, A, C] == 0


def test_kept_precision_and_cpu_bench(restatement, gdplib):
    """The batched kept-precision resolver (used to time the CPU baselines)
    agrees with the per-pair rerun rule, and the reference and the
    restatement timed at those precisions give the same score checksum."""
    genome, blocks = gdp.make_genome(gdplib, 93, 1 << 20)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_SHORT, 94, genome, 400)
    restatement.set_genome(blocks, None, genome.size)
    kept = restatement.kept_precision(pairs, arena, 4)
    assert set(np.unique(kept)) <= {8, 16}
    for i in range(0, pairs.size, 7):
        q = pairs[i:i + 1].copy()
        q["precision"] = 8
        q["flags"] = q["flags"] & ~gdp.FLAG_RERUN16
        o8 = restatement.align(q.copy(), 0, arena)
        assert kept[i] == _golden_precision(pairs, i, o8, restatement, arena), i
    _, cs = restatement.bench(pairs, arena, 3, kept)
    if orc.reference_available():
        ref = orc.reference()
        ref.set_genome(blocks, None, genome.size)
        _, cs_ref = ref.bench(pairs, arena, 3, kept)
        assert cs_ref == cs


def test_outputs_and_record_digests(restatement, gdplib):
    """The per-pair outputs the benchmark's parity sample compares: the
    multi-threaded runs of the reference and of the restatement give the
    same final score, traceback totals and record digest per pair, and the
    digest equals gdp.record_digests over the records of a one-pair run (the
    digest the benchmark computes for the device's records)."""
    genome, blocks = gdp.make_genome(gdplib, 95, 1 << 20)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_MIX, 96, genome, 60)
    restatement.set_genome(blocks, None, genome.size)
    kept = restatement.kept_precision(pairs, arena, 4)
    _, out = restatement.outputs(pairs, arena, 3, kept)
    for i in range(pairs.size):
        q = pairs[i:i + 1].copy()
        q["precision"] = kept[i]
        q["flags"] = q["flags"] & ~gdp.FLAG_RERUN16
        o = restatement.align(q, 0, arena, want_matrix=False)
        assert out[i, 0] == o["score"], i
        if q["flags"][0] & gdp.FLAG_TRACEBACK:
            assert list(out[i, 1:7]) == list(o["stats"]), i
            dig = gdp.record_digests(o["recs"], [0], [o["recs"].size])[0]
            assert np.uint32(out[i, 7]) == dig, i
    assert (pairs["variant"] == gdp.LOWER).any() and (pairs["variant"] == gdp.UPPER).any()
    if orc.reference_available():
        ref = orc.reference()
        ref.set_genome(blocks, None, genome.size)
        _, out_ref = ref.outputs(pairs, arena, 3, kept)
        assert np.array_equal(out_ref, out)


def test_workload_tie_rules_and_cdna_halves(gdplib):
    """The seeded workloads alternate the tie rule by draw, and every cDNA
    gap is an upper fill with a traceback followed by the lower fill of the
    same sequences (lband 14, no traceback); the standalone generator
    library gives the same pairs as libgdp.so."""
    genome, _ = gdp.make_genome(gdplib, 97, 1 << 20)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_CDNA, 98, genome, 40)
    up, lo = pairs[0::2], pairs[1::2]
    assert (up["variant"] == gdp.UPPER).all() and (lo["variant"] == gdp.LOWER).all()
    assert (lo["lband"] == 14).all() and (lo["uband"] == 0).all()
    assert (up["flags"] & gdp.FLAG_TRACEBACK).all() and not (lo["flags"] & gdp.FLAG_TRACEBACK).any()
    for k in ("rseq", "gseq", "rlength", "glength"):
        assert np.array_equal(up[k], lo[k])
    late = (up["flags"] & gdp.FLAG_JUMP_LATE) != 0
    assert late[0::2].all() and not late[1::2].any()
    short, _ = gdp.make_pairs(gdplib, gdp.WL_SHORT, 99, genome, 100)
    assert ((short["flags"] & gdp.FLAG_JUMP_LATE) != 0).sum() == 50
    wl = gdp.load_workload()
    g2, _ = gdp.make_genome(wl, 97, 1 << 20)
    p2, a2 = gdp.make_pairs(wl, gdp.WL_CDNA, 98, g2, 40)
    assert p2.tobytes() == pairs.tobytes() and a2.tobytes() == arena.tobytes()
