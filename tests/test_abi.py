"""C-ABI checks that need no GPU: libgdp.so loads, exports every function
include/gdp.h and include/gdp_dynprog_simd.h declare, and its host-side
helpers behave."""
import os
import re
import subprocess

import numpy as np

import gdp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(gdp_[a-z0-9_]+|Dynprog_[A-Za-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def _exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_library_exports_every_declared_symbol(gdplib):
    exported = _exported(gdp.LIB_PATH)
    headers = sorted(h for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h"))
    assert "gdp.h" in headers and "gdp_dynprog_simd.h" in headers
    declared = [n for h in headers for n in _declared(h)]
    assert sum(n.startswith("Dynprog_") for n in declared) == 12
    missing = [n for n in declared if n not in exported]
    assert not missing, missing


def test_version(gdplib):
    assert gdplib.gdp_version().decode().startswith("gdp-b200")


def test_workload_generator_is_seeded(gdplib):
    g, blocks = gdp.make_genome(gdplib, 5, 1 << 16)
    p1, a1 = gdp.make_pairs(gdplib, gdp.WL_SHORT, 3, g, 200)
    p2, a2 = gdp.make_pairs(gdplib, gdp.WL_SHORT, 3, g, 200)
    assert p1.tobytes() == p2.tobytes() and a1.tobytes() == a2.tobytes()
    assert ((p1["rlength"] >= 75) & (p1["rlength"] <= 300)).all()
    assert ((p1["lband"] >= 3) & (p1["lband"] <= 30)).all()
    d = p1["glength"] - p1["rlength"]
    assert ((d >= -p1["lband"]) & (d <= p1["uband"])).all()


def test_cell_counts_agree(gdplib):
    g, _ = gdp.make_genome(gdplib, 6, 1 << 16)
    for kind in (gdp.WL_FIXED, gdp.WL_SHORT, gdp.WL_CDNA):
        pairs, _ = gdp.make_pairs(gdplib, kind, 4, g, 20)
        assert np.array_equal(gdp.pair_cells(gdplib, pairs), gdp.band_cells(pairs))
    pairs, _ = gdp.make_pairs(gdplib, gdp.WL_FIXED, 4, g, 3)
    assert (gdp.pair_cells(gdplib, pairs) == 3095).all()   # 150 x 160, lband = uband = 10


def test_genomecomp_encoder_matches_tests_encoder(gdplib):
    import cases
    g = np.frombuffer(b"ACGTNacgtnAAAACCCCGGGGTTTTNNNNACGTACGTACGTACGTACGT", np.uint8)
    blocks = np.zeros(3 * ((g.size + 31) // 32), np.uint32)
    gdplib.gdp_workload_genomecomp(gdp._ptr(g), g.size, gdp._ptr(blocks))
    assert np.array_equal(blocks, cases.encode_genomecomp(g))
