"""The reference-signature entry points (include/gdp_dynprog_simd.h).

GPU tests run GMAP's own host code (oracle/_ref/libgmapenv.so: the
reference's dynprog.c, pairpool.c, list.c, mem.c and except.c with
src/dynprog_simd.c left out) on top of libgdp.so in a child process
(tests/dropin_driver.py) and require its fills and tracebacks to equal the
reference's bit for bit.  The CPU test checks the declarations against the
reference's header where the reference tree is available.
"""
import os
import re
import subprocess
import sys

import pytest

import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "dropin_driver.py")


def _ref_header():
    """src/dynprog_simd.h of the reference: under GDP_REFSRC, else under the
    directory oracle/Makefile compiled the reference from (recorded in
    oracle/_ref/refsrc.txt); None when neither is present."""
    src = os.environ.get("GDP_REFSRC")
    if not src:
        rec = os.path.join(ROOT, "oracle", "_ref", "refsrc.txt")
        if os.path.exists(rec):
            src = open(rec).read().strip()
    path = os.path.join(src, "dynprog_simd.h") if src else None
    return path if path and os.path.exists(path) else None


def _run(*args):
    if not (orc.reference_available() and orc.gmap_environment_available()):
        pytest.skip("oracle/_ref (reference and GMAP environment) not built")
    out = subprocess.run([sys.executable, DRIVER, *map(str, args)], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    return out.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [11, 12])
def test_dropin_random_cases(seed):
    """All six fills and six tracebacks, both tie rules, revp, IUPAC /
    lower-case / '*' characters, bands from 0 to the full rectangle."""
    print(_run("--seed", seed, "--n", 250))


@pytest.mark.gpu
def test_dropin_long_pairs():
    """Pairs long enough for the one-warp-per-pair fill kernels."""
    print(_run("--seed", 13, "--n", 12, "--min-len", 520, "--max-len", 700))


@pytest.mark.gpu
def test_dropin_uses_gmap_tables():
    """A non-standard mode: the tables come from GMAP's Dynprog_init."""
    print(_run("--seed", 14, "--n", 120, "--mode", 2))


def _params(text, name):
    m = re.search(r"\b" + name + r"\s*\((.*?)\)\s*;", text, flags=re.S)
    assert m, name
    body = re.sub(r"#if.*?#endif", "", m.group(1), flags=re.S)
    out = []
    for prm in body.split(","):
        prm = " ".join(prm.split())
        prm = re.sub(r"\bbool\b", "gdp_bool_t", prm)
        prm = re.sub(r"\bT\b", "Dynprog_T", prm)
        prm = re.sub(r"\bdynprog\b|\bthis\b", "SELF", prm)
        out.append(prm.replace(" *", "* ").replace("* ", "*"))
    return out


def test_dropin_declarations_match_the_reference():
    ref_header = _ref_header()
    if ref_header is None:
        pytest.skip("reference sources not present (set GDP_REFSRC)")
    ours = open(os.path.join(ROOT, "include", "gdp_dynprog_simd.h")).read()
    ours = re.sub(r"/\*.*?\*/", "", ours, flags=re.S)
    theirs = open(ref_header).read()
    names = sorted(set(re.findall(r"\b(Dynprog_(?:simd|traceback)_[0-9a-z_]+)\s*\(", theirs)))
    names = [n for n in names if "nonavx2" not in n]
    assert len(names) == 12, names
    for n in names:
        assert _params(ours, n) == _params(theirs, n), n
