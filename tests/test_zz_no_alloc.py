"""The fill for callers that cannot allocate device memory.

gdp_fill16_noalloc (include/gdp.h) serves callers that cannot call cudaMalloc
themselves, for example code inside another framework's memory pool or a
host that forbids allocation on its hot path. The caller hands over device
inputs and outputs, and the entry point keeps its working memory in a
fixed file-scope device array. This test is such a caller. It allocates its
own buffers and then calls the entry point twice in a row through the C
ABI. Both times, the scores and every in-band E/F/nogap direction must
equal those of the regular entry point (gdp_fill_dump) and of the CPU
oracle (the reference compiled from its sources, or its C restatement),
bit for bit. Run alone in a fresh process, the first call also performs
the entry point's one-time device set-up.
"""
import ctypes

import numpy as np
import pytest

import cases
import gdp
import oracle as orc

pytestmark = pytest.mark.gpu


def _decode(pairs, i, words, base):
    """Dense (c, r) directions of full-band 16-bit pair i from its words."""
    p = pairs[i]
    rl, gl, lb, ub = int(p["rlength"]), int(p["glength"]), int(p["lband"]), int(p["uband"])
    nb = rl // 16 + 1
    sweeps, boff = [], [0]
    for b in range(nb):
        xlo = 16 * b
        y0 = max(0, xlo - lb)
        y1 = min(min(xlo + 15, rl) + ub, gl)
        sweeps.append((y0, y1))
        boff.append(boff[-1] + max(0, y1 - y0 + 1) * 2)
    n = (rl + 1) * (gl + 1)
    dN = np.zeros(n, np.int8)
    dE = np.zeros(n, np.int8)
    dF = np.zeros(n, np.int8)
    m = orc.domain_mask(0, rl, gl, lb, ub)
    cs, rs = np.nonzero(m)
    for c, r in zip(cs.tolist(), rs.tolist()):
        b, lane = r // 16, r % 16
        y0, y1 = sweeps[b]
        if not (y0 <= c <= y1):
            continue
        # 16-lane columns: even lanes in word 0, odd lanes in word 1, bit lane // 2
        w = int(words[base + boff[b] + (c - y0) * 2 + (lane & 1)])
        sh = lane >> 1
        at = c * (rl + 1) + r
        dN[at] = -2 if (w >> (8 + sh)) & 1 else (-1 if (w >> sh) & 1 else 0)
        dE[at] = -1 if (w >> (16 + sh)) & 1 else 0
        dF[at] = -2 if (w >> (24 + sh)) & 1 else 0
    return dN, dE, dF, m.ravel()


def test_noalloc_fill_matches_batch_entry_point(gdplib, restatement):
    import torch
    pairs, arena = cases.random_cases(4242, 200, variants=(0,), precisions=(16,), max_len=120)
    pairs["flags"] &= ~gdp.FLAG_TRACEBACK
    ref = orc.reference() if orc.reference_available() else restatement
    ref.init(0)
    expect = [ref.align(pairs, i, arena) for i in range(pairs.size)]
    # the regular entry point, for comparison
    ctx = gdp.Context(gdplib)
    offs, H, dN, dE, dF, res_ref = ctx.fill_dump(pairs, arena)
    ctx.close()
    assert (res_ref["status"] == 0).all()

    dev = torch.device("cuda", 0)
    d_pairs = torch.from_numpy(pairs.view(np.uint8).copy()).to(dev)
    d_arena = torch.from_numpy(arena.copy()).to(dev)
    cap = 4 * int(sum(((int(p["rlength"]) // 16 + 1) * (16 + int(p["lband"]) + int(p["uband"]) + 2) * 2 + 4)
                      for p in pairs))
    d_dirs = torch.zeros(cap, dtype=torch.int32, device=dev)
    d_res = torch.zeros(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        d_dirs.zero_()
        d_res.zero_()
        rc = gdplib.gdp_fill16_noalloc(0, 0, ctypes.c_void_p(d_pairs.data_ptr()), pairs.size,
                                       ctypes.c_void_p(d_arena.data_ptr()), arena.size,
                                       ctypes.c_void_p(d_dirs.data_ptr()), cap, ctypes.c_void_p(d_res.data_ptr()),
                                       ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, f"call {call}: {gdp.STATUS.get(rc, rc)}"
        torch.cuda.synchronize()
        res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
        words = d_dirs.cpu().numpy().view(np.uint32)
        assert (res["status"] == 0).all(), f"call {call}"
        assert np.array_equal(res["score"], res_ref["score"]), f"call {call}"
        for i in range(pairs.size):
            n = (int(pairs[i]["rlength"]) + 1) * (int(pairs[i]["glength"]) + 1)
            a0 = int(offs[i])
            gN, gE, gF, m = _decode(pairs, i, words, int(res["rec_offset"][i]))
            o = expect[i]
            assert int(res["score"][i]) == o["score"], (call, i, "score vs oracle")
            for name, got, batch in (("dN", gN, dN), ("dE", gE, dE), ("dF", gF, dF)):
                assert np.array_equal(got[m], batch[a0:a0 + n][m]), (call, i, name, "vs batch entry point")
                assert np.array_equal(got[m], o[name][m]), (call, i, name, "vs oracle")


def test_noalloc_rejects_oversize_requests(gdplib):
    import torch
    # more pairs than the fixed array holds: rejected before any device work
    rc = gdplib.gdp_fill16_noalloc(0, 0, None, 65537, None, 0, None, 0, None, None)
    assert rc == 1   # GDP_ERR_LEN
    # a pair longer than the fixed column limit, one that is not full-band
    # 16-bit, one whose genome window lies past the arena's end, and one
    # asking for a genome window this entry point does not fetch
    pairs, arena = cases.random_cases(7, 2, variants=(0,), precisions=(16,), max_len=40)
    pairs["flags"] &= ~gdp.FLAG_TRACEBACK
    pairs = np.concatenate([pairs, pairs, pairs])
    pairs["glength"][0] = 1024
    pairs["precision"][1] = 8
    pairs["gseq"][2] = arena.size - int(pairs["glength"][2]) + 1
    pairs["flags"][3] |= gdp.FLAG_GWINDOW
    dev = torch.device("cuda", 0)
    d_pairs = torch.from_numpy(pairs.view(np.uint8).copy()).to(dev)
    big = np.zeros(4096, np.uint8)
    big[:arena.size] = arena
    d_arena = torch.from_numpy(big).to(dev)
    d_dirs = torch.zeros(1 << 16, dtype=torch.int32, device=dev)
    d_res = torch.zeros(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    rc = gdplib.gdp_fill16_noalloc(0, 0, ctypes.c_void_p(d_pairs.data_ptr()), pairs.size,
                                   ctypes.c_void_p(d_arena.data_ptr()), arena.size,
                                   ctypes.c_void_p(d_dirs.data_ptr()), 1 << 16, ctypes.c_void_p(d_res.data_ptr()),
                                   None)
    assert rc == 0
    torch.cuda.synchronize()
    res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE)
    assert list(res["status"][:4]) == [1, 3, 1, 3], res["status"]
    assert (res["status"][4:] == 0).all()
    assert torch.cuda.current_device() == 0
