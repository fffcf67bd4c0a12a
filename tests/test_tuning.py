"""Plan graphs and the routing autotuner.

* A plan executed as a CUDA graph (gdp_plan_use_graph) gives the same
  results and Pair records as the plain launches, call after call.
* The autotuner (gdp_autotune) picks routing parameters (which pairs go to
  one thread, a lane group or a CTA; the traceback mapping) from timings of
  a sample; the results of a batch aligned with the tuned parameters are
  identical to those with the defaults.
* The plan's stream layouts (concurrent chains, one stream, footprint cap)
  give identical results.
"""
import ctypes

import numpy as np
import pytest

import gdp

pytestmark = pytest.mark.gpu

KEYS = ("status", "score", "precision", "rerun", "tb_score", "nmatches", "nmismatches", "nopens", "nindels",
        "nrecs")


def _same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in KEYS)


def test_plan_graph_matches_plain_launches(gdplib):
    import torch
    genome, blocks = gdp.make_genome(gdplib, 61, 1 << 22)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_MIX, 62, genome, 600)
    ctx = gdp.Context(gdplib)
    ctx.set_genome(blocks, None, genome.size)
    dp = torch.from_numpy(pairs.view(np.uint8)).cuda()
    da = torch.from_numpy(arena).cuda()
    outs = []
    for graph in (0, 1):
        plan = ctypes.c_void_p()
        assert gdplib.gdp_plan_create(ctx.h, gdp._ptr(pairs), pairs.size, ctypes.byref(plan)) == 0, ctx.error()
        assert gdplib.gdp_plan_use_graph(plan, graph) == 0
        tr = int(gdplib.gdp_plan_total_recs(plan))
        for call in range(3):
            dr = torch.zeros(pairs.size * gdp.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
            dc = torch.zeros(max(tr, 1) * gdp.REC_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
            if call == 0:
                keep = (dr, dc)          # later calls reuse the first call's buffers (same graph key)
            else:
                dr, dc = keep
                dr.zero_()
                dc.zero_()
            before = ctx.launches()
            rc = gdplib.gdp_plan_execute(ctx.h, plan, ctypes.c_void_p(dp.data_ptr()), ctypes.c_void_p(da.data_ptr()),
                                         ctypes.c_void_p(dr.data_ptr()), ctypes.c_void_p(dc.data_ptr()))
            assert rc == 0, ctx.error()
            torch.cuda.synchronize()
            assert ctx.launches() > before
            res = np.frombuffer(dr.cpu().numpy().tobytes(), dtype=gdp.RESULT_DTYPE).copy()
            recs = dc.cpu().numpy().tobytes()
            outs.append((graph, call, res, recs))
        gdplib.gdp_plan_destroy(plan)
    ctx.close()
    _, _, r0, c0 = outs[0]
    assert (r0["status"] == 0).all()
    for graph, call, r, c in outs[1:]:
        assert _same(r, r0), (graph, call)
        assert c == c0, (graph, call)


def test_autotuned_routing_gives_identical_results(gdplib):
    genome, blocks = gdp.make_genome(gdplib, 71, 1 << 22)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_MIX, 72, genome, 1500)
    ctx = gdp.Context(gdplib)
    ctx.set_genome(blocks, None, genome.size)
    ref, ref_recs = ctx.align(pairs, arena)
    params, best = ctx.autotune(pairs[:600], arena)
    assert best > 0
    assert set(params) == {"warp_min_x", "warp_max_sweep", "group_slack", "tb_warp", "check_groups", "check_min_x"}
    got, got_recs = ctx.align(pairs, arena)
    # a forced, very different routing gives the same results too
    ctx.set_param("warp_min_x", 1 << 30)
    ctx.set_param("tb_warp", 0)
    ctx.set_param("check_groups", 0)
    ctx.set_param("check_min_x", 1 << 30)
    thr, thr_recs = ctx.align(pairs, arena)
    with pytest.raises(ValueError):
        ctx.set_param("no_such_parameter", 1)
    ctx.close()
    assert (ref["status"] == 0).all()
    assert _same(got, ref) and got_recs.tobytes() == ref_recs.tobytes()
    assert _same(thr, ref) and thr_recs.tobytes() == ref_recs.tobytes()


def test_stream_layouts_give_identical_results(gdplib):
    """The concurrent layout of a plan (jump-late chain and lane-group kinds
    on side streams, each chain tracing its own pairs back), the one-stream
    layout of per-launch timing, and the layout under a grid footprint cap
    (two side streams, one chain) give the same results and records."""
    genome, blocks = gdp.make_genome(gdplib, 81, 1 << 22)
    a, arena_a = gdp.make_pairs(gdplib, gdp.WL_MIX, 82, genome, 800)
    b, arena_b = gdp.make_pairs(gdplib, gdp.WL_SHORT, 83, genome, 2000)
    b = b.copy()
    for f in ("rseq", "rseq_uc", "gseq", "gseq_alt"):
        b[f] += arena_a.size
    pairs, arena = np.concatenate([a, b]), np.concatenate([arena_a, arena_b])
    ctx = gdp.Context(gdplib)
    ctx.set_genome(blocks, None, genome.size)
    ref, ref_recs = ctx.align(pairs, arena)
    ctx.profile(True)
    prof, prof_recs = ctx.align(pairs, arena)
    ctx.profile(False)
    ctx.set_param("grid_blocks_per_sm", 2)
    cap, cap_recs = ctx.align(pairs, arena)
    ctx.close()
    assert (ref["status"] == 0).all()
    late = (pairs["flags"] & gdp.FLAG_JUMP_LATE) != 0
    assert late.any() and (~late).any()
    assert _same(prof, ref) and prof_recs.tobytes() == ref_recs.tobytes()
    assert _same(cap, ref) and cap_recs.tobytes() == ref_recs.tobytes()


def test_direction_budget_splits_waves(gdplib):
    """A context whose direction-memory budget holds only a few pairs' words
    cuts the host-buffer batch into many waves; the results and records are
    the same bytes as one wave's."""
    genome, blocks = gdp.make_genome(gdplib, 81, 1 << 22)
    pairs, arena = gdp.make_pairs(gdplib, gdp.WL_MIX, 82, genome, 800)
    outs = []
    for budget in (0, 1 << 20):
        ctx = gdp.Context(gdplib, budget=budget)
        ctx.set_genome(blocks, None, genome.size)
        before = ctx.launches()
        res, recs = ctx.align(pairs, arena)
        outs.append((res, recs, ctx.launches() - before))
        ctx.close()
    (r0, c0, l0), (r1, c1, l1) = outs
    assert (r0["status"] == 0).all()
    assert _same(r0, r1) and c0.tobytes() == c1.tobytes()
    assert l1 > 2 * l0          # many more waves ran
