"""The multi-GPU path on the CPU: two gloo ranks.

Pairs are independent, so the batch is sharded across ranks with no
collective on the data path (weak scaling): each rank aligns its own shard
and the only collectives are the max of the ranks' times and the sums of
their cell and pair counts.  These tests run that plumbing with world_size
2 on the gloo backend: the shards of one batch are disjoint, cover it and
carry balanced work, the bench's reductions give the max and the sums, and
outputs aligned rank by rank and gathered equal the whole batch's.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))
    sys.path.insert(0, ROOT)
    import datetime
    import torch
    import torch.distributed as dist
    import gdp
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    lib = gdp.load()
    genome, _ = gdp.make_genome(lib, 777, 1 << 20)
    pairs, _ = gdp.make_pairs(lib, gdp.WL_MIX, 5, genome, 400)
    mine = gdp.shard_indices(pairs, world, rank)
    cells = float(gdp.band_cells(pairs[mine]).sum())
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine.tolist(), cells))
    tmax = bench.max_over_ranks(world, float(rank + 1) * 1.5)
    tsum = bench.sum_over_ranks(world, cells)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"),
            np.array([tmax, tsum, float(sum(c for _, c in gathered))], dtype=np.float64))
    if rank == 0:
        allidx = sorted(i for idx, _ in gathered for i in idx)
        np.save(os.path.join(out_dir, "union.npy"), np.array(allidx, dtype=np.int64))
        np.save(os.path.join(out_dir, "cells.npy"), np.array([c for _, c in gathered], dtype=np.float64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    union = np.load(tmp_path / "union.npy")
    assert np.array_equal(union, np.arange(400))          # disjoint shards covering the batch
    cells = np.load(tmp_path / "cells.npy")
    assert abs(cells[0] - cells[1]) / cells.sum() < 0.05  # balanced work
    for r in range(world):
        tmax, tsum, total = np.load(tmp_path / f"rank{r}.npy")
        assert tmax == 3.0                                  # max over ranks of (rank + 1) * 1.5
        assert tsum == total == cells.sum()


def _align_rank_main(rank, world, port, out_dir):
    """One rank aligns its own shard (the oracle's C restatement standing
    in for the device) and the shards' outputs are gathered on rank 0."""
    sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime
    import hashlib
    import torch.distributed as dist
    import gdp
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    lib = gdp.load_workload()
    genome, blocks = gdp.make_genome(lib, 778, 1 << 20)
    pairs, arena = gdp.make_pairs(lib, gdp.WL_FIXED, 6, genome, 120)
    ref = oracle.restatement()
    ref.init(0)
    ref.set_genome(blocks, None, genome.size)
    out = {}
    for i in gdp.shard_indices(pairs, world, rank).tolist():
        o = ref.align(pairs, i, arena, want_matrix=False)
        out[i] = (int(o["score"]), [int(v) for v in o["stats"]], hashlib.sha1(o["recs"].tobytes()).hexdigest())
    gathered = [None] * world
    dist.all_gather_object(gathered, out)
    if rank == 0:
        merged = {}
        for g in gathered:
            assert not set(g) & set(merged)                 # every pair aligned by one rank only
            merged.update(g)
        whole = {}
        for i in range(pairs.size):                         # the same batch in one process
            o = ref.align(pairs, i, arena, want_matrix=False)
            whole[i] = (int(o["score"]), [int(v) for v in o["stats"]], hashlib.sha1(o["recs"].tobytes()).hexdigest())
        np.save(os.path.join(out_dir, "same.npy"), np.array([merged == whole, len(merged)], dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_align_their_shards(tmp_path):
    """The sharded data path: each rank aligns only its shard and the
    gathered outputs equal the whole batch aligned in one process."""
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    mp.start_processes(_align_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    same, n = np.load(tmp_path / "same.npy")
    assert n == 120 and same == 1


def test_shards_are_deterministic_and_balanced():
    sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))
    import gdp
    lib = gdp.load()
    genome, _ = gdp.make_genome(lib, 7, 1 << 20)
    pairs, _ = gdp.make_pairs(lib, gdp.WL_SHORT, 9, genome, 1000)
    for world in (2, 4, 8):
        shards = [gdp.shard_indices(pairs, world, r) for r in range(world)]
        assert np.array_equal(np.sort(np.concatenate(shards)), np.arange(pairs.size))
        c = np.array([gdp.band_cells(pairs[s]).sum() for s in shards], dtype=np.float64)
        assert (c.max() - c.min()) / c.mean() < 0.02
        assert all(np.array_equal(s, gdp.shard_indices(pairs, world, r)) for r, s in enumerate(shards))
