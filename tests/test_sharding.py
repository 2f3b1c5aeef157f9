"""Host logic of the multi-GPU medoid pass (opendba_b200/sharding.py) on CPU:
cell-balanced pair ranges, and the all-gather that assembles the triangle,
run as two gloo ranks.  The CPU oracle stands in for each rank's kernel."""
import os
import socket

import numpy as np
import pytest

from opendba_b200 import sharding


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_ranges_cover_and_balance(world):
    rng = np.random.default_rng(world)
    lens = np.sort(rng.integers(2000, 8001, size=400))
    ranges = sharding.shard_ranges(lens, world)
    n = len(lens)
    assert ranges[0][0] == 0 and ranges[-1][1] == n * (n - 1) // 2
    for (b0, e0), (b1, _) in zip(ranges, ranges[1:]):
        assert e0 == b1 and b0 <= e0
    # cells per range
    L = lens.astype(np.float64)
    starts = sharding.pair_row_starts(n)
    rows = np.repeat(np.arange(n), n - 1 - np.arange(n))
    cols = np.arange(n * (n - 1) // 2) - starts[rows] + rows + 1
    cost = L[rows] * L[cols]
    per = np.array([cost[b:e].sum() for b, e in ranges])
    assert per.max() / per.mean() < 1.01


def test_shard_ranges_tiny_inputs():
    assert sharding.shard_ranges([5], 4) == [(0, 0)] * 4
    r = sharding.shard_ranges([5, 6, 7], 8)
    assert r[0][0] == 0 and r[-1][1] == 3
    assert all(b <= e for b, e in r)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, result_dir):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(11)
        series = sorted([rng.standard_normal(int(L)).astype(np.float32)
                         for L in rng.integers(50, 400, size=23)], key=len)
        lens = [len(s) for s in series]
        ranges = sharding.shard_ranges(lens, world)
        b, e = ranges[rank]
        local = O.pairwise(series, 0, 0, fma_mode=1, pair_list=np.arange(b, e))
        full = sharding.gather_triangle(torch.from_numpy(local), ranges, rank, world)
        np.save(os.path.join(result_dir, f"rank{rank}.npy"), full.numpy())
    finally:
        dist.destroy_process_group()


def test_all_gather_assembles_the_triangle_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    rng = np.random.default_rng(11)
    series = sorted([rng.standard_normal(int(L)).astype(np.float32)
                     for L in rng.integers(50, 400, size=23)], key=len)
    want = O.pairwise(series, 0, 0, fma_mode=1)
    lens = np.array([len(s) for s in series], dtype=np.uint64)
    want_med, _ = O.medoid(want, lens)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert O.medoid(got, lens)[0] == want_med


# ---- DBA rounds dealt by member (sharding.dba_round_sharded) ----------------

@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_member_shards_cover_and_balance(world):
    rng = np.random.default_rng(50 + world)
    lens = rng.integers(500, 8001, size=300)
    shards = sharding.member_shards(lens, world)
    assert shards[0][0] == 0 and shards[-1][1] == len(lens) and len(shards) == world
    for (b0, e0), (b1, _) in zip(shards, shards[1:]):
        assert e0 == b1 and b0 <= e0
    per = np.array([lens[b:e].sum() for b, e in shards], dtype=np.float64)
    assert per.max() / per.mean() < 1.05


def test_member_shards_fewer_members_than_ranks():
    s = sharding.member_shards([10, 20, 30], 8)
    assert s[0][0] == 0 and s[-1][1] == 3 and all(b <= e for b, e in s)
    assert sum(e - b for b, e in s) == 3


def _round_inputs(dtype, seed):
    rng = np.random.default_rng(seed)
    members = [rng.standard_normal(int(L)).astype(dtype) for L in rng.integers(40, 260, size=11)]
    centroid = rng.standard_normal(150).astype(dtype)
    return centroid, members


def _round_rank_main(rank, world, port, result_dir, dtype_name, open_start, open_end):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dtype = np.dtype(dtype_name)
        centroid, members = _round_inputs(dtype, 21)
        shards = sharding.member_shards([len(m) for m in members], world)
        b, e = shards[rank]
        # the oracle stands in for this rank's path DTW and backtrack
        local = torch.from_numpy(O.member_ranges(centroid, members[b:e], open_start, open_end))
        full = sharding.gather_member_ranges(local, shards, rank, world).numpy()
        mean, counts, delta = O.reduce_ranges(centroid, members, full)
        np.save(os.path.join(result_dir, f"rank{rank}_mean.npy"), mean)
        np.save(os.path.join(result_dir, f"rank{rank}_counts.npy"), counts)
        np.save(os.path.join(result_dir, f"rank{rank}_delta.npy"), np.array([delta]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dtype_name,open_start,open_end", [("float32", 0, 0), ("float32", 0, 1),
                                                            ("float64", 1, 1)])
def test_sharded_round_equals_one_rank_round_two_gloo_ranks(tmp_path, dtype_name, open_start, open_end):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    world = 2
    mp.start_processes(_round_rank_main,
                       args=(world, _free_port(), str(tmp_path), dtype_name, open_start, open_end),
                       nprocs=world, start_method="spawn", join=True)
    centroid, members = _round_inputs(np.dtype(dtype_name), 21)
    want_mean, want_counts, _, want_delta = O.dba_update(centroid, members, open_start, open_end)
    for r in range(world):
        mean = np.load(tmp_path / f"rank{r}_mean.npy")
        assert np.array_equal(mean.view(np.uint8), want_mean.view(np.uint8))
        assert np.array_equal(np.load(tmp_path / f"rank{r}_counts.npy"), want_counts)
        assert np.load(tmp_path / f"rank{r}_delta.npy")[0] == want_delta
