"""The medoid pass and DBA rounds over several GPUs: one process per GPU.
The medoid pass takes pair ranges balanced by DTW cell count and one
all-gather of the distance triangle; a DBA round takes member blocks balanced
by cells and one all-gather of per-member sample ranges (below).

The reference deals whole rows of the pair triangle to its devices in turn
(approximateMedoidIndices, dba.hpp:67-161) and gathers the distances on the
host.  Here each rank takes a contiguous range of pair indices in the
reference's upper-triangle order (clustering.cuh:4-6) holding about 1/world
of the cells, computes it with odba_dtw_pairwise_range_*, and the ranges are
exchanged with one all-gather (NCCL over NVLink on B200, gloo on CPU); every
rank then holds the full triangle and picks the same medoid.  The exchange is
the only collective: 8 MB for 2000 series.
"""
from __future__ import annotations

import numpy as np


def pair_row_starts(n: int) -> np.ndarray:
    """Index of the first pair (s, s+1) of every row s (clustering.cuh:4-6)."""
    s = np.arange(n, dtype=np.int64)
    return s * n - s * (s + 1) // 2


def shard_ranges(lens, world: int):
    """Contiguous [begin, end) pair ranges, one per rank, of near-equal cell
    counts (pair (s, j) costs lens[s] * lens[j])."""
    L = np.asarray(lens, dtype=np.float64)
    n = len(L)
    npairs = n * (n - 1) // 2
    if world <= 1 or npairs == 0:
        return [(0, npairs)] + [(npairs, npairs)] * max(0, world - 1)
    suffix = np.concatenate([np.cumsum(L[::-1])[::-1][1:], [0.0]])  # sum_{j>s} L_j
    row_cells = L * suffix
    row_cum = np.concatenate([[0.0], np.cumsum(row_cells)])
    total = row_cum[-1]
    starts = pair_row_starts(n)
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        s = int(np.searchsorted(row_cum, target, side="right")) - 1
        s = min(max(s, 0), n - 2)
        # within row s: pairs (s, j) for j = s+1.., cumulative L_s * sum L_j
        within = L[s] * np.cumsum(L[s + 1:])
        k = int(np.searchsorted(within, target - row_cum[s], side="left"))
        p = int(starts[s] + min(k, n - s - 1))
        bounds.append(max(p, bounds[-1]))
    bounds.append(npairs)
    return [(bounds[i], bounds[i + 1]) for i in range(world)]


def gather_triangle(dists, ranges, rank: int, world: int, group=None):
    """All ranks' ranges of a full-size triangle tensor, exchanged with one
    all-gather; returns the assembled triangle (a new tensor, same device)."""
    import torch
    import torch.distributed as dist
    width = max(e - b for b, e in ranges) if ranges else 0
    b, e = ranges[rank]
    mine = torch.zeros(max(width, 1), dtype=dists.dtype, device=dists.device)
    if e > b:
        mine[: e - b] = dists[b:e]
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = torch.empty_like(dists)
    for r, (rb, re_) in enumerate(ranges):
        if re_ > rb:
            out[rb:re_] = parts[r][: re_ - rb]
    return out


def medoid_pass_sharded(ds, host_lens, rank: int, world: int, open_start=0, open_end=0,
                        group=None, workspace=None, stream=None):
    """One medoid pass over all ranks (every rank passes the same series):
    (full distance triangle on this rank's device, medoid index)."""
    import torch
    from . import _native, api
    n = ds.n
    npairs = n * (n - 1) // 2
    ranges = shard_ranges(host_lens, world)
    b, e = ranges[rank]
    dists = torch.zeros(max(npairs, 1), dtype=ds.data.dtype, device=ds.data.device)
    if workspace is None:
        lib = _native.lib()
        nbytes = lib.odba_dtw_pairwise_workspace_bytes(ds.dtype.itemsize, ds.max_len)
        workspace = torch.empty(nbytes, dtype=torch.uint8, device=ds.data.device)
    _native.call(f"odba_dtw_pairwise_range_{api._SFX[ds.dtype]}", ds.data.data_ptr(),
                 ds.offsets.data_ptr(), ds.lens.data_ptr(), n, ds.max_len, int(open_start),
                 int(open_end), b, e, dists.data_ptr(), workspace.data_ptr(), workspace.numel(),
                 api._stream_ptr(stream))
    full = gather_triangle(dists[:npairs], ranges, rank, world, group) if world > 1 else dists[:npairs]
    _, med = api.medoid(full, ds, stream=stream)
    return full, med


# ---------------------------------------------------------------------------
# DBA rounds over several GPUs.
#
# The reference deals the members of a round to its devices in turn
# (DBAUpdate, dba.hpp:484-486: currDevice = seq_index % deviceCount) and adds
# every aligned sample into one centroid sum with atomics.  Float sums depend
# on their order, so here each rank aligns a contiguous block of members
# (odba_dba_round_ranges_*: path DTW and backtrack) and emits, per member and
# centroid index, the range of member samples that index receives; one
# all-gather gives every rank all members' ranges in the round's member order,
# and every rank runs the ordered reducer (odba_dba_reduce_ranges_*) over them.
# The new centroid is therefore bit-identical to the one-GPU round, and every
# rank holds it for the next round without a broadcast.  An all-reduce of
# per-rank partial sums would change the rounding.

def member_shards(lens, world: int):
    """Contiguous [begin, end) member blocks, one per rank, of near-equal DTW
    cells (every member is aligned to the same centroid, so cells are
    proportional to the member's length)."""
    L = np.asarray(lens, dtype=np.float64)
    n = len(L)
    if world <= 1 or n == 0:
        return [(0, n)] + [(n, n)] * max(0, world - 1)
    cum = np.concatenate([[0.0], np.cumsum(L)])
    bounds = [0]
    for r in range(1, world):
        k = int(np.searchsorted(cum, cum[-1] * r / world, side="left"))
        bounds.append(min(max(k, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[i], bounds[i + 1]) for i in range(world)]


def gather_member_ranges(local, shards, rank: int, world: int, group=None):
    """All ranks' [count, Lc, 2] int32 range blocks, exchanged with one
    all-gather (blocks padded to the largest); returns [n, Lc, 2] in member
    order."""
    import torch
    import torch.distributed as dist
    width = max(e - b for b, e in shards)
    Lc = local.shape[1]
    mine = torch.zeros((max(width, 1), Lc, 2), dtype=torch.int32, device=local.device)
    b, e = shards[rank]
    if e > b:
        mine[: e - b] = local
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    return torch.cat([parts[r][: re_ - rb] for r, (rb, re_) in enumerate(shards)], dim=0)


def dba_round_sharded(centroid, ds, rank: int, world: int, open_start=0, open_end=0, group=None,
                      stream=None):
    """One full-path DBA round over all ranks (every rank passes the same
    centroid and members): (new centroid, counts, delta), the same on every
    rank and bit-identical to api.dba_round on one GPU."""
    from . import api
    shards = member_shards(ds.host_lens, world)
    b, e = shards[rank]
    local = api.dba_round_ranges(centroid, ds.subset(b, e), open_start, open_end, stream=stream)
    full = gather_member_ranges(local, shards, rank, world, group) if world > 1 else local
    return api.dba_reduce_ranges(centroid, ds, full, open_start, open_end, stream=stream)
