"""Sharding mesh pairs across ranks (one process per GPU).

Mesh pairs are independent until their outputs, so the collision path shards
by pair with no exchange on the data path.  Costs are estimated by the tet
counts of the two meshes; pairs go largest first to the least-loaded rank
(longest-processing-time greedy), so uneven batches stay balanced.  Outputs
(candidate rows, contacts) of the ranks are gathered once at the end with
torch.distributed (NCCL on GPUs, gloo on CPU), keeping the callers' global
pair indices.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np


def pair_costs(pairs: np.ndarray, tets_per_mesh: Sequence[int]) -> np.ndarray:
    t = np.asarray(tets_per_mesh, np.int64)
    p = np.asarray(pairs, np.int64).reshape(-1, 2)
    return t[p[:, 0]] + t[p[:, 1]]


def partition(pairs: np.ndarray, tets_per_mesh: Sequence[int], world: int) -> List[np.ndarray]:
    """Global pair indices of each rank; every pair appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = pair_costs(pairs, tets_per_mesh)
    order = np.argsort(-cost, kind="stable")
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(i))
        heapq.heappush(heap, (load + int(cost[i]), r))
    return [np.array(sorted(s), np.int64) for s in shards]


def shard(pairs: np.ndarray, tets_per_mesh: Sequence[int], rank: int, world: int) -> np.ndarray:
    return partition(pairs, tets_per_mesh, world)[rank]


def gather_rows(rows: np.ndarray, global_pair_ids: np.ndarray, group=None) -> np.ndarray:
    """All-gather candidate rows (local pair index, a, b) of every rank as
    rows with global pair indices, sorted; every rank gets the full set."""
    import torch.distributed as dist

    rows = np.asarray(rows, np.int64).reshape(-1, 3).copy()
    if len(rows):
        rows[:, 0] = np.asarray(global_pair_ids, np.int64)[rows[:, 0]]
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, rows, group=group)
    out = np.concatenate([p for p in parts if p is not None and len(p)] or [np.zeros((0, 3), np.int64)])
    if len(out):
        out = out[np.lexsort((out[:, 2], out[:, 1], out[:, 0]))]
    return out


def gather_row_buffers(mine, n_rows: int, row_bytes: int, gathered, out, rank: int) -> List[int]:
    """The exchange step of a traversal split over ranks (kdop_traverse_shard):
    every rank's first n_rows rows (row_bytes bytes each) of `mine`, a byte
    tensor of the same fixed capacity on every rank, reach rank 0 packed in
    rank order into `out`.  The row counts are all-gathered first, then the
    fixed-size buffers into `gathered` (one tensor like `mine` per rank);
    works on CUDA tensors over NCCL and on CPU tensors over gloo.  Returns the
    per-rank row counts (on every rank)."""
    import torch
    import torch.distributed as dist

    world = len(gathered)
    if world > 1:
        counts = torch.tensor([n_rows], dtype=torch.int64, device=mine.device)
        all_counts = [torch.empty_like(counts) for _ in range(world)]
        dist.all_gather(all_counts, counts)
        dist.all_gather(gathered, mine)
        cnt = [int(c.item()) for c in all_counts]
    else:
        gathered[0].copy_(mine)
        cnt = [int(n_rows)]
    if rank == 0:
        off = 0
        for r, c in enumerate(cnt):
            if c:
                out[off: off + c * row_bytes].copy_(gathered[r][: c * row_bytes], non_blocking=True)
            off += c * row_bytes
    return cnt
