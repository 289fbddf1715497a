"""Matrix sharding for the served and batched forms on several GPUs.

The forms shard by matrix: every rank (one process per GPU) owns a subset of
the global matrix table, serves the requests addressed to its matrices, and
no data-path collective is needed.  The partition is a deterministic greedy
balance of device bytes (largest first onto the least-loaded rank, ties to the
lower rank), so every rank computes the same owner table without
communication.  The only collective is the final aggregation of counts and
wall times (a sum and a max over ranks).
"""
from __future__ import annotations

import heapq

import numpy as np


def matrix_bytes(n_rows: int, n_cols: int, nnz: int, value_size: int = 4, slack: float = 2.0,
                 spare: float = 2.0, max_segs: int = 4) -> int:
    """Device bytes of a resident DCSR matrix: pool (entries x slack x spare,
    column + value), row lengths, segment table."""
    pitch = ((2 * n_rows + 31) // 32) * 32
    return int(nnz * slack * spare * (4 + value_size) + 4 * (n_rows + 1) + 4 * pitch * max_segs)


def partition(sizes, world: int) -> np.ndarray:
    """owner[i] in [0, world) for matrix i, balancing the sum of sizes."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world)]
    owner = np.empty(len(sizes), dtype=np.int32)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return owner


def local_view(owner: np.ndarray, rank: int):
    """(global ids owned by rank, map global id -> local index or -1)."""
    mine = np.nonzero(owner == rank)[0]
    local = np.full(len(owner), -1, dtype=np.int64)
    local[mine] = np.arange(len(mine))
    return mine, local


def route(matrix_ids: np.ndarray, owner: np.ndarray, rank: int):
    """Positions of the requests this rank serves and their local matrix ids."""
    _, local = local_view(owner, rank)
    sel = np.nonzero(owner[matrix_ids] == rank)[0]
    return sel, local[matrix_ids[sel]]


def aggregate(requests: int, wall_s: float, group=None):
    """Whole-job throughput: requests of all ranks / the slowest rank's wall
    time (one sum and one max over ranks; a single process needs none)."""
    import torch
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return requests / wall_s, requests, wall_s
    c = torch.tensor([float(requests)], dtype=torch.float64)
    w = torch.tensor([float(wall_s)], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        c, w = c.cuda(), w.cuda()
    dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(w, op=dist.ReduceOp.MAX, group=group)
    total, slowest = float(c.item()), float(w.item())
    return total / slowest, total, slowest
