"""Sharding of the served/batched forms across ranks, as 2 gloo processes on
the CPU: every rank computes the same owner table, the shards cover the
matrix table exactly once with balanced bytes, every request of a global
trace is served by exactly one rank, and the aggregate throughput is the
total requests over the slowest rank's wall time."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from dcsr_b200 import shard
    from dcsr_b200 import workloads as W
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        specs = W.batched_specs(5, count=300)
        sizes = [shard.matrix_bytes(s["n"], s["n"], int(s["n"] * s["degree"])) for s in specs]
        owner = shard.partition(sizes, world)
        gathered = [torch.zeros(len(owner), dtype=torch.int32) for _ in range(world)]
        dist.all_gather(gathered, torch.from_numpy(owner))
        same = all(torch.equal(g, gathered[0]) for g in gathered)
        kind, mat, size = W.served_trace(6, len(specs), 5000)
        sel, local = shard.route(mat, owner, rank)
        mine, _ = shard.local_view(owner, rank)
        served = torch.zeros(len(mat), dtype=torch.int32)
        served[torch.from_numpy(sel)] = 1
        dist.all_reduce(served)
        load = torch.tensor([float(sum(sizes[i] for i in mine))], dtype=torch.float64)
        loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(loads, load)
        # rank r "served" its requests in (r + 1) seconds
        thr, total, slowest = shard.aggregate(len(sel), float(rank + 1))
        out[rank] = dict(same=same, each_once=bool((served == 1).all()), local_ok=bool(
            (np.asarray(mine)[local] == mat[sel]).all()), loads=[float(x) for x in loads],
            max_size=max(sizes), thr=thr, total=total, slowest=slowest, n=len(mat))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for r in (0, 1):
        assert res[r]["same"], "ranks disagree on the owner table"
        assert res[r]["each_once"], "a request is served by zero or two ranks"
        assert res[r]["local_ok"]
    loads = res[0]["loads"]
    assert abs(loads[0] - loads[1]) <= res[0]["max_size"], loads
    assert res[0]["total"] == res[0]["n"] and res[0]["slowest"] == 2.0
    assert res[0]["thr"] == pytest.approx(res[0]["n"] / 2.0)
    assert res[1]["thr"] == res[0]["thr"]


def test_single_process_partition():
    from dcsr_b200 import shard
    owner = shard.partition([5, 1, 1, 1, 1, 1], 2)
    assert owner.tolist() == [0, 1, 1, 1, 1, 1]  # largest first, then onto the least-loaded rank
    assert shard.partition([3, 3, 2, 2], 2).tolist() == [0, 1, 0, 1]
    assert shard.partition([7, 1], 1).tolist() == [0, 0]
    thr, total, slowest = shard.aggregate(100, 2.0)
    assert thr == 50.0 and total == 100 and slowest == 2.0
