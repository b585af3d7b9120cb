"""The N > 1 path on the CPU: instances split across ranks with no collective
in the timed loop, results merged afterwards, time taken as the max over ranks.

A single instance does not shard (every step needs global Poisson solves), so
more GPUs run replicas of the 3D gradient; the batched 2D instances are
independent units split by cost.  These tests run the host logic of that split
as two ``gloo`` ranks on the CPU (the kernels need a GPU; what the ranks
compute here is a stand-in for a gradient).
"""
import importlib
import json
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

B = importlib.import_module("differentiable-flowmap_b200.batch")


def test_partition_covers_every_instance_once_and_balances():
    sizes, steps = B.DEFAULT_SIZES, 100
    costs = [B.instance_cost(n, steps) for n in sizes]
    for world in (1, 2, 3, 4, 8, 16, 20):
        parts = B.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # greedy LPT: no rank exceeds the ideal share by more than the largest instance
        assert max(loads) <= sum(costs) / world + max(costs)
        assert parts == B.partition(costs, world)  # deterministic
        assert all(p == sorted(p) for p in parts)
    two = B.partition(costs, 2)
    assert abs(sum(costs[i] for i in two[0]) - sum(costs[i] for i in two[1])) <= max(costs)
    with pytest.raises(ValueError):
        B.partition(costs, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _stand_in(i, n, steps):
    """What rank-local work returns for instance i (deterministic in i only)."""
    return [float(n * steps + i), float(i) * 0.5]


def _worker(rank, world, port, out_path):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        sizes, steps = B.DEFAULT_SIZES, 100
        mine = B.rank_share(sizes, steps, rank, world)
        local = {i: _stand_in(i, sizes[i], steps) for i in mine}
        merged = B.gather_results(local)
        t = torch.tensor([10.0 + rank], dtype=torch.float64)  # this rank's elapsed time
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
        if rank == 0:
            with open(out_path, "w") as f:
                json.dump({"merged": {str(k): v for k, v in merged.items()}, "max_time": float(t.item()),
                           "shares": [B.rank_share(sizes, steps, r, world) for r in range(world)]}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_merge(tmp_path):
    out = str(tmp_path / "rank0.json")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    res = json.load(open(out))
    sizes, steps = B.DEFAULT_SIZES, 100
    want = {str(i): _stand_in(i, sizes[i], steps) for i in range(len(sizes))}
    assert res["merged"] == want                # every instance once, from the rank that owns it
    assert res["max_time"] == 11.0              # the slower rank's time
    a, b = res["shares"]
    assert not set(a) & set(b) and len(a) + len(b) == len(sizes)


def test_gather_results_without_a_process_group():
    assert B.gather_results({3: [1.0]}) == {3: [1.0]}
