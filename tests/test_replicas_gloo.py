"""The multi-rank host logic (aerolume_b200/replicas.py, used by bench.py) on two gloo ranks on
the CPU: the max of the ranks' times, the sweep's instance partition and the gather of the
per-instance results to rank 0."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from aerolume_b200.replicas import gather_results, max_over_ranks, shard_instances


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = max_over_ranks(1.5 + rank, dist, device="cpu")
        shards = shard_instances(sizes, world)
        mine = {k: ("rank", rank, sizes[k]) for k in shards[rank]}
        merged = gather_results(mine, dist)
        q.put((rank, t, shards, merged))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_partition_and_gather():
    sizes = [32768 * (1 + (k * 7) % 16) for k in range(64)]
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict((r, (t, s, m)) for r, t, s, m in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][0] == res[1][0] == 2.5          # both ranks see the max
    assert res[0][1] == res[1][1]                  # the same partition on both ranks
    merged = res[0][2]
    assert res[1][2] is None and sorted(merged) == list(range(64))
    for k, (_, r, size) in merged.items():
        assert k in res[0][1][r] and size == sizes[k]


def test_partition_is_balanced_and_complete():
    sizes = [32768, 73728, 131072, 294912, 524288] * 12 + [32768] * 4
    for world in (1, 2, 3, 8):
        shards = shard_instances(sizes, world)
        assert sorted(k for s in shards for k in s) == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in s) for s in shards]
        assert max(loads) - min(loads) <= max(sizes)
    with pytest.raises(ValueError):
        shard_instances(sizes, 0)


def test_single_process_fallbacks():
    assert max_over_ranks(3.0) == 3.0
    assert gather_results({1: "a"}) == {1: "a"}
