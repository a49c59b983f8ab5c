"""Multi-rank host logic on CPU (gloo, world size 2): batch sharding is
consistent across ranks, covers every text once and balances bytes; the
max-over-ranks timing reduction used by bench.py picks the slowest rank."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from psacak_b200.batch import shard_lpt


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, lengths, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard_lpt(lengths, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    # the reduction bench.py applies to every per-rank time
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    slowest = bench._max_over_ranks(torch, dist, torch.device("cpu"), 10.0 * (rank + 1))
    q.put((rank, got, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_lpt_two_ranks():
    lengths = [int(x) for x in torch.randint(1, 1 << 20, (257,), generator=torch.Generator().manual_seed(3))]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, lengths, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] == res[1][1]  # both ranks computed the same assignment
    shards = res[0][1]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(lengths)))
    loads = [sum(lengths[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(lengths)
    assert all(r[2] == 20.0 for r in res)  # max over ranks


def test_shard_lpt_single_and_empty():
    assert shard_lpt([5, 3, 9], 1) == [[0, 1, 2]]
    assert shard_lpt([], 3) == [[], [], []]
