"""CPU, world size 2 over gloo: the multi-GPU host logic (texture sharding and
max-over-ranks timing) that bench.py and multi-GPU users run, without a GPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp

import workloads as syn
from quicktex_b200.shard import block_cost, max_over_ranks, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = syn.mixed_batch(500, workload=4)
        mine = shard(items, world, rank, lambda i: block_cost(i.width, i.height, i.fmt, i.level))
        load = sum(block_cost(items[i].width, items[i].height, items[i].fmt, items[i].level) for i in mine)
        worst = max_over_ranks(load)
        dist.barrier()
        q.put((rank, mine, load, worst))
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, l0, w0), (r1, m1, l1, w1) = res
    assert set(m0).isdisjoint(m1) and len(m0) + len(m1) == 500       # every texture exactly once
    assert w0 == w1 == max(l0, l1)                                    # both ranks agree on the max
    assert max(l0, l1) / min(l0, l1) < 1.05                            # balanced by cost


def test_shard_is_deterministic_and_validates():
    items = list(range(50))
    a = shard(items, 3, 1, lambda i: i % 7 + 1)
    assert a == shard(items, 3, 1, lambda i: i % 7 + 1)
    assert sorted(shard(items, 3, 0, float) + shard(items, 3, 1, float) + shard(items, 3, 2, float)) == items
    with pytest.raises(ValueError):
        shard(items, 2, 2, float)
    assert max_over_ranks(3.5) == 3.5  # no process group: identity
