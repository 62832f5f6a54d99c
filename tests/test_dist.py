"""Two-rank gloo tests (CPU) of the multi-process plumbing."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hfscf_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = D.max_over_ranks(1.5 + rank)
        items = D.shard(11, rank, world)
        q.put((rank, m, items))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_shards_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    maxes = {r: m for r, m, _ in out}
    assert maxes == {0: 2.5, 1: 2.5}
    items = sorted(i for _, _, its in out for i in its)
    assert items == list(range(11))


def test_without_process_group_is_identity():
    assert D.max_over_ranks(3.25) == 3.25
    assert D.shard(5, 0, 1) == [0, 1, 2, 3, 4]
