"""Multi-rank plumbing on CPU (gloo, world size 2): the timing reduction used by
bench.py under torchrun and the footprint partition of independent decks."""
import datetime
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from ferrix_b200 import multi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = multi.max_over_ranks(float(10 * (rank + 1)))
        s = multi.sum_over_ranks(1.0)
        parts = multi.partition_by_footprint(sizes, world)
        dist.barrier()
        q.put((rank, m, s, parts))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_partition_with_two_gloo_ranks():
    world = 2
    sizes = [5e3, 6e4, 2e3, 3.3e4, 1.2e4, 4.4e4, 9e3, 2.5e4, 7e3]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [20.0, 20.0]          # max over ranks, on every rank
    assert [o[2] for o in out] == [2.0, 2.0]
    assert out[0][3] == out[1][3]                        # every rank computes the same partition
    parts = out[0][3]
    assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)         # greedy balance bound


def test_partition_single_rank_and_errors():
    assert multi.partition_by_footprint([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    assert multi.partition_by_footprint([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        multi.partition_by_footprint([1.0], 0)
    assert multi.max_over_ranks(3.5) == 3.5  # no process group: identity
