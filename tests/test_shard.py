"""Sharding of independent lattices over ranks: the partition (CPU) and the
rank-level reductions with world_size 2 over gloo on CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dynlattice_b200.shard import partition_by_elements


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    sizes = rng.integers(100, 20000, size=256)
    for world in (1, 2, 3, 8):
        parts = partition_by_elements(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [int(sizes[p].sum()) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(loads) / world + sizes.max()
    assert partition_by_elements([5, 5, 5], 2) == [[0, 2], [1]]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, out):
    import datetime

    import torch.distributed as dist

    from dynlattice_b200.shard import max_over_ranks, partition_by_elements, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    parts = partition_by_elements(sizes, world)
    mine = parts[rank]
    work = float(sum(sizes[i] for i in mine))
    got = [None] * world
    dist.all_gather_object(got, mine)
    tmax = max_over_ranks(work)
    tsum = sum_over_ranks(work)
    out.put((rank, got, tmax, tsum))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    sizes = [int(x) for x in np.random.default_rng(1).integers(10, 1000, size=17)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = partition_by_elements(sizes, 2)
    for rank, got, tmax, tsum in res:
        assert got == parts
        assert tsum == sum(sizes)
        assert tmax == max(sum(sizes[i] for i in p) for p in parts)
