"""Multi-rank host logic on CPU with the gloo backend (world size 2): instance sharding and the
max-over-ranks timing rule used by bench.py."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cfd_solver_withcuda_b200.shard import max_over_ranks, shard_instances, sum_over_ranks


def test_shard_instances_partition():
    cells = [2048 * (i % 7 + 1) for i in range(50)]
    for world in (1, 2, 3, 8):
        parts = [shard_instances(cells, r, world) for r in range(world)]
        flat = [i for p in parts for i in p]
        assert flat == list(range(len(cells)))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells) + 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + rank  # each rank's own device time
        out[rank] = (max_over_ranks(ms, dist), sum_over_ranks(100.0 * (rank + 1), dist))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (11.0, 300.0)
