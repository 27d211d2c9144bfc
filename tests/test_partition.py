"""Multi-rank ensemble sharding on CPU: two gloo ranks each take their share
of the boxes (bench.partition_boxes, greedy by N^3 log N); together the
shares are disjoint, cover every box and are balanced in cost."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    boxes = bench.ensemble_boxes(96)
    costs = [p.nx * p.ny * p.nz * np.log2(p.nx * p.ny * p.nz) for _, p in boxes]
    mine = bench.partition_boxes(costs, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, float(sum(costs[i] for i in mine))))
    if rank == 0:
        out.put(gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_partition_the_ensemble():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (a, ca), (b, cb) = gathered
    assert set(a).isdisjoint(b)
    assert sorted(a + b) == list(range(96))
    assert abs(ca - cb) / max(ca, cb) < 0.05
