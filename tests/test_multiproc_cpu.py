"""Multi-process host paths on CPU (gloo, world size 2, 127.0.0.1)."""
from __future__ import annotations

import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, out):
    from psierra_b200.batched import partition_instances

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = partition_instances(sizes, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine.tolist())
        # the benchmark's timing rule: every rank's device time, reduced with MAX
        t = torch.tensor([1.5 + rank, 2.0 * (world - rank)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = (gathered, t.tolist())
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_and_max_over_ranks():
    from psierra_b200 import meshgen

    sizes = [c.mesh.n_elements for c in meshgen.beam_batch(n=40, target_tets=1e5, seed=3)]
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), sizes, out), nprocs=world, join=True)
    g0, t0 = out[0]
    g1, t1 = out[1]
    assert g0 == g1  # every rank computes the same partition
    allidx = sorted(g0[0] + g0[1])
    assert allidx == list(range(len(sizes)))  # complete and disjoint
    load = [sum(sizes[i] for i in part) for part in g0]
    assert max(load) - min(load) <= max(sizes)  # greedy balance bound
    assert t0 == t1 == [2.5, 4.0]
