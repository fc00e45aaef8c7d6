"""Replica aggregation across ranks (gloo, world size 2, CPU): max of device times, sum of
particles, as bench.py reports for --gpus N."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from ariel_b200.replicas import aggregate, replica_seed
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
    n = 1000 * (rank + 1)
    out[rank] = aggregate(ms, n, dist) + (replica_seed(rank),)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregation():
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0][:2] == (15.0, 3000) and out[1][:2] == (15.0, 3000)
    assert out[0][2] != out[1][2]


def test_single_process_is_identity():
    from ariel_b200.replicas import aggregate
    assert aggregate(7.5, 42) == (7.5, 42)
