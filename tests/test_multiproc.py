"""Replica aggregation of bench.py on two CPU ranks (gloo): the whole-job
value uses the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import bench
    total, value = bench.aggregate_ranks(100.0 * (rank + 1), steps=5, world_size=world, device="cpu")
    out[rank] = (total, value)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_value_uses_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    for r in (0, 1):
        total, value = res[r]
        assert total == pytest.approx(200.0)
        assert value == pytest.approx(2 * 5 / 0.2)
