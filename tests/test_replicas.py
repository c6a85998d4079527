"""Multi-GPU runs are independent replicas (the multiply path has no exchange
step): bench.py combines them as all ranks' work over the slowest rank's
time.  Checked here with world_size 2 on the gloo backend (CPU)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    units = 1000.0 * (rank + 1)          # rank 0 did 1000 units, rank 1 2000
    ms = 10.0 * (rank + 1)               # in 10 ms and 20 ms
    out[rank] = (bench.allreduce_max(dist, ms), bench.allreduce_sum(dist, units),
                 bench.replica_value(dist, units, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_combination_gloo():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        mx, sm, val = out[r]
        assert mx == 20.0 and sm == 3000.0
        assert val == pytest.approx(3000.0 / 0.020)


def test_single_process_combination():
    import bench
    assert bench.allreduce_max(None, 5.0) == 5.0
    assert bench.replica_value(None, 100.0, 10.0) == pytest.approx(10000.0)
