"""The multi-GPU leg of bench.py is replicas only: each rank decomposes its own
copy and the step time is the max over ranks.  Checked with two gloo ranks on
CPU (the aggregation is backend-independent)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [12.5, 40.0][rank]
    worst = bench.replica_max(ms, world, torch.device("cpu"))
    dist.barrier()
    out[rank] = (worst, bench.replica_value(926648, world, worst))
    dist.destroy_process_group()


def test_two_rank_replica_aggregation():
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 40.0
    assert res[0][1] == pytest.approx(2 * 926648 / 0.040)


def test_single_rank_is_identity():
    import bench
    assert bench.replica_max(3.0, 1, None) == 3.0
    assert bench.replica_value(10, 1, 1000.0) == 10.0
