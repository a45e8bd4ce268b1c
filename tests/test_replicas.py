"""The multi-GPU legs of bench.py: the single-graph form is replicas only (each
rank decomposes its own copy, the step time is the max over ranks); the batched
and served forms split their independent graphs / requests over the ranks and
pool the per-rank results.  Checked with two gloo ranks on CPU (the aggregation
is backend-independent)."""
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


def _shard_worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = bench.shard(range(11), rank, world)
    # each rank reports the items it handled; every rank receives all of them
    out[rank] = (mine, bench.gather_values([10 * i for i in mine], world),
                 bench.gather_values([{"launches": 3 + rank}], world))
    dist.destroy_process_group()


def test_two_rank_shard_and_gather():
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_shard_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == [0, 2, 4, 6, 8, 10] and res[1][0] == [1, 3, 5, 7, 9]
    # the shares are disjoint and cover every item once
    assert sorted(res[0][0] + res[1][0]) == list(range(11))
    for r in (0, 1):
        assert sorted(res[r][1]) == [10 * i for i in range(11)]
        assert res[r][2] == [{"launches": 3}, {"launches": 4}]


def test_single_rank_is_identity():
    import bench
    assert bench.replica_max(3.0, 1, None) == 3.0
    assert bench.replica_value(10, 1, 1000.0) == 10.0
    assert bench.shard(range(4), 0, 1) == [0, 1, 2, 3]
    assert bench.gather_values((1, 2), 1) == [1, 2]
