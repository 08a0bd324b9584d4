"""bench.py --gpus N runs N independent replicas (the path has no exchange step to shard): the
job time is the max over ranks and the throughput is all ranks' work over it.  Checked with two
gloo ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t_ms = [100.0, 150.0][rank]
        work = [1.0e9, 3.0e9][rank]
        e2e = [5.0, 7.0][rank]
        out[rank] = bench.aggregate_replicas(dist, torch, "cpu", t_ms, work, e2e)
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        t_all, value, e2e = res[r]
        assert t_all == 150.0
        assert value == pytest.approx(4.0e9 / 0.150)
        assert e2e == 12.0
