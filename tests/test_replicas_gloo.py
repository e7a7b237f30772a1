"""Host logic of the multi-GPU benchmark (independent replicas, one process per GPU): the job's time is the
slowest rank's and the value aggregates all replicas. Run here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")  # rank 1 is the slower replica
        out[rank] = (ms, bench.replica_value(4, world, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_aggregate_value():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms, value = res[0]
    assert ms == 15.0
    assert value == pytest.approx(4 * 2 / 0.015)


def test_single_process_passthrough():
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.replica_value(10, 1, 100.0) == pytest.approx(100.0)
