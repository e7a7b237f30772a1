"""Host logic of the multi-GPU benchmark, one process per GPU: independent replicas of the cross (the job's
time is the slowest rank's and the value aggregates all replicas) and the batched workload split between
ranks (every problem solved by exactly one rank, the split balanced by cells, the value from the slowest
rank). Run here as two gloo ranks on the CPU."""
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
    with mp.get_context("spawn").Manager() as m:
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


def _shard_rank(rank, world, port, out):
    from focalors_poisson_b200 import workloads as W

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        probs = W.batched_uneven(bench.BATCH_PROBLEMS, bench.SEED, rhs=False)[0]
        cells = [g.cells() for g in probs]
        mine = bench.partition_problems(cells, world)[rank]
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        my_cells = sum(cells[p] for p in mine)
        ms = bench.max_over_ranks(1e-6 * my_cells, dist, "cpu")  # a rank's time grows with its cells
        out[rank] = (shares, my_cells, ms, bench.sharded_value(bench.BATCH_PROBLEMS, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_batched_problems_split_between_ranks():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_shard_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    shares = res[0][0]
    assert shares == res[1][0]  # every rank computed the same split without communicating it
    together = sorted(p for s in shares for p in s)
    assert together == list(range(bench.BATCH_PROBLEMS))  # each problem exactly once
    c0, c1 = res[0][1], res[1][1]
    assert abs(c0 - c1) <= 0.01 * (c0 + c1)  # balanced by cells
    assert res[0][2] == res[1][2] == pytest.approx(1e-6 * max(c0, c1))  # the slowest rank's time
    assert res[0][3] == pytest.approx(bench.BATCH_PROBLEMS / (1e-6 * max(c0, c1) / 1e3))


def test_partition_single_rank_and_balance():
    cells = [5, 1, 4, 4, 3, 2]
    assert bench.partition_problems(cells, 1) == [list(range(6))]
    parts = bench.partition_problems(cells, 3)
    assert sorted(p for x in parts for p in x) == list(range(6))
    assert sorted(sum(cells[p] for p in x) for x in parts) == [6, 6, 7]
