"""Multi-GPU path of the benchmark on CPU: two ranks over gloo.  NRG runs do
not shard, so N GPUs run N replicas; the only exchange is the max over ranks
of the timed spans, and the whole-job value is N x runs / slowest span."""
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


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # replica spans differ per rank; every rank must see the slowest
        spans = bench.max_over_ranks(dist, [10.0 + rank, 20.0 - rank], "cpu")
        q.put((rank, spans))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got[0] == got[1] == [11.0, 20.0]


def test_replica_value_is_weak_scaling_sum():
    one = bench.replica_value(1, 128, 40.0)
    assert bench.replica_value(2, 128, 40.0) == pytest.approx(2 * one)
    # a slower replica sets the span of the whole job
    assert bench.replica_value(2, 128, 80.0) == pytest.approx(one)
