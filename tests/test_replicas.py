"""Replica bookkeeping of multi-GPU runs, exercised on CPU with gloo ranks (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpu_recip_b200 import replicas as R


def test_partition_covers_every_unit_once():
    for n in (0, 1, 7, 256, 1001):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in R.partition(n, world, r)]
            assert got == list(range(n))
            sizes = [len(R.partition(n, world, r)) for r in range(world)]
            assert max(sizes) - min(sizes) <= (1 if n else 0)
    with pytest.raises(ValueError):
        R.partition(4, 2, 2)


def test_seeds_differ_per_rank_and_repeat():
    seeds = [R.replica_seed(11, r) for r in range(8)]
    assert len(set(seeds)) == 8
    assert seeds == [R.replica_seed(11, r) for r in range(8)]


def test_aggregate_rate():
    assert R.aggregate_rate([100, 100], 2.0) == 100.0
    with pytest.raises(ValueError):
        R.aggregate_rate([1], 0.0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    assert R.rank_world() == (rank, world, rank)
    assert R.init("gloo", timeout_s=60)
    R.barrier()
    # each rank "measures" a different time; every rank must see the slowest
    t = R.max_over_ranks(1.0 + rank)
    units = R.sum_over_ranks(len(R.partition(10, world, rank)))
    R.shutdown()
    out.put((rank, t, units))


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2.0, 10.0), (1, 2.0, 10.0)]
