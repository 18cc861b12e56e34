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


def test_bench_gpus_flag_means_replicas():
    """`bench.py --gpus N` starts N rank processes itself unless a launcher already did; a
    launcher world size other than N is refused."""
    import bench
    assert bench.replica_plan(1, {}) == ("run", 1)
    assert bench.replica_plan(4, {}) == ("spawn", 4)
    assert bench.replica_plan(2, {"WORLD_SIZE": "2"}) == ("run", 2)
    assert bench.replica_plan(1, {"WORLD_SIZE": "1"}) == ("run", 1)
    with pytest.raises(SystemExit):
        bench.replica_plan(8, {"WORLD_SIZE": "2"})
    cmd = bench.torchrun_command(["--gpus", "2", "--steps", "5"], 2, 29555)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=2" in cmd and "--master-addr=127.0.0.1" in cmd and "--master-port=29555" in cmd
    assert cmd[-4:] == ["--gpus", "2", "--steps", "5"] and cmd[-5].endswith("bench.py")


def _bench_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    assert bench.replica_plan(world) == ("run", world)
    assert R.init("gloo", timeout_s=60)
    # rank r timed 10 (r + 1) ms for 100 evaluations: the job took the slowest rank's 20 ms and
    # did 200 evaluations
    total_ms, value = bench.rank_summary(10.0 * (rank + 1), 100, world)
    R.shutdown()
    out.put((rank, total_ms, value))


def test_bench_rank_summary_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for _, total_ms, value in res:
        assert total_ms == 20.0 and abs(value - 200 / 0.020) < 1e-6



def test_bench_fft_schedule_pins_without_autotuning():
    """`--fft-schedule` (for profilers that cannot launch the cluster build) pins the y/z
    schedule on every handle the bench makes and skips the autotuner; `auto` autotunes."""
    import bench

    class FakeHandle:
        def __init__(self):
            self.calls = []

        def set_fft_schedule(self, s):
            self.calls.append(("schedule", s))

        def autotune(self, *a, **k):
            self.calls.append(("autotune",))
            return {"schedule": 0}

        def get_tune_config(self):
            return {"schedule": 0, "x_lines": 16, "y_lines": 16, "z_columns": 16, "grid_ctas": 0}

    class Args:
        fft_schedule = "passes"

    h = FakeHandle()
    tune = bench.tune_single(h, Args(), [1.0] * 3, None, 0, 0.3, 3)
    assert ("autotune",) not in h.calls and tune["schedule"] == bench.SCHEDULES["passes"] and tune["pinned"]
    Args.fft_schedule = "auto"
    h = FakeHandle()
    assert bench.tune_single(h, Args(), [1.0] * 3, None, 0, 0.3, 3) == {"schedule": 0}
    assert h.calls == [("autotune",)]
    assert set(bench.SCHEDULES) == {"auto", "planes", "passes", "cluster"}
