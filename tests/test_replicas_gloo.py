"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks (no GPU).

bench.py runs N independent replicas (the path does not shard); the job's
time is the slowest rank's, taken by an all-reduce MAX, and the throughput is
N x the units each rank processed over that time.  The reference arm runs on
rank 0 only.
"""

import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(0.5 + rank, world, "cpu")
        out.put((rank, t, bench.job_throughput(3, t, world)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the max (1.5 s) and the job throughput 2 x 3 units / 1.5 s
    assert [r[1] for r in res] == [1.5, 1.5]
    assert all(r[2] == pytest.approx(4.0) for r in res)


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(0.25, 1, "cpu") == 0.25
    assert bench.job_throughput(3, 0.25, 1) == pytest.approx(12.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference(None) is None  # returns before reading its arguments
    assert capsys.readouterr().out == ""
