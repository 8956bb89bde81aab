"""Replicas on several GPUs: the bench's cross-rank steps (the job time is the
slowest rank's, throughput counts every rank's work) run here as two gloo
ranks on the CPU."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench._dist()
        t = bench.reduce_max(1.5 + 2.0 * rank, dist)  # rank 1 is the slower one
        q.put((r, w, local, t, bench.job_rate(w, 10, t)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_and_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == pytest.approx(3.5) for o in out)       # both ranks see the slowest time
    assert all(o[4] == pytest.approx(2 * 10 / 3.5) for o in out)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_max(4.25) == 4.25 and bench.job_rate(1, 8, 2.0) == 4.0
