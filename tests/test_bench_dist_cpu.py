"""The multi-rank timing of bench.py (one replica per rank, no data-path collective): the
reported time is the slowest rank's and the rate counts every rank's elements.  Two gloo
ranks on the CPU."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    import bench
    local_ms = 100.0 + 50.0 * rank                 # rank 1 is slower
    t = bench.max_over_ranks(local_ms, ws, "cpu")
    q.put((rank, t, bench.job_rate(1000, ws, 10, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, rate in got:
        assert t == pytest.approx(150.0)
        assert rate == pytest.approx(2 * 1000 * 10 / 0.150)


def test_single_rank_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.job_rate(100, 1, 4, 200.0) == pytest.approx(2000.0)
