"""The multi-rank path of bench.py on CPU: two gloo ranks in separate processes (replicas only: no data-path
collective; the ranks agree on the slowest rank's time and the job's throughput sums every rank's work), the
environment parsing torchrun feeds it, and the reference arm's non-zero ranks leaving at once."""
from __future__ import annotations

import datetime
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, lr = bench.ranks_from_env()
        ms = 10.0 + 5.0 * rank                     # rank 1 is the slow one
        dist.barrier()
        m = bench.max_over_ranks(ms, "cpu")
        q.put((r, w, lr, m, bench.job_rate(100.0, w, m)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[:3] for r in res] == [(0, 2, 0), (1, 2, 1)]
    for r in res:
        assert r[3] == 15.0                               # max over ranks
        assert r[4] == pytest.approx(100.0 * 2 / 15e-3)  # both ranks' units over the slowest time


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, "cpu") == 12.5
    assert bench.job_rate(3.0, 1, 1000.0) == 3.0


def test_reference_arm_non_zero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == ""
