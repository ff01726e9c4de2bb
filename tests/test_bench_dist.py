"""The multi-rank path of bench.py on the CPU (world size 2, gloo): the path shards with no
exchange step, so N ranks run N replicas of the map; the only collectives are the barrier
and the max-over-ranks reduction of the timings, and rank 0 alone prints. The reference
arm runs on rank 0 only; the other ranks exit 0 without work."""
import multiprocessing as mp
import os
import socket
import subprocess
import sys
from datetime import timedelta
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        env = bench.dist_env()
        slowest = bench.max_over_ranks(100.0 + 25.0 * rank, world)   # this rank's step ms
        e2e = bench.max_over_ranks(7.0 - rank, world)
        dist.barrier()
        q.put((rank, env, slowest, e2e, bench.aggregate_rate(world, 1024 * 1024, slowest)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_max_and_aggregate_the_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (env, slowest, e2e, rate) for r, env, slowest, e2e, rate in out}
    for r in (0, 1):
        env, slowest, e2e, rate = by_rank[r]
        assert env == (r, 2, r)
        assert slowest == 125.0 and e2e == 7.0          # both ranks see the slowest rank
        assert rate == pytest.approx(2 * 1024 * 1024 / 0.125)   # two replicas' cells


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.aggregate_rate(1, 1000, 500.0) == 2000.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
