"""The N > 1 path of bench.py on CPU: two gloo ranks (one process each, rendezvous on
127.0.0.1) run the replica plumbing -- barrier, max-over-ranks timing and the whole-job
rate -- with no data exchanged between replicas."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    w, r, local = bench.dist_setup(world, backend="gloo")
    bench.barrier(w)
    ms = 10.0 + 5.0 * r  # rank 1 is the slower one
    slowest = bench.max_over_ranks(ms, w)
    rate = bench.job_rate(w, 1000, 20, slowest)
    q.put((r, local, w, slowest, rate))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for r, (rank, local, world, slowest, rate) in enumerate(out):
        assert (rank, local, world) == (r, r, 2)
        assert slowest == 15.0
        # 2 ranks x 1000 units x 20 steps in 15 ms
        assert abs(rate - 2 * 1000 * 20 / 0.015 / 1e6) < 1e-9


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    assert bench.dist_setup(1, backend="gloo") == (1, 0, 0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_rate(1, 2_097_152, 2000, 416.0) == pytest.approx(10082.46, rel=1e-5)
