"""Replica plumbing on CPU: two gloo ranks, each with its own timing, agree on the
max-over-ranks time and the whole-job throughput (the bench's multi-GPU arithmetic)."""
from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from fire_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=30)
    r.barrier()
    seconds = 1.0 + rank  # rank 1 is the slow one
    out.put((rank, r.max(seconds), r.throughput(1_000_000, 10, seconds)))
    r.close()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=60) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [m for _, m, _ in res] == [2.0, 2.0]
    # 2 ranks x 1e6 cells x 10 steps over the slowest rank's 2 s
    assert all(abs(t - 0.01) < 1e-12 for _, _, t in res)


def test_single_process_needs_no_group():
    os.environ.pop("WORLD_SIZE", None)
    from fire_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.world == 1 and r.max(3.5) == 3.5 and abs(r.throughput(100, 2, 0.5) - 4e-7) < 1e-18
    r.close()
