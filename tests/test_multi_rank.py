"""The benchmark's multi-rank plumbing on CPU: two gloo ranks (one process each, as torchrun
launches them) set up the process group the way bench.py does, meet at its barrier and agree on
the max-over-ranks step time that the whole-job value is computed from."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    assert dist.get_backend() == "gloo"  # no CUDA device here
    dist.barrier()
    ms = bench.max_over_ranks(10.0 + rank)  # each rank's mean step time
    out.put((rank, ms))
    dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_step():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0), (1, 11.0)]
