"""Ray sharding across ranks (renderlab_b200.shard) on CPU: two gloo ranks, one process each as
torchrun launches them, each with a replica of the scene and the oracle's traversal as its
per-rank tracer. The hits gathered from the two slices -- contiguous, or in the Morton order of
the origins, gathered to every rank or to one -- must equal, bit for bit, the hits of the whole
batch traced by one rank, for closest and any-hit queries and a batch that does not split
evenly."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from renderlab_b200 import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    from renderlab_b200 import api as A
    from renderlab_b200 import scenes as S
    from tests import helpers as H
    mesh, rays = H.small_cubes(24, 64, 48)
    words = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    rnd = H.random_rays(1_001, -24.0, 24.0, seed=3, tmax=300.0)
    return words, np.concatenate([rays, rnd])


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from oracle import oracle as O
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    words, rays = _workload()

    def trace(r, mode):  # this rank's tracer: the oracle over its scene replica
        h, _ = O.rs_trace(words, r.numpy(), mode != 0, threads=2)
        if mode:  # any hit: the engine's one word a ray, 1 when something blocks it
            return torch.from_numpy((h[:, 1] != 0).astype(np.int32))
        return torch.from_numpy(h.view(np.int32))

    res = {}
    for order in (None, "origin"):
        t = shard.ShardedTrace(trace, order=order)
        res[(order, "closest")] = t(rays, 0, 5).numpy()
        res[(order, "any")] = t(rays, 2, 1).numpy()
        g = t(rays, 0, 5, dst=1)
        res[(order, "dst")] = None if g is None else g.numpy()
    out.put((rank, res))
    dist.destroy_process_group()


def test_slices_cover_the_batch_once():
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            b = [shard.slice_bounds(n, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[k][1] == b[k + 1][0] for k in range(world - 1))
            assert max(hi - lo for lo, hi in b) - min(hi - lo for lo, hi in b) <= 1
    with pytest.raises(ValueError):
        shard.slice_bounds(10, 2, 2)


def test_morton_order_is_a_permutation_that_groups_origins():
    rng = np.random.default_rng(1)
    rays = np.zeros((4096, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-50, 50, (4096, 3))
    p = shard.morton_order(rays)
    assert np.array_equal(np.sort(p), np.arange(4096))
    o = rays[p, 0:3]
    # consecutive rays in Morton order are far closer than consecutive rays in random order
    assert np.linalg.norm(np.diff(o, axis=0), axis=1).mean() < 0.25 * np.linalg.norm(np.diff(rays[:, 0:3], axis=0),
                                                                                      axis=1).mean()


def test_two_ranks_gather_the_hits_of_one():
    import torch.multiprocessing as mp

    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    words, rays = _workload()
    assert len(rays) % 2 == 1  # the batch does not split evenly
    want_c = O.rs_trace(words, rays, False)[0].view(np.int32)
    want_a = (O.rs_trace(words, rays, True)[0][:, 1] != 0).astype(np.int32)
    assert 0.1 < (want_c[:, 1] != 0).mean() < 0.9 and 0.05 < want_a.mean() < 0.95
    for rank in (0, 1):
        for order in (None, "origin"):
            assert np.array_equal(got[rank][(order, "closest")], want_c), (rank, order)
            assert np.array_equal(got[rank][(order, "any")].reshape(-1), want_a), (rank, order)
        assert (got[rank][(None, "dst")] is None) == (rank != 1)
    assert np.array_equal(got[1][("origin", "dst")], want_c)
