"""The serving loop (rt_server_*): requests for several resident scenes, submitted together from
two threads, must each get exactly the hits that the same rays get traced alone with the same
kernel -- although the server splits them into chunks, packs chunks of different requests into
shared launches and runs its launch slots concurrently. Also: admission by the HBM budget,
the busy scene that cannot be removed, and the latency statistics."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H

pytestmark = pytest.mark.gpu


def _scenes():
    cubes, inst = S.cubes_instanced(20)
    inst.casts = (np.arange(len(inst)) % 3) != 1
    clusters = S.clusters(40_000, config=2)
    return [
        (A.LAYOUT_REFLECTION, A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(cubes.positions, cubes.indices)], inst)),
        (A.LAYOUT_GI, A.pack_scene(A.LAYOUT_GI, [A.Blas(clusters.positions, clusters.indices)], S.identity_instances(1))),
        (A.LAYOUT_REFLECTION, A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(clusters.positions, clusters.indices)],
                                           S.identity_instances(1))),
    ]


def _requests(n_scenes, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(24):
        n = int(rng.integers(0, 60_000)) if k % 7 else 0
        rays = H.random_rays(n, -60.0, 60.0, seed=seed * 100 + k, tmax=300.0) if n else np.zeros((0, 8), np.float32)
        out.append((int(rng.integers(0, n_scenes)), [A.CLOSEST, A.ANY_CASTERS, A.ANY_SKY][k % 3], rays))
    return out


@pytest.mark.parametrize("kernel", ["fast", "wide8"])
def test_results_alone_equal_results_in_the_mix(engine, kernel):
    import torch
    scenes = _scenes()
    reqs = _requests(len(scenes))
    # alone: each request traced by itself through the same kernel
    alone = []
    for sid, mode, rays in reqs:
        layout, words = scenes[sid]
        sc = engine.upload(layout, words)
        if kernel == "wide8":
            sc.prepare("wide8")
        if len(rays):
            h = engine.trace(sc, torch.from_numpy(rays).cuda(), mode, kernel)
            torch.cuda.synchronize()
            alone.append(h.cpu().numpy().view(np.uint32))
        else:
            alone.append(None)
        sc.release()
    # in the mix: two submitting threads, small launch slots (requests span and share them)
    srv = A.Server(engine, hbm_budget=8 << 30, launch_rays=50_000, slots=3, kernel=kernel)
    try:
        ids = [srv.add_scene(layout, words) for layout, words in scenes]
        tickets = [None] * len(reqs)

        def submit(parity):
            for k in range(parity, len(reqs), 2):
                sid, mode, rays = reqs[k]
                tickets[k] = srv.submit(ids[sid], rays, mode)

        threads = [threading.Thread(target=submit, args=(p,)) for p in (0, 1)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for k, t in enumerate(tickets):
            got = srv.wait(t)
            if alone[k] is None:
                assert got.size == 0
                continue
            assert np.array_equal(got.reshape(alone[k].shape), alone[k]), f"request {k} differs in the mix"
        st = srv.stats()
        assert st["requests"] == len(reqs) and st["rays"] == sum(len(r) for _, _, r in reqs)
        assert st["launches"] >= sum(len(r) for _, _, r in reqs) // 50_000
        assert 0.0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    finally:
        srv.close()


def test_admission_by_budget_and_busy_scene(engine):
    scenes = _scenes()
    slot_bytes = 50_000 * (32 + 40) + 16 * 4096
    srv = A.Server(engine, hbm_budget=2 * slot_bytes + 200_000, launch_rays=50_000, slots=2, kernel="fast")
    try:
        with pytest.raises(A.RtError, match="OOM"):  # the cluster scene does not fit what is left
            srv.add_scene(*scenes[2])
        assert srv.stats()["device_bytes"] == 2 * slot_bytes
    finally:
        srv.close()
    with pytest.raises(A.RtError, match="OOM"):  # slots alone over the budget
        A.Server(engine, hbm_budget=slot_bytes, launch_rays=50_000, slots=2, kernel="fast")
    srv = A.Server(engine, hbm_budget=4 << 30, launch_rays=1 << 20, slots=1, kernel="fast")
    try:
        sid = srv.add_scene(*scenes[2])
        rays = H.random_rays(2_000_000, -60.0, 60.0, seed=9, tmax=300.0)
        t = srv.submit(sid, rays, A.CLOSEST)
        with pytest.raises(A.RtError, match="BUSY"):
            srv.remove_scene(sid)
        srv.wait(t)
        srv.remove_scene(sid)
    finally:
        srv.close()


def test_a_bounded_wait_times_out_and_the_request_stays_waitable(engine):
    """rt_server_wait with a limit returns RT_ERR_TIMEOUT while the request runs and keeps it:
    a later wait returns its hits, equal to the rays traced alone."""
    import torch
    layout, words = _scenes()[2]
    rays = H.random_rays(3_000_000, -60.0, 60.0, seed=11, tmax=300.0)
    srv = A.Server(engine, hbm_budget=4 << 30, launch_rays=1 << 19, slots=2, kernel="fast")
    try:
        sid = srv.add_scene(layout, words)
        t = srv.submit(sid, rays, A.CLOSEST)
        with pytest.raises(A.RtError, match="TIMEOUT"):
            srv.wait(t, timeout_ms=0)  # 3M rays through two 512k-ray slots: not done at once
        got = srv.wait(t, timeout_ms=120_000)
        sc = engine.upload(layout, words)
        want = engine.trace(sc, torch.from_numpy(rays).cuda(), A.CLOSEST, "fast").cpu().numpy().view(np.uint32)
        sc.release()
        assert np.array_equal(got.reshape(want.shape), want)
        with pytest.raises(A.RtError, match="INVALID_ARG"):  # a ticket is waited for once
            srv.wait(t, timeout_ms=0)
    finally:
        srv.close()


@pytest.mark.parametrize("kernel", ["fast", "wide8"])
def test_a_failed_launch_fails_its_requests_and_the_server_carries_on(engine, kernel):
    """A slot launch that fails on the host (injected: a fake of a failing copy or launch call,
    no device fault) finishes every request with rays in that slot with the failure's status
    instead of hanging them; the slot returns to service, later requests get correct hits, and
    a submit for a scene that does not exist is refused at once."""
    import torch
    layout, words = _scenes()[1]
    rays = H.random_rays(120_000, -60.0, 60.0, seed=12, tmax=300.0)
    srv = A.Server(engine, hbm_budget=4 << 30, launch_rays=50_000, slots=1, kernel=kernel)
    try:
        sid = srv.add_scene(layout, words)
        srv.fail_next(1, 6)  # RT_ERR_CUDA
        t = srv.submit(sid, rays, A.CLOSEST)  # three slot launches: the first fails
        with pytest.raises(A.RtError, match="CUDA"):
            srv.wait(t, timeout_ms=120_000)
        small = rays[:40_000]
        t = srv.submit(sid, small, A.ANY_CASTERS)
        got = srv.wait(t, timeout_ms=120_000)
        sc = engine.upload(layout, words)
        if kernel == "wide8":
            sc.prepare("wide8")
        want = engine.trace(sc, torch.from_numpy(small).cuda(), A.ANY_CASTERS, kernel).cpu().numpy().view(np.uint32)
        sc.release()
        assert np.array_equal(got.reshape(want.shape), want)
        with pytest.raises(A.RtError, match="INVALID_ARG"):
            srv.submit(sid + 7, small, A.CLOSEST)
        assert srv.stats()["pending"] == 0
    finally:
        srv.close()
