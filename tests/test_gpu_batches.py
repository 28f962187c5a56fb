"""Many batches in one persistent launch (rt_trace_batches) and prepared plans (rt_plan_*):
every batch's results must equal, word for word, what the same kernel writes for that batch
traced alone, whatever the mix of sizes (empty ones included) and modes in the launch, with or
without a ray sort, launched directly or replayed from a CUDA graph; and the FAST kernel's must
equal the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _scene_and_batches(layout, seed=3, modes="mixed"):
    """One cube BLAS under a top level of 900 instances (every fifth casts no shadow), and 9
    batches of uneven sizes (one empty) alternating closest / any hit."""
    mesh, inst = S.cubes_instanced(30)
    inst.casts = (np.arange(len(inst)) % 5) != 2
    words = A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], inst)
    prim = H.small_cubes(30, 96, 96)[1]
    rnd = H.random_rays(20_000, -40.0, 40.0, seed=seed, tmax=200.0)
    sizes = [1000, 0, 7, 4096, 1, 2500, 9216, 333, 5000]
    pool = np.concatenate([prim, rnd])
    rng = np.random.default_rng(seed)
    batches, start = [], 0
    for k, n in enumerate(sizes):
        idx = rng.integers(0, len(pool), n)
        mode = A.CLOSEST if k % 2 == 0 else (A.ANY_CASTERS if k % 4 == 1 else A.ANY_SKY)
        if modes != "mixed":  # every batch closest, or every batch any hit
            mode = A.CLOSEST if modes == "closest" else (A.ANY_CASTERS if k % 2 else A.ANY_SKY)
        batches.append((np.ascontiguousarray(pool[idx]), mode))
    return words, batches


def _device(batches):
    torch = _torch()
    return [(torch.from_numpy(r).cuda(), m) for r, m in batches]


def _alone(engine, scene, dev, kernel):
    torch = _torch()
    out = []
    for r, m in dev:
        out.append(engine.trace(scene, r, m, kernel) if r.shape[0] else None)
    torch.cuda.synchronize()
    return out


def _same(got, want, what):
    torch = _torch()
    for k, (g, w) in enumerate(zip(got, want)):
        if w is None:
            continue
        assert torch.equal(g, w), f"{what}: batch {k}: {(g != w).reshape(len(g), -1).any(1).sum().item()} rays differ"


@pytest.mark.parametrize("modes", ["mixed", "closest", "any"])
@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
@pytest.mark.parametrize("kernel", ["plain", "fast", "wide8"])
def test_batches_equal_alone(engine, layout, kernel, modes):
    torch = _torch()
    words, batches = _scene_and_batches(layout, modes=modes)
    scene = engine.upload(layout, words)
    try:
        if kernel == "wide8":
            scene.prepare("wide8")
        dev = _device(batches)
        want = _alone(engine, scene, dev, kernel)
        got = engine.trace_batches(scene, dev, kernel)
        torch.cuda.synchronize()
        _same(got, want, f"{kernel} one launch")
        if kernel != "wide8":  # and the oracle's, for the bit-exact kernels
            for (r, m), g in zip(batches, got):
                if len(r) == 0:
                    continue
                if layout == A.LAYOUT_GI:
                    w, _ = O.gi_trace(words, r, m)
                    w = (w[:, 1] != A.MISS).astype(np.uint32) if m else w
                else:
                    w, _ = O.rs_trace(words, r, m != 0)
                    w = (w[:, 1] != 0).astype(np.uint32) if m else w
                assert np.array_equal(g.cpu().numpy().view(np.uint32).reshape(w.shape), w)
    finally:
        scene.release()


@pytest.mark.parametrize("kernel", ["fast", "wide8"])
@pytest.mark.parametrize("order", ["none", "octant"])
def test_plan_graph_replays_and_follows_new_rays(engine, kernel, order):
    """A graph-captured plan replays the launch; new ray contents in the same buffers give the
    new results; a sorted plan gives the unsorted results."""
    torch = _torch()
    words, batches = _scene_and_batches(A.LAYOUT_REFLECTION)
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    try:
        scene.prepare("wide8")
        dev = _device(batches)
        plan = engine.plan(scene, dev, kernel, refill=8, order=order, graph=True)
        assert plan.info()["rays"] == sum(len(r) for r, _ in batches)
        for _ in range(2):
            plan.launch()
        torch.cuda.synchronize()
        _same(plan.hits, _alone(engine, scene, dev, kernel), f"{kernel} plan")
        _, other = _scene_and_batches(A.LAYOUT_REFLECTION, seed=11)
        for (r, _), (r2, _) in zip(dev, other):
            if r.shape[0]:
                r.copy_(torch.from_numpy(r2[: r.shape[0]]))
        plan.launch()
        torch.cuda.synchronize()
        _same(plan.hits, _alone(engine, scene, dev, kernel), f"{kernel} plan, new rays")
        plan.close()
    finally:
        scene.release()


def test_batch_rejections(engine):
    torch = _torch()
    words, batches = _scene_and_batches(A.LAYOUT_REFLECTION)
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    try:
        dev = _device(batches[:2])
        with pytest.raises(A.RtError, match="UNSUPPORTED"):
            engine.trace_batches(scene, dev, "wide8")  # not prepared
        r = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
        with pytest.raises(A.RtError, match="INVALID_ARG"):
            engine.trace_batches(scene, [(r.view(-1)[1:17].view(2, 8), A.CLOSEST)], "fast")  # 4-byte offset
        many = [(r, A.CLOSEST)] * (4096 + 1)
        with pytest.raises(A.RtError, match="INVALID_ARG"):
            engine.trace_batches(scene, many, "fast")
        assert engine.trace_batches(scene, [], "fast") == []
    finally:
        scene.release()


def test_tuner_plan_matches_plain(engine):
    """The autotuner's chosen plan (WIDE8 allowed) gives the plain kernel's hits, near ties
    aside, and its trial table covers both kernels."""
    from renderlab_b200 import tune as T
    torch = _torch()
    words, batches = _scene_and_batches(A.LAYOUT_REFLECTION)
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    try:
        scene.prepare("wide8")
        dev = _device(batches)
        ch = T.tune(engine, scene, dev, refills=(8, 32), orders=("none", "octant"), reps=1)
        # plain 1, fast 2 x 2, wide8 2 x 2 with the local stack and 2 unsorted with the shared one
        # (the cube BLAS is shallow), and the packet walk (over the top level too) with 2 orders
        assert {t.kernel for t in ch.trials} == {"plain", "fast", "wide8", "wide8p"} and len(ch.trials) == 13
        assert {t.stack for t in ch.trials if t.kernel == "wide8"} == {"local", "shared"}
        ch.plan.launch()
        torch.cuda.synchronize()
        plain = _alone(engine, scene, dev, "plain")
        for g, w in zip(ch.plan.hits, plain):
            if w is None:
                continue
            if w.dim() == 2:
                same = (g[:, 1:3] == w[:, 1:3]).all(1).float().mean().item()
            else:
                same = (g == w).float().mean().item()
            assert same >= 0.999, same
        ch.plan.close()
    finally:
        scene.release()
