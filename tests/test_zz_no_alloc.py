"""rt_trace_static, the allocation-free entry point.

It serves callers that cannot allocate device memory while they trace: an engine whose frame
loop forbids cudaMalloc, or a renderer that keeps the packed words in its own device buffer and
never creates an rt_ctx. Its only scratch (the persistent warps' ray counter and the overflow
count) is a static device array shared by every call. These tests call it through the C ABI
twice in a row on caller-owned device buffers and require each result to equal, bit for bit,
what the context-based FAST traversal (rt_trace_ex) returns for the same rays: on a flat
cluster scene and on instanced cubes under a top level, in all three query modes. They also
check that its overflow count reads back as the context counts it, and that an oversized batch
or a misaligned hit buffer is refused before anything runs. They pass on their own in a fresh
process and after the rest of the suite."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _clusters(layout):
    mesh = S.clusters(40_000, config=2)
    words = A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    rays = S.cluster_camera_rays(192, 192)
    return words, rays


def _instanced(layout):
    """30 x 30 cube instances: past the 40 instances a top level needs (instance_bvh.rs:72)."""
    mesh, inst = S.cubes_instanced(30)
    inst.casts = (np.arange(len(inst)) % 5) != 2
    words = A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], inst)
    rays = S.cube_camera_rays(160, 160)
    rays[:, 0:3] *= 0.3
    return words, rays


def _torch_or_skip():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("scene_kind", ["clusters", "instanced"])
@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_static_trace_matches_context_trace_twice(layout, scene_kind):
    torch = _torch_or_skip()
    words, rays = (_clusters if scene_kind == "clusters" else _instanced)(layout)
    info = A.validate(layout, words)
    if scene_kind == "instanced":
        assert info["top"] != 0, "the instanced scene must carry a top level"
    d_words = torch.from_numpy(words.view(np.int32)).cuda()  # the caller's own buffer
    d_rays = torch.from_numpy(rays).cuda()
    engine = A.Engine(0)
    scene = engine.upload(layout, words)
    try:
        for mode in (A.CLOSEST, A.ANY_SKY, A.ANY_CASTERS):
            want = engine.trace(scene, d_rays, mode, "fast")
            torch.cuda.synchronize()
            for _ in range(2):  # the shared scratch starts from zero on every call
                got = A.trace_static(layout, d_words, d_rays, mode)
                torch.cuda.synchronize()
                assert torch.equal(got, want), f"mode {mode}: {(got != want).sum().item()} words differ"
                assert A.trace_static_stack_drops() == 0
    finally:
        scene.release()
        engine.close()


def test_static_trace_reports_its_stack_drops():
    """A BLAS deeper than the 48-entry stack: the static call drops the same pushes a context
    counts, and the count reads back until the next call zeroes it."""
    torch = _torch_or_skip()
    from .test_gpu_parity import deep_chain_scene
    words = deep_chain_scene(depth=24)
    rays = np.array([[0.5, 0.5, -5.0, 0.0, 0.0, 0.0, 1.0, 1e30]] * 32, np.float32)
    d_words = torch.from_numpy(words.view(np.int32)).cuda()
    d_rays = torch.from_numpy(rays).cuda()
    engine = A.Engine(0)
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    try:
        before = engine.stats()["stack_overflows"]
        want = engine.trace(scene, d_rays, A.CLOSEST, "fast")
        torch.cuda.synchronize()
        counted = engine.stats()["stack_overflows"] - before
        assert counted > 0
        for _ in range(2):
            got = A.trace_static(A.LAYOUT_REFLECTION, d_words, d_rays, A.CLOSEST)
            assert A.trace_static_stack_drops() == counted
            assert torch.equal(got, want)
    finally:
        scene.release()
        engine.close()


def test_static_trace_refuses_oversized_batches():
    lib = A.lib()
    big = A.STATIC_MAX_RAYS + 1
    st = lib.rt_trace_static(A.LAYOUT_REFLECTION, ctypes.c_void_p(16), 64, A.CLOSEST, ctypes.c_void_p(16),
                             ctypes.c_void_p(16), ctypes.c_uint32(big), None)
    assert st == 1  # RT_ERR_INVALID_ARG, before any device access


def test_static_trace_refuses_a_misaligned_hit_buffer():
    """Hits are written as 4-byte words: a hit pointer off that boundary is refused before any
    launch, and the context stays usable (the next call succeeds)."""
    torch = _torch_or_skip()
    words, rays = _clusters(A.LAYOUT_REFLECTION)
    d_words = torch.from_numpy(words.view(np.int32)).cuda()
    d_rays = torch.from_numpy(rays).cuda()
    n = len(rays)
    hits = torch.zeros(n * 5 + 1, dtype=torch.int32, device="cuda")
    st = A.lib().rt_trace_static(A.LAYOUT_REFLECTION, d_words.data_ptr(), d_words.numel(), A.CLOSEST,
                                 d_rays.data_ptr(), hits.data_ptr() + 2, ctypes.c_uint32(n), None)
    assert st == 1  # RT_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert int(hits.abs().sum().item()) == 0  # nothing was written
    got = A.trace_static(A.LAYOUT_REFLECTION, d_words, d_rays, A.CLOSEST)
    torch.cuda.synchronize()
    assert int((got[:, 1] != 0).sum().item()) > 0
