"""rt_trace_static, the allocation-free entry point.

It serves callers that cannot allocate device memory while they trace: an engine whose frame
loop forbids cudaMalloc, or a renderer that keeps the packed words in its own device buffer and
never creates an rt_ctx. Its only scratch (the persistent warps' ray counter and the overflow
count) is a static device array shared by every call. This test calls it through the C ABI twice
in a row on caller-owned device buffers and requires each result to equal, bit for bit, what
the context-based FAST traversal (rt_trace_ex) returns for the same rays; it also checks that a
batch above RT_STATIC_MAX_RAYS is refused before anything runs. It passes on its own in a fresh
process and after the rest of the suite."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _scene(layout):
    mesh = S.clusters(40_000, config=2)
    words = A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    A.validate(layout, words)
    rays = S.cluster_camera_rays(192, 192)
    return words, rays


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_static_trace_matches_context_trace_twice(layout):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    words, rays = _scene(layout)
    d_words = torch.from_numpy(words.view(np.int32)).cuda()  # the caller's own buffer
    d_rays = torch.from_numpy(rays).cuda()
    engine = A.Engine(0)
    scene = engine.upload(layout, words)
    try:
        for mode in (A.CLOSEST, A.ANY_CASTERS):
            want = engine.trace(scene, d_rays, mode, "fast")
            torch.cuda.synchronize()
            for _ in range(2):  # the shared scratch starts from zero on every call
                got = A.trace_static(layout, d_words, d_rays, mode)
                torch.cuda.synchronize()
                assert torch.equal(got, want), f"mode {mode}: {(got != want).sum().item()} words differ"
    finally:
        scene.release()
        engine.close()


def test_static_trace_refuses_oversized_batches():
    lib = A.lib()
    big = A.STATIC_MAX_RAYS + 1
    st = lib.rt_trace_static(A.LAYOUT_REFLECTION, ctypes.c_void_p(16), 64, A.CLOSEST, ctypes.c_void_p(16),
                             ctypes.c_void_p(16), ctypes.c_uint32(big), None)
    assert st == 1  # RT_ERR_INVALID_ARG, before any device access
