"""The GI cache's ray producers on the GPU: a cell's 64 fixed directions (gi_direction about
gi_basis of its normal, from gi_origin_offset) must equal the oracle's restatement bit for bit;
and traced inside the FAST kernel (no ray buffer) they must give exactly the hits of the same rays
traced from a buffer, and the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H

pytestmark = pytest.mark.gpu


def _cells(mesh, rays, n):
    import torch
    words = A.pack_scene(A.LAYOUT_GI, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1),
                         primitives=[True])
    h, _ = O.gi_trace(words, rays, 0)
    hit = h[:, 1] != A.MISS
    pts = S.hit_points(rays[hit], h[hit, 0].view(np.float32))[:n]
    nrm = S.triangle_normals(mesh, h[hit, 2])[:n]
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    cells = S.gi_cells(pts, nrm, 0.5, S.Stream(21))
    return words, cells, torch.from_numpy(cells.view(np.int32)).cuda()


@pytest.mark.parametrize("rotate", [False, True])
def test_cell_rays_equal_the_oracle(engine, rotate):
    mesh, rays = H.small_clusters(20_000, 96, 96)
    _, cells, d_cells = _cells(mesh, rays, 600)
    got = engine.gi_cell_rays(d_cells, rotate).cpu().numpy()
    want = O.gi_cell_rays(cells, rotate)
    assert got.shape == want.shape == (len(cells) * 64, 8)
    bad = np.nonzero((got.view(np.uint32) != want.view(np.uint32)).any(axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} rays differ; first {bad[:3]}: {got[bad[:1]]} vs {want[bad[:1]]}"
    assert np.allclose(np.linalg.norm(want[:, 4:7], axis=1), 1.0, atol=1e-5)


@pytest.mark.parametrize("mode", [A.CLOSEST, A.ANY_SKY])
def test_cells_traced_in_the_kernel_equal_buffered_rays_and_the_oracle(engine, mode):
    import torch
    mesh, rays = H.small_clusters(20_000, 96, 96)
    words, cells, d_cells = _cells(mesh, rays, 600)
    scene = engine.upload(A.LAYOUT_GI, words)
    try:
        fused = engine.trace_gi_cells(scene, d_cells, mode, rotate=True)
        produced = engine.gi_cell_rays(d_cells, rotate=True)
        buffered = engine.trace(scene, produced, mode, "fast")
        torch.cuda.synchronize()
        assert torch.equal(fused, buffered)
        want, _ = O.gi_trace(words, produced.cpu().numpy(), mode)
        if mode:
            want = (want[:, 1] != A.MISS).astype(np.uint32)
        got = fused.cpu().numpy().view(np.uint32)
        assert np.array_equal(got.reshape(want.shape), want)
        if mode == A.CLOSEST:
            assert 0.05 < (want[:, 1] != A.MISS).mean() < 0.95
    finally:
        scene.release()
