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


def _lights(n: int, seed: int = 5) -> np.ndarray:
    """n light records (rt_gi_light, 20 words): point lights with and without a range, spot
    lights with cones of several widths, directional lights, and a few black ones (which reach
    nothing), around the small cluster scene."""
    s = S.Stream(seed)
    out = np.zeros((n, 20), np.uint32)
    for l in range(n):
        f = np.zeros(20, np.float32)
        kind = (0, 1, 1, 2)[l % 4]
        f[0:3] = s.range(-120.0, 120.0, 1, 3)[0]
        f[3] = 0.0 if l % 3 == 0 else float(s.range(20.0, 300.0, 1)[0])
        d = s.unit_vectors(1)[0]
        f[4:7] = d
        f[7] = float(s.range(-0.2, 0.95, 1)[0])
        f[8:11] = 0.0 if l % 7 == 5 else 1.0
        w = f.view(np.uint32).copy()
        w[12] = kind
        out[l] = w
    return out


@pytest.mark.parametrize("kernel", ["fast", "wide8"])
def test_light_visibility_words_equal_the_oracle(engine, kernel):
    """gi_light's words traced on the device, rays made in the ray refill: FAST must equal the
    oracle's words bit for bit (the same f32 arithmetic); WIDE8 must equal the FP64 oracle's
    visibility on every (cell, light) pair except where the FP64 hit lies within 1e-5 relative of
    the ray's tmin or tmax. 40 lights: two words a cell."""
    import torch
    mesh, rays = H.small_clusters(20_000, 96, 96)
    words, cells, d_cells = _cells(mesh, rays, 700)
    lights = _lights(40)
    scene = engine.upload(A.LAYOUT_GI, words)
    try:
        if kernel == "wide8":
            scene.prepare("wide8")
        got = engine.trace_gi_lights(scene, d_cells, torch.from_numpy(lights.view(np.int32)).cuda(), kernel)
        got = got.cpu().numpy().view(np.uint32)
        assert got.shape == (len(cells), 2)
        lrays, affects = O.gi_light_rays(cells, lights)
        if kernel == "fast":
            want = O.gi_light_bits(words, cells, lights)
            assert np.array_equal(got, want), f"{int((got != want).sum())} words differ"
        else:
            ref, _ = O.fp64_trace(words, lrays, A.LAYOUT_GI, any_hit=True)
            visible = affects.reshape(-1) & ~(ref[:, 0] > 0)
            bit = np.array([(got[i // 40, (i % 40) // 32] >> ((i % 40) % 32)) & 1 for i in range(len(lrays))], bool)
            t64 = ref[:, 1]
            near = (ref[:, 0] > 0) & (np.abs(t64 - lrays[:, 7]) <= 1e-5 * np.abs(lrays[:, 7]))
            bad = np.nonzero((bit != visible) & ~near)[0]
            assert len(bad) == 0, f"{len(bad)} of {len(lrays)} pairs differ from FP64; first {bad[:4]}"
        vis = np.unpackbits(got.view(np.uint8), bitorder="little").reshape(len(cells), -1)[:, :40]
        assert 0.05 < vis.mean() < 0.95 and affects.mean() > vis.mean()
    finally:
        scene.release()
