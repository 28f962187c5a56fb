"""GPU refit (rt_scene_refit): new positions for a BLAS of an uploaded scene, refit on the device,
must give exactly the words of the host refit (near_field::refit_bvh restated: rt_blas_refit)
followed by packing: node boxes, quantised planes and (reflection) pre-edged triangles, bit for
bit; other meshes untouched; and, once the records are rewritten, traversal equal to a fresh
upload of the host-packed words."""
from __future__ import annotations

import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H

pytestmark = pytest.mark.gpu


def _mesh_base(layout, words):
    """Word offset of the first mesh: everything before it is header, records and top level."""
    return int(words[16 + 18]) if layout == A.LAYOUT_GI else int(words[8 + 18]) & ~3


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_gpu_refit_equals_host_refit(engine, layout):
    import torch
    moving = S.clusters(30_000, config=2)
    still, _ = H.small_cubes(6)
    inst = S.identity_instances(2)
    b_moving, b_still = A.Blas(moving.positions, moving.indices), A.Blas(still.positions, still.indices)
    w0 = A.pack_scene(layout, [b_moving, b_still], inst)
    scene = engine.upload(layout, w0)
    idx = torch.from_numpy(moving.indices.view(np.int32)).cuda()
    rng = np.random.default_rng(11)
    try:
        for step in range(2):  # the second call reuses the cached topology
            new = (moving.positions + rng.normal(0, 0.2, moving.positions.shape)).astype(np.float32)
            new[::97] *= np.float32(1.5)  # and some large moves
            b_moving.refit(new)
            want = A.pack_scene(layout, [b_moving, b_still], inst)
            scene.refit(0, torch.from_numpy(new).cuda(), idx if layout == A.LAYOUT_REFLECTION else None)
            torch.cuda.synchronize()
            got = scene.words()
            base = _mesh_base(layout, want)
            bad = np.nonzero(got[base:] != want[base:])[0]
            assert len(bad) == 0, f"step {step}: {len(bad)} words differ, first at {base + bad[:5]}"
            scene.update_records(want[:base])
            fresh = engine.upload(layout, want)
            try:
                rays = torch.from_numpy(S.cluster_camera_rays(128, 128)).cuda()
                for mode in (A.CLOSEST, A.ANY_CASTERS):
                    a = engine.trace(scene, rays, mode, "plain")
                    b = engine.trace(fresh, rays, mode, "plain")
                    assert torch.equal(a, b)
            finally:
                fresh.release()
    finally:
        scene.release()


def test_gpu_refit_rejections_and_wide8(engine):
    import torch
    mesh, _ = H.small_clusters(5_000)
    w = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    scene = engine.upload(A.LAYOUT_REFLECTION, w)
    try:
        scene.prepare("wide8")
        pos = torch.from_numpy(mesh.positions).cuda()
        with pytest.raises(A.RtError, match="INVALID_ARG"):
            scene.refit(0, pos)  # the reflection layout needs the triangle list
        with pytest.raises(A.RtError, match="INVALID_ARG"):
            scene.refit(5, pos, torch.from_numpy(mesh.indices.view(np.int32)).cuda())
        scene.refit(0, pos, torch.from_numpy(mesh.indices.view(np.int32)).cuda())
        rays = torch.from_numpy(S.cluster_camera_rays(32, 32)).cuda()
        with pytest.raises(A.RtError, match="UNSUPPORTED"):  # the 8-wide layout was dropped
            engine.trace(scene, rays, A.CLOSEST, "wide8")
        scene.prepare("wide8")
        engine.trace(scene, rays, A.CLOSEST, "wide8")
    finally:
        scene.release()
