"""Moving instances on the device (rt_scene_move_instances): the scene's words equal the host
move's (rt_move_instances_host), bit for bit, over moves in a row (the top level refit each time,
header word 3 counting), across the rebuild after 64 refits (made on the device) and over the
refits after it (in the rebuilt tree's level order); traced rays see the moved scene as the
oracle does; and the 8-wide walk, derived before the moves, finds the same triangles after them,
through the packed top level while its own 8-wide top level is stale and through the rebuilt one
after a new prepare."""
import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A

from . import helpers as H
from .test_move_instances import _placements, _scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_device_move_equals_the_host_move(engine, layout):
    import torch
    meshes, inst = _scene(layout, n=64, seed=4)
    words = A.pack_scene(layout, meshes, inst)
    boxes = A.object_boxes(layout, meshes)
    scene = engine.upload(layout, words)
    scene.prepare("wide8")  # derived before the moves: they must not invalidate it
    try:
        host = words
        rng = np.random.default_rng(21)
        for step in range(5):
            new = _placements(len(inst), rng)
            new.mesh = inst.mesh.copy()
            if step == 2:  # the refit count at its limit: the next move rebuilds the top level
                host = host.copy()
                host[3] = 64
                scene.update_records(host[:8])
            host = A.move_instances_host(layout, host, new, boxes)
            scene.move_instances(new, boxes)
            torch.cuda.synchronize()
            dev = scene.words()
            assert np.array_equal(dev, host), f"move {step}: {int((dev != host).sum())} words differ"
        # rays through the moved scene: the oracle's hits over the host-moved words
        rays = H.random_rays(20_000, -120.0, 120.0, seed=8, tmax=500.0)
        got = engine.trace(scene, torch.from_numpy(rays).cuda(), A.CLOSEST, "fast").cpu().numpy().view(np.uint32)
        want = (O.gi_trace(host, rays, 0) if layout == A.LAYOUT_GI else O.rs_trace(host, rays, False))[0]
        assert np.array_equal(got.reshape(want.shape), want)
        assert (want[:, 1] != (A.MISS if layout == A.LAYOUT_GI else 0)).any()
        # the 8-wide walk over the moved records and top level finds the same closest triangles
        w8 = engine.trace(scene, torch.from_numpy(rays).cuda(), A.CLOSEST, "wide8").cpu().numpy().view(np.uint32)
        ids = slice(1, 5) if layout == A.LAYOUT_GI else slice(1, 3)
        same = (w8.reshape(want.shape)[:, ids] == want[:, ids]).all(axis=1)
        assert same.mean() >= 0.999, same.mean()
        # the moves left the 8-wide top level stale (the walk read the packed one); preparing again
        # rebuilds it from the moved records, and the walk through it returns the same records
        scene.prepare("wide8")
        again = engine.trace(scene, torch.from_numpy(rays).cuda(), A.CLOSEST, "wide8").cpu().numpy().view(np.uint32)
        assert np.array_equal(again, w8)
    finally:
        scene.release()
