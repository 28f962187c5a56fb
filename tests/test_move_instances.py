"""Moving instances of packed words on the host (rt_move_instances_host), checked against the
packer and the top-level refit: the moved records are the records rt_pack_scene writes for the
new placements, the top level keeps its topology and holds rt_tlas_refit's boxes (header word 3
counting refits, a rebuild after 64, as instance_bvh::place does for a moved set), and the
reflection scene bounds are the packer's."""
import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S


def _scene(layout, n=60, seed=0):
    rng = np.random.default_rng(seed)
    meshes = []
    for k, tris in enumerate((400, 150)):
        c = rng.uniform(-3, 3, (tris, 3)).astype(np.float32)
        pos = (c[:, None, :] + rng.normal(0, 0.4, (tris, 3, 3))).astype(np.float32).reshape(-1, 3)
        meshes.append(A.Blas(pos, np.arange(3 * tris, dtype=np.uint32)))
    return meshes, _placements(n, rng)


def _placements(n, rng):
    q = S.quaternion_matrices(S.Stream(int(rng.integers(1 << 30))), n)
    model = np.zeros((n, 3, 4), np.float32)
    model[:, :, :3] = q * rng.uniform(0.5, 2.0, (n, 1, 1))
    model[:, :, 3] = rng.uniform(-100, 100, (n, 3))
    return S.Instances(model.astype(np.float32), S.affine_inverse_rows(model.astype(np.float32)),
                       (np.arange(n) % 2).astype(np.uint32))


def _head(layout):
    return (16, 32) if layout == A.LAYOUT_GI else (8, 24)


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_moved_records_top_level_and_bounds(layout):
    meshes, inst = _scene(layout)
    words = A.pack_scene(layout, meshes, inst)
    boxes = A.object_boxes(layout, meshes)
    header, stride = _head(layout)
    n = len(inst)
    assert words[1] != 0  # 60 instances: the top level is on
    rng = np.random.default_rng(5)
    new = _placements(n, rng)
    new.mesh = inst.mesh.copy()
    moved = A.move_instances_host(layout, words, new, boxes)
    fresh = A.pack_scene(layout, meshes, new)  # the packer's records for the new placements
    rec = lambda w: w[header:header + stride * n].reshape(n, stride)
    assert np.array_equal(rec(moved)[:, :18], rec(fresh)[:, :18])
    assert np.array_equal(rec(moved)[:, 18:], rec(words)[:, 18:])  # the rest of each record stays
    base = int(words[1]) & ~3
    span = 32 * (n - 1)
    top_old = words[base:base + span]
    want = A.tlas_refit(top_old, np.concatenate([rec(moved)[:, 12:15], rec(moved)[:, 15:18]], 1).view(np.float32))
    assert np.array_equal(moved[base:base + span], want)
    assert moved[3] == words[3] + 1
    assert moved[0] == words[0]
    if layout == A.LAYOUT_REFLECTION:
        at = int(words[4])
        assert np.array_equal(moved[at:at + 8], fresh[int(fresh[4]):int(fresh[4]) + 8])


def test_the_top_level_is_rebuilt_after_64_refits():
    layout = A.LAYOUT_REFLECTION
    meshes, inst = _scene(layout, seed=2)
    words = A.pack_scene(layout, meshes, inst)
    boxes = A.object_boxes(layout, meshes)
    words[3] = 64
    rng = np.random.default_rng(9)
    new = _placements(len(inst), rng)
    new.mesh = inst.mesh.copy()
    moved = A.move_instances_host(layout, words, new, boxes)
    fresh = A.pack_scene(layout, meshes, new)
    base, span = int(words[1]) & ~3, 32 * (len(inst) - 1)
    assert moved[3] == 0 and np.array_equal(moved[base:base + span], fresh[base:base + span])


def test_moves_that_would_change_the_layout_are_refused():
    layout = A.LAYOUT_GI
    meshes, inst = _scene(layout, n=45, seed=3)
    words = A.pack_scene(layout, meshes, inst)
    boxes = A.object_boxes(layout, meshes)
    fewer = S.Instances(inst.model[:-1], inst.rows[:-1], inst.mesh[:-1])
    with pytest.raises(A.RtError, match="LAYOUT"):
        A.move_instances_host(layout, words, fewer, boxes)
    flat = S.Instances(inst.model.copy(), inst.rows.copy(), inst.mesh.copy())
    flat.model[3, :, :3] = 0.0  # singular
    with pytest.raises(A.RtError, match="LAYOUT"):
        A.move_instances_host(layout, words, flat, boxes)
