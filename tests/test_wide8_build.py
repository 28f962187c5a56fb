"""The engine's derived 8-wide layout, built on the host and checked without a GPU
(rt_wide8_check): every child box encloses its child in exact arithmetic, every triangle sits in
exactly one leaf, indices are in range, empty slots are inverted boxes, and the recorded depth is
the tree's. Also the sizes that the SAH-optimal collapse and one-triangle leaves give."""
import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S


def _blob(seed, tris):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-50, 50, (tris, 3)).astype(np.float32)
    pos = (centres[:, None, :] + rng.normal(0, 0.7, (tris, 3, 3))).astype(np.float32).reshape(-1, 3)
    return pos, np.arange(3 * tris, dtype=np.uint32)


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_cluster_soup_layout_checks(layout):
    mesh = S.clusters(20_000, config=2)
    w = A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    info = A.wide8_check(layout, w)
    assert info["triangles"] == 20_000 and info["blas"] == 1
    # one-triangle leaves: every triangle is a slot of its own, so nodes hold > 4 children on average
    assert (info["triangles"] + info["nodes"] - 1) / info["nodes"] > 4.0
    assert 1 < info["depth"] <= 16


def test_instanced_meshes_share_their_blas():
    a, b = _blob(1, 3000), _blob(2, 500)
    meshes = [A.Blas(*a), A.Blas(*b)]
    n = 50
    model = np.zeros((n, 3, 4), np.float32)
    model[:, 0, 0] = model[:, 1, 1] = model[:, 2, 2] = 1.0
    model[:, :, 3] = np.arange(n)[:, None] * np.array([7.0, 0.0, -3.0], np.float32)
    inst = S.Instances(model, S.affine_inverse_rows(model), (np.arange(n) % 2).astype(np.uint32))
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        info = A.wide8_check(layout, A.pack_scene(layout, meshes, inst))
        assert info["blas"] == 2 and info["triangles"] == 3500


def test_degenerate_and_tiny_meshes():
    # one triangle; a flat grid (zero extent on an axis); coincident centroids
    one = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.arange(3, dtype=np.uint32))
    g = np.array([[x, 0.0, z] for z in range(9) for x in range(9)], np.float32)
    gi = np.array([[a, a + 9, a + 1, a + 1, a + 9, a + 10] for a in [z * 9 + x for z in range(8) for x in range(8)]],
                  np.uint32).reshape(-1)
    same = (np.tile(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), (40, 1)) +
            np.repeat(np.linspace(-1e-3, 1e-3, 40, dtype=np.float32), 3)[:, None] * np.array([0, 0, 1], np.float32),
            np.arange(120, dtype=np.uint32))
    for pos, idx in (one, (g, gi), same):
        w = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(pos, idx)], S.identity_instances(1))
        info = A.wide8_check(A.LAYOUT_REFLECTION, w)
        assert info["triangles"] == len(idx) // 3


def test_the_check_rejects_what_the_upload_rejects():
    w = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(*_blob(3, 200))], S.identity_instances(1))
    bad = w.copy()
    bad[0] = 1 << 20  # more instance records than words
    with pytest.raises(A.RtError, match="LAYOUT"):
        A.wide8_check(A.LAYOUT_REFLECTION, bad)


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_top_level_encloses_every_instance(layout):
    """Scenes with a top level also get an 8-wide one over the instances' world boxes: the check
    walks it from its root and requires every instance in exactly one leaf, every child box to
    enclose the world boxes below it in exact arithmetic, and the depth the walk's stack allows --
    for 900 cube instances and for rotated, scaled instances of several meshes."""
    mesh, inst = S.cubes_instanced(30)
    A.wide8_check(layout, A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], inst))
    ms = S.multi_blas(n_blas=6, n_instances=2_000, tri_lo=500.0, tri_hi=4_000.0, config=9)
    w = A.pack_scene(layout, [A.Blas(m.positions, m.indices) for m in ms.meshes], ms.instances)
    assert w[1] != 0
    info = A.wide8_check(layout, w)
    assert info["blas"] == 6
