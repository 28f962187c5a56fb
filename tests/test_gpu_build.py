"""GPU BLAS build (rt_blas_build_device): the binned-SAH / median BVH4-Q8 built level by level on
the device must equal the host build (near_field::build_bvh_sah / build_bvh restated:
rt_blas_build) word for word: node records, reordered indices, leaves and their source offsets
(through the RLB image, which carries all of them). The meshes cover ranges split by several
blocks and by one, bin and centroid ties, signed zeros, shared vertices, identical triangles
(median splits inside an SAH build, past one block's size), meshes of one leaf and of two, and a
mesh whose SAH tree passes 15 node levels and is rebuilt by median splits."""
from __future__ import annotations

import numpy as np
import pytest

from renderlab_b200 import api as A
from renderlab_b200 import cooked as C
from renderlab_b200 import scenes as S

from .helpers import deep_sah_mesh

pytestmark = pytest.mark.gpu


def _soup(rng, n, lo=-10.0, hi=10.0):
    p = rng.uniform(lo, hi, (3 * n, 3)).astype(np.float32)
    return p, np.arange(3 * n, dtype=np.uint32)


def meshes():
    rng = np.random.default_rng(5)
    out = {}
    m = S.clusters(200_000, config=2)
    out["clusters_200k"] = (m.positions, m.indices)
    m = S.clusters(20_000, config=3)
    out["clusters_20k"] = (m.positions, m.indices)
    p, i = _soup(rng, 6000)
    out["rounded"] = (np.round(p).astype(np.float32), i)
    p, i = _soup(rng, 4000)
    p[:, 1] = np.where(rng.random(len(p)) < 0.5, np.float32(0.0), np.float32(-0.0))
    out["signed_zeros"] = (p, i)
    out["shared_vertices"] = (rng.uniform(-10, 10, (64, 3)).astype(np.float32),
                              rng.integers(0, 64, 3 * 20_000).astype(np.uint32))
    tri = rng.uniform(-1, 1, (3, 3)).astype(np.float32)
    out["identical_5000"] = (np.tile(tri, (5000, 1)), np.arange(15000, dtype=np.uint32))
    for n in (1, 5, 8, 9, 17):
        out[f"soup_{n}"] = _soup(rng, n)
    out["deep_15_levels"] = deep_sah_mesh(350)
    out["deep_fallback"] = deep_sah_mesh(390)
    return out


def _same(host: A.Blas, dev: A.Blas, name: str):
    assert dev.info() == host.info(), name
    assert np.array_equal(dev.nodes(), host.nodes()), name
    assert np.array_equal(dev.bvh_indices(), host.bvh_indices()), name
    assert C.encode_rlb(dev, 1 << 40) == C.encode_rlb(host, 1 << 40), name


@pytest.mark.parametrize("median", [False, True])
def test_device_build_equals_host_build(engine, median):
    for name, (p, i) in meshes().items():
        _same(A.Blas(p, i, median=median), A.Blas.build_device(engine, p, i, median=median), name)


def test_device_build_rejects_what_the_host_rejects(engine):
    p = np.zeros((3, 3), np.float32)
    for bad_p, bad_i in ((p, np.zeros(0, np.uint32)), (p, np.arange(4, dtype=np.uint32)),
                         (p, np.array([0, 1, 3], np.uint32)), (np.full((3, 3), np.inf, np.float32), np.arange(3, dtype=np.uint32))):
        with pytest.raises(A.RtError):
            A.Blas.build_device(engine, bad_p, bad_i)


def test_device_build_traces_like_the_host_build(engine):
    import torch
    m = S.clusters(100_000, config=2)
    inst = S.identity_instances(1)
    host = A.pack_scene(A.LAYOUT_GI, [A.Blas(m.positions, m.indices)], inst)
    dev = A.pack_scene(A.LAYOUT_GI, [A.Blas.build_device(engine, m.positions, m.indices)], inst)
    assert np.array_equal(host, dev)
    scene = engine.upload(A.LAYOUT_GI, dev)
    try:
        rays = torch.from_numpy(S.cluster_camera_rays(256, 256)).cuda()
        hits = engine.trace(scene, rays, A.CLOSEST, "plain")
        assert int((hits.view(torch.int32)[:, 1] != -1).sum()) > 0
    finally:
        scene.release()
