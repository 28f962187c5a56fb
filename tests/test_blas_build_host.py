"""Host-side pins for the device builds' test inputs: the exponentially spaced mesh's SAH tree is
exactly 15 node levels deep at 350 triangles and passes 15 at 390, where build_bvh_sah falls
back to median splits (near_field.rs:184-190); the exponentially spaced boxes' top level fits a
48-entry stack at 200 boxes and not at 400 (instance_bvh.rs:346-366). So the GPU tests cover both
sides of each rule."""
from __future__ import annotations

import numpy as np

from renderlab_b200 import api as A

from .helpers import deep_sah_mesh


def test_deep_mesh_sits_on_both_sides_of_the_fallback():
    p, i = deep_sah_mesh(350)
    sah, med = A.Blas(p, i), A.Blas(p, i, median=True)
    assert sah.info()["depth"] == 15
    assert not np.array_equal(sah.nodes(), med.nodes())
    p, i = deep_sah_mesh(390)
    sah, med = A.Blas(p, i), A.Blas(p, i, median=True)
    assert np.array_equal(sah.nodes(), med.nodes()) and np.array_equal(sah.bvh_indices(), med.bvh_indices())


def test_deep_boxes_sit_on_both_sides_of_the_top_level_fallback():
    from .helpers import deep_tlas_boxes
    shallow, deep = deep_tlas_boxes(200), deep_tlas_boxes(400)
    assert not np.array_equal(A.tlas_build(shallow, True), A.tlas_build(shallow, False))
    assert np.array_equal(A.tlas_build(deep, True), A.tlas_build(deep, False))
