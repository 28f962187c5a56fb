"""Host-side pins for the device build's test meshes: the exponentially spaced mesh's SAH tree is
exactly 15 node levels deep at 350 triangles and passes 15 at 390, where build_bvh_sah falls
back to median splits (near_field.rs:184-190), so the GPU test covers both sides of that rule."""
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
