"""GPU top-level build (rt_tlas_build_device): instance_bvh's SAH / median binary tree, collapsed
into BVH4 nodes, built level by level on the device, must give rt_tlas_build's node words exactly.
The boxes cover random placements at 10k and 100k instances, many equal centres, identical boxes
(median splits inside an SAH build, in shared memory and past it), zero-area boxes, signed zeros,
two to five instances, and a set whose SAH tree is too deep for a 48-entry stack (the median
rebuild)."""
from __future__ import annotations

import numpy as np
import pytest

from renderlab_b200 import api as A

from .helpers import deep_tlas_boxes

pytestmark = pytest.mark.gpu


def box_sets():
    rng = np.random.default_rng(9)

    def placed(n, half=500.0, lo=0.5, hi=4.0):
        c = rng.uniform(-half, half, (n, 3)).astype(np.float32)
        h = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
        return np.concatenate([c - h, c + h], 1).astype(np.float32)

    out = {"random_10k": placed(10_000), "random_100k": placed(100_000)}
    b = placed(20_000)
    c = np.round((b[:, :3] + b[:, 3:]) / 200.0) * 100.0
    out["equal_centres"] = np.concatenate([c - 1.0, c + 1.0], 1).astype(np.float32)
    out["identical_3000"] = np.tile(np.array([[-1, -1, -1, 1, 1, 1]], np.float32), (3000, 1))
    out["identical_9000"] = np.tile(np.array([[-1, -2, -3, 1, 2, 3]], np.float32), (9000, 1))
    b = placed(5000)
    b[:, 1] = b[:, 4]
    b[:, 2] = b[:, 5]
    out["zero_area"] = b
    b = placed(5000)
    z = np.where(rng.random(5000) < 0.5, np.float32(0.0), np.float32(-0.0))
    b[:, 1] = b[:, 4] = z
    out["signed_zeros"] = b
    for n in (2, 3, 5):
        out[f"n{n}"] = placed(n)
    out["deep_fallback"] = deep_tlas_boxes(400)
    out["deep_no_fallback"] = deep_tlas_boxes(200)
    return out


@pytest.mark.parametrize("sah", [True, False])
def test_device_top_level_equals_host(engine, sah):
    for name, boxes in box_sets().items():
        want = A.tlas_build(boxes, sah)
        got = A.tlas_build_device(engine, boxes, sah)
        assert got.shape == want.shape and np.array_equal(got, want), name


def test_device_top_level_needs_two_boxes(engine):
    with pytest.raises(A.RtError):
        A.tlas_build_device(engine, np.zeros((1, 6), np.float32))
