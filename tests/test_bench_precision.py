"""The benchmark's FP64 classification (bench.fp64_classify) on hand-made records: a matching hit
is status 0 with its t and barycentric errors, a differing hit within 1e-6 of FP64's t a near tie,
anything else unexplained; any-hit flags differ acceptably only where FP64's hit lies within 1e-5
of tmin or tmax."""
from __future__ import annotations

import numpy as np

import bench


def _rs(t, slot, prim, u, v):
    r = np.zeros(5, np.uint32)
    r[0] = np.float32(t).view(np.uint32)
    r[1], r[2] = slot, prim
    r[3], r[4] = np.float32(u).view(np.uint32), np.float32(v).view(np.uint32)
    return r


def test_closest_hit_classes():
    got = np.stack([_rs(2.0, 1, 7, 0.25, 0.5),          # the FP64 hit
                    _rs(3.0, 1, 8, 0.1, 0.1),           # another triangle at FP64's t (a tie)
                    _rs(4.0, 1, 9, 0.1, 0.1),           # another triangle, farther: unexplained
                    _rs(1e30, 0, 0, 0.0, 0.0)])         # a miss where FP64 hits: unexplained
    r64 = np.array([[1, 2.0000001, 0.2500001, 0.5], [1, 3.000001, 0.1, 0.1], [1, 3.0, 0.1, 0.1],
                    [1, 5.0, 0.3, 0.3]], np.float64)
    ident = np.zeros((4, 6), np.uint32)
    ident[:, 2] = 1
    ident[:, 3] = [7, 9, 8, 4]
    rays = np.zeros((4, 8), np.float32)
    status, t_rel, bary = bench.fp64_classify(1, 0, got, rays, r64, ident)
    assert status.tolist() == [0, 1, 2, 2]
    assert abs(t_rel[0] - 0.1 / 2.0000001 * 1e-6) < 1e-9 and np.isnan(t_rel[1:]).all()
    assert bary[0] < 1e-6 and np.isnan(bary[1:]).all()


def test_any_hit_classes():
    rays = np.zeros((3, 8), np.float32)
    rays[:, 7] = 10.0
    got = np.array([1, 0, 0], np.uint32)
    r64 = np.array([[1, 4.0, 0, 0], [1, 9.99999, 0, 0], [1, 5.0, 0, 0]], np.float64)
    status, _, _ = bench.fp64_classify(1, 2, got, rays, r64, np.zeros((3, 6), np.uint32))
    assert status.tolist() == [0, 1, 2]
