"""Shared scene/ray fixtures for the tests: small versions of the benchmark configurations and
the meshes the reference's own tests use."""
from __future__ import annotations

import numpy as np

from renderlab_b200 import scenes as S


def grid(n: int):
    """near_field.rs:634-651 / gi_bvh.rs:280-297: an n x n quad grid on y = 0."""
    p, i = [], []
    for y in range(n + 1):
        for x in range(n + 1):
            p.append([x / n, 0.0, y / n])
    for y in range(n):
        for x in range(n):
            a = y * (n + 1) + x
            b, c = a + 1, a + n + 1
            i += [a, c, b, b, c, c + 1]
    return np.array(p, np.float32), np.array(i, np.uint32)


def oracle_instances(inst: S.Instances, layout: int):
    n = len(inst)
    if layout == 0:
        aux = np.zeros((n, 9), np.uint32)
        aux[:, 4] = (~inst.casts).astype(np.uint32)  # extra word 27 bit 0: casts no shadow
    else:
        aux = np.stack([np.arange(n), inst.casts.astype(np.uint32)], axis=1).astype(np.uint32)
    return dict(model=inst.model, rows=inst.rows, mesh=inst.mesh, aux=aux)


def small_cubes(n_side=24, width=192, height=192):
    mesh = S.cubes_merged(n_side)
    rays = S.cube_camera_rays(width, height)
    # keep the camera framing of the full grid: scale the eye with the grid
    scale = n_side / 100.0
    rays[:, 0:3] *= scale
    return mesh, rays


def small_clusters(n_tris=60_000, width=256, height=256, config=2):
    mesh = S.clusters(n_tris, config=config)
    rays = S.cluster_camera_rays(width, height)
    return mesh, rays


def random_rays(n, lo, hi, seed=7, tmax=1e30):
    s = S.Stream(seed)
    o = s.range(lo, hi, n, 3)
    d = s.unit_vectors(n)
    return S.pack_rays(o, d, 0.0, tmax)


def deep_sah_mesh(n: int = 390):
    """Triangles at exponentially spaced x (x_i = 1.25^(0.999 i)): binned SAH peels a few off the
    far end at each split, so its tree passes 15 node levels and build_bvh_sah falls back to
    median splits (near_field.rs:184-190)."""
    x = np.power(np.float32(1.25), np.arange(n, dtype=np.float32) * np.float32(0.999)).astype(np.float32)
    p = np.zeros((3 * n, 3), np.float32)
    p[0::3, 0] = p[1::3, 0] = p[2::3, 0] = x
    p[1::3, 1] = 1.0
    p[2::3, 2] = 1.0
    return p, np.arange(3 * n, dtype=np.uint32)


def deep_tlas_boxes(n: int = 400):
    """Unit boxes at exponentially spaced x (x_i = 1.25^(i / 2)): instance_bvh's SAH peels a few off
    the far end at each split, so past about 300 boxes the collapsed tree is too deep for a
    48-entry stack and the build falls back to median splits (instance_bvh.rs:346-366)."""
    x = np.power(np.float32(1.25), np.arange(n, dtype=np.float32) * np.float32(0.5)).astype(np.float32)
    b = np.zeros((n, 6), np.float32)
    b[:, 0], b[:, 3] = x - np.float32(0.5), x + np.float32(0.5)
    b[:, 1] = b[:, 2] = np.float32(-0.5)
    b[:, 4] = b[:, 5] = np.float32(0.5)
    return b
