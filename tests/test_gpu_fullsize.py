"""Size-independent properties at the benchmark's full size: the clusters-1M scene (1,000,000
triangles, reflection layout) with 4,194,304 primaries (2048 x 2048) and 4,194,304 GI hemisphere
rays from their hits, the step bench.py times. The oracle is too slow for this size. So the
checks are properties that hold at any size; the smaller parity tests pin each one against the
oracle:
- FAST equals PLAIN bit for bit: both restate rs_trace exactly;
- the host-buffer pipeline returns the device path's bits;
- a ray permutation changes no result;
- WIDE8 finds PLAIN's closest primitive on all but a few rays, with t within 1e-5 relative,
  for both of its walks (one ray per lane, and warp-wide packets). WIDE8 uses conservative
  boxes and breaks ties in f64, so it may differ from PLAIN's f32 arithmetic; every ray where it
  does goes to the FP64 oracle, and WIDE8 must agree with FP64 there (a near tie aside) -- the
  difference is then PLAIN's f32 error, which the reference's arithmetic shares. A strided
  sample of 16,384 rays of each batch is checked against FP64 too (ids, t, barycentrics)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from .test_gpu_wide8 import check_closest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def clusters_1m(engine):
    import torch
    mesh = S.clusters(1_000_000, config=2)
    words = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    primary = S.cluster_camera_rays(2048, 2048)
    h = engine.trace(scene, torch.from_numpy(primary).cuda(), A.CLOSEST, "plain").cpu().numpy().view(np.uint32)
    hit = h[:, 1] != 0
    t, prim = h[:, 0].view(np.float32), h[:, 2]
    pts = S.hit_points(primary[hit], t[hit])
    normals = S.triangle_normals(mesh, prim[hit])
    gi = S.hemisphere_rays(pts, normals, primary[hit, 4:7], len(primary), S.Stream(S.seed_for(2) + 1))
    assert len(primary) == len(gi) == 4_194_304 and hit.mean() > 0.2
    yield scene, primary, gi, words
    scene.release()


def _trace(engine, scene, rays, kernel, order=None):
    import torch
    return engine.trace(scene, torch.from_numpy(rays).cuda(), A.CLOSEST, kernel, order=order).cpu().numpy().view(np.uint32)


def test_fast_equals_plain_at_full_size(engine, clusters_1m):
    scene, primary, gi, _ = clusters_1m
    for rays in (primary, gi):
        assert np.array_equal(_trace(engine, scene, rays, "fast"), _trace(engine, scene, rays, "plain"))


def test_host_pipeline_and_ray_order_change_no_result_at_full_size(engine, clusters_1m):
    import torch
    scene, primary, gi, _ = clusters_1m
    want = [_trace(engine, scene, r, "fast") for r in (primary, gi)]
    got = engine.trace_host_batches(scene, [(primary, A.CLOSEST, "fast"), (gi, A.CLOSEST, "fast")])
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g).reshape(w.shape), w)
    order = engine.order(scene, torch.from_numpy(gi).cuda(), "octant")
    assert np.array_equal(np.sort(order.cpu().numpy().view(np.uint32)), np.arange(len(gi), dtype=np.uint32))
    assert np.array_equal(_trace(engine, scene, gi, "fast", order=order), want[1])


@pytest.mark.parametrize("kernel", ["wide8", "wide8p"])
def test_wide8_agrees_with_plain_at_full_size(engine, clusters_1m, kernel):
    scene, primary, gi, words = clusters_1m
    scene.prepare("wide8")
    for what, rays in (("primary", primary), ("gi", gi)):
        p, w = _trace(engine, scene, rays, "plain"), _trace(engine, scene, rays, kernel)
        same = (p[:, 1] == w[:, 1]) & (p[:, 2] == w[:, 2])
        assert same.mean() >= 0.9999, same.mean()
        both = same & (p[:, 1] != 0)
        tp, tw = p[both, 0].view(np.float32).astype(np.float64), w[both, 0].view(np.float32).astype(np.float64)
        rel = np.abs(tw - tp) / np.maximum(tp, 1e-30)
        assert np.mean(rel <= 1e-5) >= 0.9999, np.quantile(rel, 0.9999)
        # every disagreement with PLAIN, settled by FP64
        diff = np.nonzero(~same)[0]
        if len(diff):
            ref, ident = O.fp64_trace(words, rays[diff], A.LAYOUT_REFLECTION)
            check_closest(A.LAYOUT_REFLECTION, w[diff], ref, ident, f"{kernel} {what}: rays differing from PLAIN")
        smp = np.arange(0, len(rays), len(rays) // 16_384)
        ref, ident = O.fp64_trace(words, rays[smp], A.LAYOUT_REFLECTION)
        stats = check_closest(A.LAYOUT_REFLECTION, w[smp], ref, ident, f"{kernel} {what}: strided sample")
        print(f"{kernel} {what}: {len(diff)} rays differ from PLAIN; sample t max/mean, ties, bary max: {stats}")
