"""GPU parity: the CUDA kernels against the oracle's restatement of the WGSL loops, through the
C ABI. Integer results (hit ids, records, flags) and float results (t, barycentrics, normals) of
the PLAIN and FAST kernels must be bit-identical to the oracle's."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H

pytestmark = pytest.mark.gpu

BIT_EXACT_KERNELS = ["plain", "fast"]


def _torch():
    import torch
    return torch


def product_words(layout, meshes, inst, tlas_mode=-1, primitives=None):
    return A.pack_scene(layout, [A.Blas(m.positions, m.indices) for m in meshes], inst, tlas_mode, primitives)


def oracle_words(layout, meshes, inst, tlas_mode=-1, primitives=None):
    ms = [(m.positions, m.indices, 1 if (primitives and primitives[k]) else 0) for k, m in enumerate(meshes)]
    return O.scene_words(layout, ms, H.oracle_instances(inst, layout), tlas_mode)


def gpu_trace(engine, scene, rays, mode, kernel):
    torch = _torch()
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    h = engine.trace(scene, r, mode, kernel)
    torch.cuda.synchronize()
    return h.cpu().numpy().view(np.uint32)


def check_same(got, want, what):
    got = got.reshape(want.shape)
    bad = np.nonzero((got != want).reshape(len(want), -1).any(axis=1))[0]
    assert len(bad) == 0, f"{what}: {len(bad)}/{len(want)} rays differ; first {bad[:5]}: {got[bad[:2]]} vs {want[bad[:2]]}"


def test_selftest_conventions(engine):
    """Device arithmetic matches the oracle's conventions: IEEE 754-2019 signed-zero min/max,
    correctly rounded reciprocal / square root, no flush of subnormals."""
    out = engine.selftest()
    f = out.view(np.float32)
    assert out[0] == 0x80000000 and out[1] == 0x80000000, f"fminf(+-0) -> {out[0]:#x} {out[1]:#x}"
    assert out[2] == 0 and out[3] == 0, f"fmaxf(+-0) -> {out[2]:#x} {out[3]:#x}"
    assert f[4] == np.float32(1.0) / np.float32(3.0)
    assert f[5] == np.sqrt(np.float32(2.0))
    assert f[7] == f[4]
    assert f[6] == np.float32(2.0 ** 127) and f[8] == np.float32(2.0 ** -127)


@pytest.mark.parametrize("kernel", BIT_EXACT_KERNELS)
@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_cubes_closest_and_sun(engine, layout, kernel):
    """Config 1 at reduced size: primaries closest-hit, then one sun any-hit ray per hit."""
    mesh, rays = H.small_cubes()
    inst = S.identity_instances(1)
    w = product_words(layout, [mesh], inst)
    assert np.array_equal(w, oracle_words(layout, [mesh], inst))
    scene = engine.upload(layout, w)
    try:
        got = gpu_trace(engine, scene, rays, A.CLOSEST, kernel)
        if layout == A.LAYOUT_GI:
            want, _ = O.gi_trace(w, rays, 0)
            hit = want[:, 1] != A.MISS
        else:
            want, _ = O.rs_trace(w, rays, False)
            hit = want[:, 1] != 0
        check_same(got, want, "closest")
        assert hit.mean() > 0.3
        t = want[hit, 0].view(np.float32)
        sun = S.sun_rays(S.hit_points(rays[hit], t))
        got_any = gpu_trace(engine, scene, sun, A.ANY_CASTERS, kernel)
        if layout == A.LAYOUT_GI:
            w_any, _ = O.gi_trace(w, sun, 2)
            want_any = (w_any[:, 1] != A.MISS).astype(np.uint32)
        else:
            w_any, _ = O.rs_trace(w, sun, True)
            want_any = (w_any[:, 1] != 0).astype(np.uint32)
        check_same(got_any, want_any, "sun any-hit")
        assert 0.0 < want_any.mean() < 1.0
    finally:
        scene.release()


@pytest.mark.parametrize("kernel", BIT_EXACT_KERNELS)
@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_instanced_cubes_top_level(engine, layout, kernel):
    """Config 1b at reduced size: one cube BLAS under a BVH4 top level of 900 instances, some
    of which cast no shadow."""
    mesh, inst = S.cubes_instanced(30)
    inst.casts = (np.arange(len(inst)) % 5) != 2
    w = product_words(layout, [mesh], inst)
    assert np.array_equal(w, oracle_words(layout, [mesh], inst))
    assert w[1] != 0
    rays = H.small_cubes(30, 160, 160)[1]
    scene = engine.upload(layout, w)
    try:
        for mode in (A.CLOSEST, A.ANY_SKY, A.ANY_CASTERS):
            got = gpu_trace(engine, scene, rays, mode, kernel)
            if layout == A.LAYOUT_GI:
                want, _ = O.gi_trace(w, rays, mode)
                if mode:
                    want = (want[:, 1] != A.MISS).astype(np.uint32)
            else:
                want, _ = O.rs_trace(w, rays, mode != 0)
                if mode:
                    want = (want[:, 1] != 0).astype(np.uint32)
            check_same(got, want, f"mode {mode}")
    finally:
        scene.release()


@pytest.mark.parametrize("kernel", BIT_EXACT_KERNELS)
@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_clusters_primary_and_gi(engine, layout, kernel):
    """Config 2 at reduced size: coherent primaries, then cosine-hemisphere GI rays from hits."""
    mesh, rays = H.small_clusters()
    inst = S.identity_instances(1)
    prims = [True] if layout == A.LAYOUT_GI else None
    w = product_words(layout, [mesh], inst, primitives=prims)
    assert np.array_equal(w, oracle_words(layout, [mesh], inst, primitives=prims))
    scene = engine.upload(layout, w)
    try:
        got = gpu_trace(engine, scene, rays, A.CLOSEST, kernel)
        want, _ = (O.gi_trace(w, rays, 0) if layout == A.LAYOUT_GI else O.rs_trace(w, rays, False))
        check_same(got, want, "primary")
        hit = want[:, 1] != (A.MISS if layout == A.LAYOUT_GI else 0)
        prim = want[hit, 2] if layout == A.LAYOUT_GI else want[hit, 2]
        pts = S.hit_points(rays[hit], want[hit, 0].view(np.float32))
        gi = S.hemisphere_rays(pts, S.triangle_normals(mesh, prim), rays[hit, 4:7], 40_000, S.Stream(99))
        got = gpu_trace(engine, scene, gi, A.CLOSEST, kernel)
        want, _ = (O.gi_trace(w, gi, 0) if layout == A.LAYOUT_GI else O.rs_trace(w, gi, False))
        check_same(got, want, "gi")
    finally:
        scene.release()


@pytest.mark.parametrize("kernel", BIT_EXACT_KERNELS)
def test_edge_rays(engine, kernel):
    """Axis-aligned and zero-component directions, tmax = inf and FLT_MAX, tmin > tmax, origins
    on box planes, and an empty batch."""
    p, i = H.grid(12)
    mesh = S.Mesh(p, i)
    inst = S.identity_instances(1)
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        w = product_words(layout, [mesh], inst)
        scene = engine.upload(layout, w)
        try:
            rays = []
            for d in ([0, -1, 0], [0, 1, 0], [1, 0, 0], [0.3, -1, 0], [0, -1, 1e-31], [1e-35, -1, 0]):
                for o in ([0.5, 1, 0.5], [0.0, 0.5, 0.0], [0.25, 0.0, 0.25], [1.0, 2.0, 1.0]):
                    for tmin, tmax in ((0.0, 1e30), (0.0, np.inf), (0.0, 3.4028235e38), (0.5, 0.25), (1e-4, 10.0)):
                        rays.append([*o, tmin, *d, tmax])
            rays = np.array(rays, np.float32)
            for mode in (A.CLOSEST, A.ANY_CASTERS):
                got = gpu_trace(engine, scene, rays, mode, kernel)
                if layout == A.LAYOUT_GI:
                    want, _ = O.gi_trace(w, rays, mode)
                    if mode:
                        want = (want[:, 1] != A.MISS).astype(np.uint32)
                else:
                    want, _ = O.rs_trace(w, rays, mode != 0)
                    if mode:
                        want = (want[:, 1] != 0).astype(np.uint32)
                check_same(got, want, f"edge rays layout {layout} mode {mode}")
            torch = _torch()
            empty = torch.zeros((0, 8), dtype=torch.float32, device="cuda")
            assert engine.trace(scene, empty, A.CLOSEST, kernel).shape[0] == 0
        finally:
            scene.release()


def test_empty_scene_and_rejections(engine):
    """A scene with no instances misses everything; malformed words are refused at upload."""
    inst = S.Instances(np.zeros((0, 3, 4), np.float32), np.zeros((0, 3, 4), np.float32), np.zeros(0, np.uint32))
    p, i = H.grid(2)
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        w = product_words(layout, [S.Mesh(p, i)], inst)
        scene = engine.upload(layout, w)
        rays = H.random_rays(64, -1, 1)
        got = gpu_trace(engine, scene, rays, A.CLOSEST, "plain")
        if layout == A.LAYOUT_GI:
            assert (got[:, 1] == A.MISS).all()
        else:
            assert (got[:, 1] == 0).all()
        scene.release()
    w = product_words(A.LAYOUT_GI, [S.Mesh(p, i)], S.identity_instances(1))
    bad = w.copy()
    bad[16 + 22] = 0x7FFFFFF0  # root node index far outside the buffer
    with pytest.raises(A.RtError, match="LAYOUT"):
        engine.upload(A.LAYOUT_GI, bad)
    bad = w.copy()
    bad[0] = 1 << 20  # more instance records than words
    with pytest.raises(A.RtError, match="LAYOUT"):
        engine.upload(A.LAYOUT_GI, bad)


def test_host_buffers_match_device(engine):
    """rt_trace_host (pinned chunked copies over two streams) returns the device results."""
    torch = _torch()
    mesh, rays = H.small_clusters(30_000, 320, 320)
    w = product_words(A.LAYOUT_REFLECTION, [mesh], S.identity_instances(1))
    scene = engine.upload(A.LAYOUT_REFLECTION, w)
    try:
        dev = gpu_trace(engine, scene, rays, A.CLOSEST, "plain")
        pinned = torch.from_numpy(rays).pin_memory()
        out = torch.empty((len(rays), 5), dtype=torch.int32).pin_memory()
        engine.trace_host(scene, pinned, A.CLOSEST, "plain", out=out)
        assert np.array_equal(out.numpy().view(np.uint32), dev)
        host = engine.trace_host(scene, rays, A.ANY_CASTERS, "plain")
        assert np.array_equal(host, gpu_trace(engine, scene, rays, A.ANY_CASTERS, "plain"))
        # several batches, kernels and modes in one pipeline, twice in a row, into the same buffers
        half = rays[: len(rays) // 2]
        want = [dev, gpu_trace(engine, scene, half, A.ANY_CASTERS, "fast"), gpu_trace(engine, scene, rays, A.CLOSEST, "fast")]
        outs = [torch.empty((len(rays), 5), dtype=torch.int32).pin_memory(), None, None]
        for _ in range(2):
            got = engine.trace_host_batches(scene, [(pinned, A.CLOSEST, "plain", outs[0]), (half, A.ANY_CASTERS, "fast"),
                                                    (rays, A.CLOSEST, "fast"), (rays[:0], A.CLOSEST, "plain")])
            assert np.array_equal(got[0].numpy().view(np.uint32), want[0])
            assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2]) and len(got[3]) == 0
    finally:
        scene.release()


def test_stack_overflow_is_counted_not_silent(engine):
    """A hand-built BLAS deeper than the 48-entry stack allows: pushes past the stack are
    dropped (as the WGSL does) and counted, identically to the oracle's count."""
    words = deep_chain_scene(depth=24)
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    try:
        rays = np.array([[0.5, 0.5, -5.0, 0.0, 0.0, 0.0, 1.0, 1e30]] * 32, np.float32)
        before = engine.stats()["stack_overflows"]
        got = gpu_trace(engine, scene, rays, A.CLOSEST, "plain")
        after = engine.stats()["stack_overflows"]
        want, cnt = O.rs_trace(words, rays, False, counters=True)
        check_same(got, want, "deep chain")
        assert cnt["stack_drops"] > 0
        assert after - before == cnt["stack_drops"]
    finally:
        scene.release()


def deep_chain_scene(depth: int) -> np.ndarray:
    """A reflection-layout scene whose BLAS is a chain: every node has one deeper node then three
    one-triangle leaves, all over one unit square. Equal entry distances keep slot order, so a ray
    descends first and leaves three entries a level on the stack: 16 levels fill 48 entries."""
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    n_leaves = 3 * depth + 1
    nodes = []
    box = np.array([0, 0, 0, 1, 1, 0], np.float32)
    child = 0x80000000 | ((3 * depth) << 4) | 1  # the last leaf
    for level in range(depth):
        leaves = [0x80000000 | ((3 * level + k) << 4) | 1 for k in range(3)]
        kids = np.array([child] + leaves, np.uint32)  # the deeper node first: leaves wait on the stack
        nodes.append(O.quantized_node(kids, np.tile(box, (4, 1))))
        child = level
    # nodes must be in postorder: node `level` holds node `level - 1`; the root is the last.
    node_words = np.concatenate(nodes)
    tris = np.zeros((n_leaves, 12), np.uint32)
    for k in range(n_leaves):
        t = tris[k]
        t[0:3] = tri[0].view(np.uint32)
        t[3:6] = (tri[1] - tri[0]).view(np.uint32)
        t[6:9] = (tri[2] - tri[0]).view(np.uint32)
        t[9] = k
    head = np.zeros(8, np.uint32)
    rec = np.zeros(24, np.uint32)
    rows = np.zeros((3, 4), np.float32)
    rows[0, 0] = rows[1, 1] = rows[2, 2] = 1.0
    rec[0:12] = rows.reshape(-1).view(np.uint32)
    rec[12:18] = np.array([-1, -1, -1, 2, 2, 1], np.float32).view(np.uint32)
    base = 8 + 24 + 32 + 8
    rec[18] = base
    rec[19] = base + len(node_words)
    rec[20] = depth - 1
    rec[21] = 0
    head[0] = 1
    head[4] = 8 + 24 + 32
    bounds = np.array([-1, -1, -1, 0, 2, 2, 1, 0], np.float32).view(np.uint32)
    return np.concatenate([head, rec, np.zeros(32, np.uint32), bounds, node_words, tris.reshape(-1)]).astype(np.uint32)


@pytest.mark.parametrize("key", ["origin", "octant", "direction"])
def test_ray_order_is_a_permutation_and_changes_no_result(engine, key):
    """rt_order_rays returns a permutation of the batch; tracing through it (FAST and WIDE8) gives
    every ray the same result as tracing in the given order."""
    torch = _torch()
    mesh, rays = H.small_clusters()
    w = product_words(A.LAYOUT_REFLECTION, [mesh], S.identity_instances(1))
    scene = engine.upload(A.LAYOUT_REFLECTION, w)
    try:
        want, _ = O.rs_trace(w, rays, False)
        hit = want[:, 1] != 0
        pts = S.hit_points(rays[hit], want[hit, 0].view(np.float32))
        gi = S.hemisphere_rays(pts, S.triangle_normals(mesh, want[hit, 2]), rays[hit, 4:7], 30_000, S.Stream(7))
        batch = np.concatenate([rays, gi])
        d = torch.from_numpy(batch).cuda()
        order = engine.order(scene, d, key)
        torch.cuda.synchronize()
        perm = order.cpu().numpy()
        assert np.array_equal(np.sort(perm), np.arange(len(batch)))
        assert not np.array_equal(perm, np.arange(len(batch)))
        scene.prepare("wide8")
        for kernel in ("fast", "wide8"):
            plain = engine.trace(scene, d, A.CLOSEST, kernel)
            sorted_ = engine.trace(scene, d, A.CLOSEST, kernel, order=order)
            torch.cuda.synchronize()
            assert torch.equal(plain, sorted_), kernel
        got = engine.trace(scene, d, A.CLOSEST, "fast", order=order).cpu().numpy().view(np.uint32)
        want_all, _ = O.rs_trace(w, batch, False)
        check_same(got, want_all, "ordered fast")
    finally:
        scene.release()


@pytest.mark.parametrize("case", ["flat", "tlas"])
def test_legacy_bvh2_kernel_matches_the_reference_replay(engine, case):
    """The PLAIN kernel over the legacy BVH2 layout against the golden vectors the reference's
    own replay (tools/sunrt/replay_geometry.py) produced: t bits and hit records (barycentric
    bits included) for closest hits; blocked flags for any hits."""
    g = np.load(Path(__file__).resolve().parent / "golden" / "replay_bvh2.npz")
    words, rays = g[case + "_words"], g[case + "_rays"]
    scene = engine.upload(A.LAYOUT_REFLECTION_BVH2, words)
    try:
        got = gpu_trace(engine, scene, rays, A.CLOSEST, "plain").reshape(-1, 5)
        assert np.array_equal(got[:, 0], g[case + "_closest_t"])
        assert np.array_equal(got[:, 1:], g[case + "_closest_record"])
        flags = gpu_trace(engine, scene, rays, A.ANY_CASTERS, "plain")
        assert np.array_equal(flags, (g[case + "_any_record"][:, 0] != 0).astype(np.uint32))
        with pytest.raises(A.RtError, match="UNSUPPORTED"):
            gpu_trace(engine, scene, rays, A.CLOSEST, "fast")
    finally:
        scene.release()
