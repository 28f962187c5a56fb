"""GPU parity of the WIDE8 kernel (compressed 8-wide BVH, watertight f32 tests, f64 re-test of
uncertain candidates) against the FP64 oracle (crates/asset/src/cluster_bvh/reference.rs
restated over the packed buffers).

Tolerances: hit identity must equal the FP64 oracle's except on near ties, defined as both
hitting with |t - t64| <= 1e-6 * t64; t within 1e-5 relative of t64 on every hit; barycentrics
u, v within 1e-5 of the oracle's on every hit with the oracle's identity (they range over [0, 1],
so the bound is relative to that range); any-hit flags equal except where the FP64 hit lies
within 1e-5 relative of tmin or tmax."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H
from .test_gpu_parity import gpu_trace, product_words

pytestmark = pytest.mark.gpu

T_REL = 1e-5
TIE_REL = 1e-6
BARY_ABS = 1e-5


def check_closest(layout, got, ref64, ident64, what):
    """Returns (max rel t error, mean rel t error, near ties, max barycentric error) and asserts
    the bar."""
    if layout == A.LAYOUT_GI:
        ghit = got[:, 1] != A.MISS
        gid = got[:, 1:5]
        oid = ident64[:, 2:6]
        guv = got[:, 5:7]
    else:
        ghit = got[:, 1] != 0
        gid = got[:, 1:3]
        oid = ident64[:, 2:4]
        guv = got[:, 3:5]
    ohit = ref64[:, 0] > 0
    t = got[:, 0].view(np.float32).astype(np.float64)
    t64 = ref64[:, 1]
    both = ghit & ohit
    rel = np.abs(t[both] - t64[both]) / np.maximum(np.abs(t64[both]), 1e-30)
    same_id = (gid == oid).all(axis=1)
    mism = (ghit != ohit) | (both & ~same_id)
    tie = mism & both & (np.abs(t - t64) <= TIE_REL * np.abs(t64))
    bad = np.nonzero(mism & ~tie)[0]
    assert len(bad) == 0, (f"{what}: {len(bad)} unexplained mismatches of {len(got)}; first {bad[:4]}: "
                           f"got {got[bad[:2]]} oracle hit {ohit[bad[:2]]} t64 {t64[bad[:2]]} ident {oid[bad[:2]]}")
    if both.any():
        assert rel.max() <= T_REL, f"{what}: max rel t error {rel.max():.3g}"
    same = both & same_id
    bary = np.abs(guv[same].view(np.float32).astype(np.float64) - ref64[same, 2:4]).max(axis=1) if same.any() else np.zeros(0)
    if len(bary):
        worst = np.nonzero(same)[0][np.argmax(bary)]
        assert bary.max() <= BARY_ABS, (f"{what}: max barycentric error {bary.max():.3g} at ray {worst}: "
                                        f"got {guv[worst].view(np.float32)} oracle {ref64[worst, 2:4]}")
    return (float(rel.max()) if both.any() else 0.0, float(rel.mean()) if both.any() else 0.0, int(tie.sum()),
            float(bary.max()) if len(bary) else 0.0)


def check_any(got, rays, ref64, what):
    ohit = ref64[:, 0] > 0
    ghit = got != 0
    mism = ghit != ohit
    t64 = ref64[:, 1]
    near = ohit & ((np.abs(t64 - rays[:, 7]) <= T_REL * np.abs(rays[:, 7])) | (np.abs(t64 - rays[:, 3]) <= T_REL * np.maximum(np.abs(rays[:, 3]), 1e-30)))
    bad = np.nonzero(mism & ~near)[0]
    assert len(bad) == 0, f"{what}: {len(bad)} any-hit mismatches; first {bad[:4]}"


@pytest.fixture(params=["wide8", "wide8p"])
def w8kernel(request):
    """Both WIDE8 walks: one ray per lane, and warp-wide packets of 32 rays (flat scenes)."""
    return request.param


def traced(engine, layout, words, rays, mode, kernel="wide8"):
    scene = engine.upload(layout, words)
    try:
        scene.prepare("wide8")
        return gpu_trace(engine, scene, rays, mode, kernel)
    finally:
        scene.release()


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_wide8_clusters_primary_and_gi(engine, w8kernel, layout):
    mesh, rays = H.small_clusters(60_000, 256, 256)
    prims = [True] if layout == A.LAYOUT_GI else None
    w = product_words(layout, [mesh], S.identity_instances(1), primitives=prims)
    got = traced(engine, layout, w, rays, A.CLOSEST, w8kernel)
    ref, ident = O.fp64_trace(w, rays, layout)
    stats = check_closest(layout, got, ref, ident, "primary")
    hit = ref[:, 0] > 0
    pts = S.hit_points(rays[hit], ref[hit, 1].astype(np.float32))
    prim = ident[hit, 1]
    gi = S.hemisphere_rays(pts, S.triangle_normals(mesh, prim if layout == A.LAYOUT_REFLECTION else ident[hit, 1]),
                           rays[hit, 4:7], 40_000, S.Stream(77))
    got = traced(engine, layout, w, gi, A.CLOSEST, w8kernel)
    ref, ident = O.fp64_trace(w, gi, layout)
    stats_gi = check_closest(layout, got, ref, ident, "gi")
    print("wide8 t error (max, mean, ties)", stats, stats_gi)


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_wide8_instanced_cubes(engine, layout):
    mesh, inst = S.cubes_instanced(30)
    inst.casts = (np.arange(len(inst)) % 5) != 2
    w = product_words(layout, [mesh], inst)
    rays = H.small_cubes(30, 160, 160)[1]
    got = traced(engine, layout, w, rays, A.CLOSEST)
    ref, ident = O.fp64_trace(w, rays, layout)
    check_closest(layout, got, ref, ident, "closest")
    hit = ref[:, 0] > 0
    sun = S.sun_rays(S.hit_points(rays[hit], ref[hit, 1].astype(np.float32)))
    got = traced(engine, layout, w, sun, A.ANY_CASTERS)
    ref_any, _ = O.fp64_trace(w, sun, layout, any_hit=True)
    check_any(got, sun, ref_any, "sun")


def test_wide8_edge_rays(engine, w8kernel):
    p, i = H.grid(12)
    mesh = S.Mesh(p, i)
    rays = []
    for d in ([0, -1, 0], [0, 1, 0], [1, 0, 0], [0.3, -1, 0], [0, -1, 1e-31], [1e-35, -1, 0]):
        for o in ([0.5, 1, 0.5], [0.0, 0.5, 0.0], [0.25, 0.0, 0.25], [1.0, 2.0, 1.0], [1 / 3, 1, 0.5]):
            for tmin, tmax in ((0.0, 1e30), (0.0, np.inf), (0.0, 3.4028235e38), (0.5, 0.25), (1e-4, 10.0)):
                rays.append([*o, tmin, *d, tmax])
    rays = np.array(rays, np.float32)
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        w = product_words(layout, [mesh], S.identity_instances(1))
        got = traced(engine, layout, w, rays, A.CLOSEST, w8kernel)
        ref, ident = O.fp64_trace(w, rays, layout)
        check_closest(layout, got, ref, ident, f"edge rays layout {layout}")


def test_wide8_grid_edges_are_watertight(engine, w8kernel):
    """Rays aimed exactly at shared edges and vertices of a grid: none slips through."""
    p, i = H.grid(16)
    mesh = S.Mesh(p * np.float32(4.0), i)
    xs = np.arange(17, dtype=np.float32) / 16 * 4
    o = np.array([[x, 1.0, z] for x in xs[1:-1] for z in np.concatenate([xs[1:-1], xs[1:-1] + 0.125])], np.float32)
    rays = S.pack_rays(o, np.tile([0.0, -1.0, 0.0], (len(o), 1)), 0.0, 10.0)
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        w = product_words(layout, [mesh], S.identity_instances(1))
        got = traced(engine, layout, w, rays, A.CLOSEST, w8kernel)
        hit = got[:, 1] != (A.MISS if layout == A.LAYOUT_GI else 0)
        assert hit.all(), f"{(~hit).sum()} rays slipped through the grid"


def test_wide8_refuses_blas_beyond_its_decode_range(engine):
    """An 8-wide node decodes its planes as 2^(e+15) / d; exponents above 13 (a BLAS wider than
    255 * 2^13 units) could overflow, so preparing such a scene is refused, and FAST still runs."""
    p = np.array([[0, 0, 0], [3.0e6, 0, 0], [0, 1, 0]], np.float32)
    i = np.array([0, 1, 2], np.uint32)
    w = product_words(A.LAYOUT_REFLECTION, [S.Mesh(p, i)], S.identity_instances(1))
    scene = engine.upload(A.LAYOUT_REFLECTION, w)
    try:
        with pytest.raises(A.RtError, match="LAYOUT"):
            scene.prepare("wide8")
        rays = np.array([[1.0, 0.25, -1.0, 0.0, 0.0, 0.0, 1.0, 10.0]], np.float32)
        got = gpu_trace(engine, scene, rays, A.CLOSEST, "fast")
        assert got[0, 1] != 0
    finally:
        scene.release()


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_packet_walk_over_a_top_level(engine, layout):
    """The packet walk also walks a scene's top level (900 cube instances, some casting no
    shadow): per ray it returns the per-ray walk's records exactly -- closest hits, and both
    any-hit modes -- and the FP64 oracle's hit ids, for coherent camera rays and random rays."""
    import torch
    mesh, inst = S.cubes_instanced(30)
    inst.casts = (np.arange(len(inst)) % 5) != 2
    w = product_words(layout, [mesh], inst)
    assert w[1] != 0
    scene = engine.upload(layout, w)
    try:
        scene.prepare("wide8")
        cam = H.small_cubes(30, 128, 96)[1]
        rnd = H.random_rays(8_000, -30.0, 30.0, seed=8, tmax=200.0)
        for rays in (cam, rnd):
            d = torch.from_numpy(rays).cuda()
            for mode in (A.CLOSEST, A.ANY_SKY, A.ANY_CASTERS):
                a = engine.trace(scene, d, mode, "wide8")
                b = engine.trace(scene, d, mode, "wide8p")
                torch.cuda.synchronize()
                assert torch.equal(a, b), f"mode {mode}: {(a != b).sum().item()} words differ"
            got = engine.trace(scene, d, A.CLOSEST, "wide8p").cpu().numpy().view(np.uint32)
            ref, ident = O.fp64_trace(w, rays, layout)
            check_closest(layout, got, ref, ident, "packet walk over a top level")
        assert (got[:, 1] != (A.MISS if layout == A.LAYOUT_GI else 0)).mean() > 0.05
    finally:
        scene.release()


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_wide8_rebraided_top_level(engine, layout):
    """The 8-wide top level splits each instance's BLAS into world-space entries (up to 256 an
    instance): over 400 rotated, scaled instances of four cluster meshes, some casting no shadow,
    and random rays through their overlap, the per-ray walk finds the FP64 oracle's closest hits
    and caster flags, and in every mode the same hits as over a top level of one entry per
    instance (ids equal, t within the f64 band; flags equal) while entering far fewer."""
    import torch
    ms = S.multi_blas(n_blas=4, n_instances=400, tri_lo=2e3, tri_hi=2e4, half=300.0, config=11)
    inst = ms.instances
    inst.casts = (np.arange(len(inst)) % 5) != 2
    w = product_words(layout, ms.meshes, inst)
    assert w[1] != 0
    rng = np.random.default_rng(21)
    o = rng.uniform(-300.0, 300.0, (20_000, 3))
    d = rng.normal(size=(20_000, 3))
    rays = S.pack_rays(o, d / np.linalg.norm(d, axis=1, keepdims=True), 0.0, 1e30)
    dev = torch.from_numpy(rays).cuda()
    got, entered = {}, {}
    try:
        for entries in (1, 256):
            engine.set_tuning(wide8_entries=entries)
            scene = engine.upload(layout, w)
            try:
                scene.prepare("wide8")
                for mode in (A.CLOSEST, A.ANY_SKY, A.ANY_CASTERS):
                    got[entries, mode] = engine.trace(scene, dev, mode, "wide8").cpu().numpy().view(np.uint32)
                c = engine.trace_counted(scene, dev[::8].contiguous(), A.CLOSEST, "wide8")
                entered[entries] = c["instance_tests"] / c["rays"]
            finally:
                scene.release()
    finally:
        engine.set_tuning(wide8_entries=256)
    ids = slice(1, 3) if layout == A.LAYOUT_REFLECTION else slice(1, 5)
    a, b = got[1, A.CLOSEST], got[256, A.CLOSEST]
    assert np.array_equal(a[:, ids], b[:, ids])
    ta, tb = a[:, 0].view(np.float32), b[:, 0].view(np.float32)
    assert np.all(np.abs(ta - tb) <= 2e-5 * np.abs(ta))
    for mode in (A.ANY_SKY, A.ANY_CASTERS):
        assert np.array_equal(got[1, mode], got[256, mode]), f"mode {mode}"
    ref, ident = O.fp64_trace(w, rays, layout)
    check_closest(layout, b, ref, ident, "re-braided top level")
    ref_any, _ = O.fp64_trace(w, rays, layout, any_hit=True)
    check_any(got[256, A.ANY_CASTERS].reshape(-1), rays, ref_any, "casters over the re-braided top level")
    assert 0.2 < (ref[:, 0] > 0).mean() < 0.98
    assert entered[256] < 0.7 * entered[1], entered


def test_tune_top_keeps_a_measured_budget_and_every_result(engine):
    """rt_scene_tune_top rebuilds only the 8-wide top level per candidate budget, keeps the fastest
    on its probe (one of the candidates, kept by a later prepare after records change), and the
    walk over the chosen top level finds the FP64 oracle's hits and caster flags. A flat scene has
    nothing to tune (0); an unprepared scene and out-of-range budgets are refused."""
    import torch
    layout = A.LAYOUT_REFLECTION
    ms = S.multi_blas(n_blas=4, n_instances=300, tri_lo=2e3, tri_hi=2e4, half=300.0, config=12)
    inst = ms.instances
    inst.casts = (np.arange(len(inst)) % 4) != 1
    w = product_words(layout, ms.meshes, inst)
    rng = np.random.default_rng(31)
    o = rng.uniform(-300.0, 300.0, (12_000, 3))
    d = rng.normal(size=(12_000, 3))
    rays = S.pack_rays(o, d / np.linalg.norm(d, axis=1, keepdims=True), 0.0, 1e30)
    dev = torch.from_numpy(rays).cuda()
    scene = engine.upload(layout, w)
    try:
        with pytest.raises(A.RtError):
            scene.tune_top()  # not prepared
        scene.prepare("wide8")
        for bad in ([0], [2000]):
            with pytest.raises(A.RtError):
                scene.tune_top(bad)
        chosen = scene.tune_top([1, 16, 256], probe=8192)
        assert chosen in (1, 16, 256)
        got = engine.trace(scene, dev, A.CLOSEST, "wide8").cpu().numpy().view(np.uint32)
        flags = engine.trace(scene, dev, A.ANY_CASTERS, "wide8").cpu().numpy()
        ref, ident = O.fp64_trace(w, rays, layout)
        check_closest(layout, got, ref, ident, f"top level tuned to {chosen} entries an instance")
        ref_any, _ = O.fp64_trace(w, rays, layout, any_hit=True)
        check_any(flags.reshape(-1), rays, ref_any, "casters over the tuned top level")
        # default candidates; the choice survives a records rewrite and re-prepare
        chosen = scene.tune_top()
        assert chosen in (1, 4, 16, 64, 256)
        before = engine.trace_counted(scene, dev[::4].contiguous(), A.CLOSEST, "wide8")
        scene.update_records(w)
        scene.prepare("wide8")
        after = engine.trace_counted(scene, dev[::4].contiguous(), A.CLOSEST, "wide8")
        assert (before["top_nodes"], before["instance_tests"]) == (after["top_nodes"], after["instance_tests"])
        again = engine.trace(scene, dev, A.CLOSEST, "wide8").cpu().numpy().view(np.uint32)
        ids = slice(1, 3)
        assert np.array_equal(again[:, ids], got[:, ids])
    finally:
        scene.release()
    mesh, _ = H.small_clusters(20_000, 16, 16)
    flat = engine.upload(layout, product_words(layout, [mesh], S.identity_instances(1)))
    try:
        flat.prepare("wide8")
        assert flat.tune_top() == 0
    finally:
        flat.release()


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_packet_walk_matches_the_per_ray_walk(engine, layout):
    """Per ray, the packet walk finds the per-ray walk's hit: ids equal, t within the f64
    band (the t of a winner the per-ray walk accepted in f32 may come back refined in f64), for
    coherent primaries, incoherent GI rays, a permutation and batches with mixed modes."""
    import torch
    mesh, rays = H.small_clusters(60_000, 256, 256)
    prims = [True] if layout == A.LAYOUT_GI else None
    w = product_words(layout, [mesh], S.identity_instances(1), primitives=prims)
    scene = engine.upload(layout, w)
    try:
        scene.prepare("wide8")
        rnd = H.random_rays(30_000, -120.0, 120.0, seed=4, tmax=400.0)
        for batch in (rays, rnd):
            d = torch.from_numpy(batch).cuda()
            order = engine.order(scene, d, "origin")
            a = engine.trace(scene, d, A.CLOSEST, "wide8").cpu().numpy().view(np.uint32)
            for kw in ({}, {"order": order}):
                b = engine.trace(scene, d, A.CLOSEST, "wide8p", **kw).cpu().numpy().view(np.uint32)
                ids = slice(1, 3) if layout == A.LAYOUT_REFLECTION else slice(1, 5)
                assert np.array_equal(a[:, ids], b[:, ids])
                ta, tb = a[:, 0].view(np.float32), b[:, 0].view(np.float32)
                assert np.all(np.abs(ta - tb) <= 2e-5 * np.abs(ta))
            flags_a = engine.trace(scene, d, A.ANY_CASTERS, "wide8").cpu().numpy()
            got = engine.trace_batches(scene, [(d[:1000], A.ANY_CASTERS), (d[1000:], A.CLOSEST)], "wide8p")
            assert np.array_equal(got[0].cpu().numpy(), flags_a[:1000])
            assert np.array_equal(got[1].cpu().numpy().view(np.uint32)[:, ids], a[1000:, ids])
    finally:
        scene.release()


def _narrow_batches(mesh, n_packets=600, seed=5):
    """Packets of 32 consecutive rays that share a direction octant within a narrow cone, with
    origins and directions spread in the ways that stress the packet walk's shared traversal:
    scattered origins, rays that graze edges and vertices, zero and sub-clamp components."""
    rng = np.random.default_rng(seed)
    p = mesh.positions.astype(np.float64)
    tri = mesh.indices.reshape(-1, 3)
    out = []
    # (1) parallel rays, as toward a directional light, from points on random triangles (origins
    # spread over the scene, or within one cluster's neighbourhood after a sort by origin)
    k = rng.integers(0, len(tri), 32 * n_packets)
    b = rng.dirichlet((1.0, 1.0, 1.0), 32 * n_packets)
    on = (p[tri[k, 0]] * b[:, :1] + p[tri[k, 1]] * b[:, 1:2] + p[tri[k, 2]] * b[:, 2:3])
    sun = np.array([0.3, 0.8, 0.2]) / np.linalg.norm([0.3, 0.8, 0.2])
    o = on + 1e-3 * sun
    out.append(S.pack_rays(o, np.tile(sun, (len(o), 1)), 0.0, 1e30))
    order = np.lexsort((o[:, 2], np.floor(o[:, 1] / 8.0), np.floor(o[:, 0] / 8.0)))
    out.append(S.pack_rays(o[order], np.tile(-sun, (len(o), 1)), 0.0, 1e30))
    # (2) one origin, each packet aimed at one triangle: rays through its vertices and through
    # points 1e-7 .. 1e-3 (relative) off its edges, inside and outside
    eye = np.array([0.0, 0.0, -250.0])
    k = np.repeat(rng.integers(0, len(tri), n_packets), 32)
    e = rng.integers(0, 3, len(k))
    t = rng.uniform(0.0, 1.0, len(k))
    t[::8] = 0.0  # a vertex
    v0, v1, v2 = p[tri[k, e]], p[tri[k, (e + 1) % 3]], p[tri[k, (e + 2) % 3]]
    on_edge = v0 * (1 - t)[:, None] + v1 * t[:, None]
    inward = v2 - on_edge
    off = rng.choice([-1.0, 1.0], len(k)) * 10.0 ** rng.uniform(-7, -3, len(k))
    target = on_edge + inward * off[:, None]
    d = target - eye
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out.append(S.pack_rays(np.tile(eye, (len(d), 1)), d, 0.0, 1e30))
    # (3) directions with a zero (+0 or -0) or tiny (below the 1e-30 clamp) component, mixed in a
    # packet, from a scattered line of origins across the scene
    n = 32 * n_packets
    o = np.stack([rng.uniform(-150, 150, n), rng.uniform(-120, 120, n), np.full(n, -260.0)], axis=1)
    d = np.tile(np.array([0.05, 0.0, 1.0]), (n, 1))
    d[:, 1] = rng.choice([0.0, -0.0, 1e-35, -1e-35, 1e-20], n)
    d[:, 0] = rng.choice([0.05, 0.0, -0.0], n) * (np.arange(n) // 32 % 2)
    out.append(S.pack_rays(o, d / np.linalg.norm(d, axis=1, keepdims=True), 0.0, 1e30))
    return out


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_packet_walk_on_narrow_packets_matches_the_per_ray_walk(engine, layout):
    """On parallel rays from scattered origins, narrow cones aimed at vertices and within 1e-7 of
    edges, and directions with zero or sub-clamp components, the packet walk returns the per-ray
    walk's hits (ids equal, t within the f64 band; any-hit flags equal) and the FP64 oracle's hit
    ids."""
    import torch
    mesh, _ = H.small_clusters(60_000, 64, 64)
    w = product_words(layout, [mesh], S.identity_instances(1))
    scene = engine.upload(layout, w)
    ids = slice(1, 3) if layout == A.LAYOUT_REFLECTION else slice(1, 5)
    try:
        scene.prepare("wide8")
        for j, batch in enumerate(_narrow_batches(mesh)):
            d = torch.from_numpy(batch).cuda()
            a = engine.trace(scene, d, A.CLOSEST, "wide8").cpu().numpy().view(np.uint32)
            b = engine.trace(scene, d, A.CLOSEST, "wide8p").cpu().numpy().view(np.uint32)
            assert np.array_equal(a[:, ids], b[:, ids]), f"batch {j}: {(a[:, ids] != b[:, ids]).any(1).sum()} rays differ"
            ta, tb = a[:, 0].view(np.float32), b[:, 0].view(np.float32)
            assert np.all(np.abs(ta - tb) <= 2e-5 * np.abs(ta)), f"batch {j}"
            for mode in (A.ANY_SKY, A.ANY_CASTERS):
                fa = engine.trace(scene, d, mode, "wide8").cpu().numpy()
                fb = engine.trace(scene, d, mode, "wide8p").cpu().numpy()
                assert np.array_equal(fa, fb), f"batch {j} mode {mode}: {(fa != fb).sum()} flags differ"
            sub = slice(0, 32 * 96)
            ref, ident = O.fp64_trace(w, batch[sub], layout)
            check_closest(layout, b[sub], ref, ident, f"packet walk, narrow batch {j}")
            assert (b[:, 1] != (A.MISS if layout == A.LAYOUT_GI else 0)).any()
    finally:
        scene.release()


def test_wide8_far_small_triangles_near_edges(engine, w8kernel):
    """Isolated small triangles (0.05 units) 200 units down the view axis and 50 units to its
    side, rays aimed within 1e-6 to 1e-3 of an edge, inside and outside. The shear's rounding grows
    with the lateral offset: here an f32 edge function can be off by ~1e-4 of the edge functions'
    sum, more than a margin relative to that sum allows, so these rays must be re-tested in f64
    and agree with the FP64 oracle (a hit its oracle triangle, a miss a miss) on every ray."""
    rng = np.random.default_rng(3)
    size, tris = 0.05, []
    for k in range(64):
        x0, y0 = 40.0 + (k % 8) * 2 * size, -30.0 + (k // 8) * 2 * size
        z = rng.uniform(-0.01, 0.01)
        tris.append([[x0, y0, z], [x0 + size, y0 + 0.2 * size, z + 0.003], [x0 + 0.1 * size, y0 + size, z - 0.003]])
    p = np.array(tris, np.float32).reshape(-1, 3)
    mesh = S.Mesh(p, np.arange(len(p), dtype=np.uint32))
    n = 8192
    t = rng.uniform(0.05, 0.95, n)
    q = rng.integers(0, 64, n)
    e = rng.integers(0, 3, n)  # which edge
    v0, v1 = p[3 * q + e].astype(np.float64), p[3 * q + (e + 1) % 3].astype(np.float64)
    other = p[3 * q + (e + 2) % 3].astype(np.float64)
    on_edge = v0 * (1 - t)[:, None] + v1 * t[:, None]
    inward = other - on_edge
    inward /= np.linalg.norm(inward, axis=1, keepdims=True)
    off = rng.choice([-1.0, 1.0], n) * size * 10.0 ** rng.uniform(-6, -3, n)
    b = on_edge + inward * off[:, None]
    o = np.array([0.0, 0.0, -200.0])
    d = b - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = S.pack_rays(np.tile(o, (n, 1)), d, 0.0, 1e30)
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        w = product_words(layout, [mesh], S.identity_instances(1))
        got = traced(engine, layout, w, rays, A.CLOSEST, w8kernel)
        ref, ident = O.fp64_trace(w, rays, layout)
        check_closest(layout, got, ref, ident, f"near edges, layout {layout}")
        assert 0.3 < (ref[:, 0] > 0).mean() < 0.7


@pytest.mark.parametrize("layout", [A.LAYOUT_GI, A.LAYOUT_REFLECTION])
def test_shared_group_stack_gives_the_local_stack_results(engine, layout):
    """WIDE8's per-ray walk with each lane's node-group stack in shared memory (16 entries)
    writes word for word what the local-memory stack writes -- through plans and through the
    context's tuning, closest and any hit, primaries and incoherent rays -- and drops no push."""
    import torch
    mesh, rays = H.small_clusters(60_000, 256, 256)
    prims = [True] if layout == A.LAYOUT_GI else None
    w = product_words(layout, [mesh], S.identity_instances(1), primitives=prims)
    scene = engine.upload(layout, w)
    drops = engine.stats()["stack_overflows"]
    try:
        scene.prepare("wide8")
        assert 1 <= scene.wide8_depth() <= 16
        rnd = H.random_rays(30_000, -120.0, 120.0, seed=6, tmax=400.0)
        d, e = torch.from_numpy(rays).cuda(), torch.from_numpy(rnd).cuda()
        batches = [(d, A.CLOSEST), (e, A.CLOSEST), (e[:7000], A.ANY_CASTERS)]
        plans = {s: engine.plan(scene, batches, "wide8", refill=8, stack=s) for s in ("local", "shared")}
        for p in plans.values():
            p.launch()
        torch.cuda.synchronize()
        for a, b in zip(plans["local"].hits, plans["shared"].hits):
            assert torch.equal(a, b)
        want = [engine.trace(scene, r, m, "wide8") for r, m in batches]
        engine.set_tuning(wide8_stack=A.STACKS["shared"])
        got = [engine.trace(scene, r, m, "wide8") for r, m in batches]
        engine.set_tuning(wide8_stack=A.STACKS["local"])
        torch.cuda.synchronize()
        for a, b, p in zip(want, got, plans["local"].hits):
            assert torch.equal(a, b) and torch.equal(a, p)
        for p in plans.values():
            p.close()
        assert engine.stats()["stack_overflows"] == drops
    finally:
        engine.set_tuning(wide8_stack=A.STACKS["local"])
        scene.release()
