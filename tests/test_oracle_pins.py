"""Pins the oracle (and the product's host builders, which must match it word for word) to the
reference: golden vectors from the reference's own Python replay, and the known-answer and
property tests of the reference's Rust suite, restated."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

from . import helpers as H

GOLDEN = H.__file__.replace("helpers.py", "golden/replay_bvh2.npz")
LEAF = 0x80000000
EMPTY = 0xFFFFFFFF


# ---------------------------------------------------------------- replay_geometry.py golden vectors

@pytest.mark.parametrize("case", ["flat", "tlas"])
@pytest.mark.parametrize("any_hit", [False, True])
def test_replay_golden_vectors(case, any_hit):
    """tools/sunrt/replay_geometry.py (the reference's f32 replay) over dyadic BVH2 scenes:
    t bits, hit records (with barycentric bits) and all nine traversal counters agree."""
    g = np.load(GOLDEN)
    names = list(g["counters"])
    idx = [O.COUNTERS.index(n) for n in names]
    key = f"{case}_{'any' if any_hit else 'closest'}"
    hits, cnt = O.rs_trace_counts(g[case + "_words"], g[case + "_rays"], any_hit=any_hit, bvh2=True)
    assert np.array_equal(hits[:, 0], g[key + "_t"])
    assert np.array_equal(hits[:, 1:], g[key + "_record"])
    assert np.array_equal(cnt[:, idx], g[key + "_counters"])
    assert (hits[:, 1] != 0).sum() > 30


GENERAL = H.__file__.replace("helpers.py", "golden/replay_bvh2_general.npz")


@pytest.mark.parametrize("case", ["flat", "tlas"])
@pytest.mark.parametrize("any_hit", [False, True])
def test_replay_general_inputs(case, any_hit):
    """tools/sunrt/replay_geometry.py over general f32 scenes (jittered height fields and
    triangle soups, instances under arbitrary rotations and scales, 600 rays aimed at triangle
    interiors, edges and vertices; tests/golden/make_replay_golden.py --general).

    - "sequential": the replay with its np.dot summed left to right in f32 (the order the WGSL
      writes and the oracle evaluates). The oracle must equal it bit for bit: t, hit records
      with barycentric bits, and all nine traversal counters, on every ray.
    - "numpy": the replay as it ships, np.dot from the host's BLAS (another summation order).
      Rays aimed at triangle interiors or past them must give the same hit identity, with t
      within 2e-5 relative; only rays aimed exactly at an edge or a vertex, where two triangles
      are both hit within the reference's RS_EDGE slack, may resolve to the other one."""
    g = np.load(GENERAL)
    names = list(g["counters"])
    idx = [O.COUNTERS.index(n) for n in names]
    hits, cnt = O.rs_trace_counts(g[case + "_words"], g[case + "_rays"], any_hit=any_hit, bvh2=True)
    key = f"{case}_{'any' if any_hit else 'closest'}"
    seq = key + "_sequential"
    assert np.array_equal(hits[:, 0], g[seq + "_t"])
    assert np.array_equal(hits[:, 1:], g[seq + "_record"])
    assert np.array_equal(cnt[:, idx], g[seq + "_counters"])
    num = key + "_numpy"
    rec, t = g[num + "_record"], g[num + "_t"].view(np.float32).astype(np.float64)
    same = (hits[:, 1:3] == rec[:, 0:2]).all(1)
    aim = np.arange(len(hits)) % 6  # 0, 1 interior; 2, 3 an edge; 4 a vertex; 5 past the triangle
    assert same[(aim < 2) | (aim == 5)].all()
    both = same & (rec[:, 0] != 0)
    tt = hits[both, 0].view(np.float32).astype(np.float64)
    assert np.all(np.abs(tt - t[both]) <= 2e-5 * np.abs(t[both]))
    assert (rec[:, 0] != 0).sum() > 300 and same.mean() > 0.9


def test_replay_known_answer_lower_instance_wins():
    """test_replay_geometry.py:43-85: two identity instances of one triangle; the equal-t hit
    resolves to the lower instance (slot 7 + 1) even when the top level visits instance 1 first."""
    for top in (False, True):
        w = np.zeros(84, np.uint32)
        f = w.view(np.float32)
        w[0] = 2
        if top:
            w[1:3] = [56, 0]
            f[56:68] = [0, 0, 0, 1, 1, 0] * 2
            w[68:70] = [LEAF | 1, LEAF]
        for i in range(2):
            at = 8 + i * 24
            f[at:at + 12] = np.eye(4, dtype=np.float32)[:3].reshape(-1)
            f[at + 12:at + 18] = [0, 0, 0, 1, 1, 0]
            w[at + 18:at + 22] = [72, 72, LEAF | 1, 7 + i]
        f[72:81] = [0, 0, 0, 1, 0, 0, 0, 1, 0]
        w[81] = 42
        rays = np.array([[.25, .25, 1, .001, 0, 0, -1, 1e6], [2, 2, 1, .001, 0, 0, -1, 1e6]], np.float32)
        hits, cnt = O.rs_trace_counts(w, rays, bvh2=True)
        assert list(hits[0, 1:3]) == [8, 42]
        assert hits[0, 0].view(np.float32) == 1.0
        assert cnt[0, O.COUNTERS.index("triangle_tests")] == 2
        assert cnt[0, O.COUNTERS.index("blas_visits")] == 2
        assert hits[1, 1] == 0 and cnt[1, O.COUNTERS.index("triangle_tests")] == 0


# ---------------------------------------------------------------- builder (near_field.rs tests)

def uneven_scene():
    """gi_bvh.rs:302-314: a dense 40 x 40 patch beside a sparse 4 x 4 plane."""
    p, i = H.grid(40)
    q, j = H.grid(4)
    base = len(p)
    p = np.concatenate([p, np.stack([q[:, 0] * 30 + 2, q[:, 1] + 0.5, q[:, 2] * 30], 1).astype(np.float32)])
    return p, np.concatenate([i, j + base]).astype(np.uint32)


def walk_leaves(nodes16, root):
    """(leaf ids reached, deepest node level) of a BVH4 in runtime words."""
    out, deepest, stack = [], 0, [(root, 0)]
    while stack:
        c, d = stack.pop()
        if c & LEAF:
            out.append(c & ~LEAF)
            continue
        deepest = max(deepest, d + 1)
        for k in nodes16[c][6:10]:
            if k != EMPTY:
                stack.append((int(k), d + 1))
    return out, deepest


def test_sah_build_partitions_every_triangle():
    """gi_bvh.rs:302-341: every triangle in exactly one leaf of <= 8, depth <= MAX_SAH_DEPTH;
    the product builder's records equal the oracle's."""
    p, i = uneven_scene()
    b = O.Bvh(p, i, 1)
    info = b.info()
    leaves, deepest = walk_leaves(b.nodes(), info["root"])
    assert sorted(leaves) == list(range(info["leaves"]))
    lv = b.leaves()
    assert (lv[:, 1] <= 24).all()
    tris = [tuple(t) for t in b.indices().reshape(-1, 3)]
    src = [tuple(t) for t in i.reshape(-1, 3)]
    assert sorted(tris) == sorted(src)
    assert deepest <= 15
    prod = A.Blas(p, i)
    assert np.array_equal(prod.nodes(), b.nodes()) and np.array_equal(prod.bvh_indices(), b.indices())


def test_builds_valid_deterministic_bvh4():
    """near_field.rs:653-672: deterministic, >= 2 children a node, one-leaf root for a small
    mesh, invalid input rejected."""
    p, i = H.grid(24)
    a, b = O.Bvh(p, i, 0), O.Bvh(p, i, 0)
    assert np.array_equal(a.nodes(), b.nodes())
    assert all(((n[6:10] != EMPTY).sum() >= 2) for n in a.nodes())
    small = O.Bvh(p, i[:6], 0)
    assert small.info()["nodes"] == 0 and small.info()["root"] & LEAF
    with pytest.raises(ValueError):
        O.Bvh(np.zeros((1, 3), np.float32), np.array([0, 0], np.uint32), 0)
    with pytest.raises(ValueError):
        O.Bvh(np.full((3, 3), np.nan, np.float32), np.array([0, 1, 2], np.uint32), 0)
    with pytest.raises(A.RtError):
        A.Blas(np.full((3, 3), np.nan, np.float32), np.array([0, 1, 2], np.uint32))
    for median in (False, True):
        prod = A.Blas(p, i, median)
        ref = O.Bvh(p, i, 0 if median else 1)
        assert np.array_equal(prod.nodes(), ref.nodes())


def decode(nodes16, fused):
    """Child boxes of every node under one decode: (n, 4, 2, 3) float32. The fused decode
    fma(step, q, origin) is formed in float64 (step * q is exact there) and rounded once."""
    n = nodes16.view(np.float32)
    o, s = n[:, 0:3], n[:, 3:6]
    out = np.zeros((len(nodes16), 4, 2, 3), np.float32)
    for slot in range(4):
        for k, base in enumerate((10, 13)):
            q = ((nodes16[:, base:base + 3] >> np.uint32(8 * slot)) & 255).astype(np.float32)
            if fused:
                out[:, slot, k] = (s.astype(np.float64) * q + o).astype(np.float32)
            else:
                out[:, slot, k] = o + s * q
    return out


def test_refit_keeps_the_tree_and_encloses_moved_triangles():
    """near_field.rs:683-713: refit to the same positions is the identity; to moved positions
    it keeps topology and every leaf vertex inside its box under both decodes."""
    p, i = H.grid(24)
    built = O.Bvh(p, i, 1)
    same = O.Bvh(p, i, 1)
    same.refit(p)
    assert np.array_equal(same.nodes(), built.nodes())
    k = np.arange(len(p), dtype=np.float32)
    moved = np.stack([p[:, 0] * 1.7 + np.sin(k * 0.37) * 0.2, np.cos(k * 0.11), p[:, 2] - 3.0], 1).astype(np.float32)
    refit = O.Bvh(p, i, 1)
    refit.refit(moved)
    refit.validate()
    assert np.array_equal(refit.indices(), built.indices())
    prod = A.Blas(p, i)
    prod.refit(moved)
    assert np.array_equal(prod.nodes(), refit.nodes())
    nodes = refit.nodes()
    lv = refit.leaves()
    idx = refit.indices()
    seen = 0
    for fused in (False, True):
        boxes = decode(nodes, fused)
        for n, node in enumerate(nodes):
            for slot in range(4):
                c = int(node[6 + slot])
                if c == EMPTY or not c & LEAF:
                    continue
                off, cnt = lv[c & ~LEAF][:2]
                v = moved[idx[off:off + cnt]].astype(np.float64)
                lo, hi = boxes[n, slot, 0].astype(np.float64), boxes[n, slot, 1].astype(np.float64)
                assert (lo <= v).all() and (v <= hi).all()
                seen += 1
    assert seen == 2 * len(lv)
    with pytest.raises(ValueError):
        refit.refit(moved[1:])


def test_quantized_node_matches_product():
    """Conservative outward codes (near_field.rs:481-525) on random boxes: oracle == product,
    and both decodes enclose every child."""
    s = S.Stream(11)
    for _ in range(50):
        n = int(s.uniform() * 3) + 2
        lo = s.range(-1e3, 1e3, n, 3)
        hi = lo + s.uniform(n, 3) * np.array([1e-3, 10, 1e3])
        boxes = np.concatenate([lo, hi], 1).astype(np.float32)
        kids = np.arange(n, dtype=np.uint32)
        w = O.quantized_node(kids, boxes)
        dec_u = decode(w[None], False)[0]
        for k in range(n):
            assert (dec_u[k, 0] <= boxes[k, :3]).all() and (dec_u[k, 1] >= boxes[k, 3:]).all()


def fib_rays():
    th = np.arange(300) * 2.399963229728653
    y = (np.arange(300) + 0.5) / 150.0 - 1.0
    r = np.sqrt(1 - y * y)
    d = np.stack([r * np.cos(th), y, r * np.sin(th)], 1)
    rays = np.zeros((300 + 6, 8))
    rays[:300, 0:3] = d * 4
    rays[:300, 4:7] = -d
    rays[:300, 7] = 10.0
    k = 300
    for ax in range(3):
        for o in (0.0, 20.0):
            rays[k, 0:3] = o
            rays[k, 4 + ax] = 1.0
            rays[k, 7] = np.inf
            k += 1
    return rays


def closed_sphere(n):
    """crates/cook/src/virtual_fixtures.rs:28-80 geometry: six subdivided faces normalised."""
    pos, idx = [], []
    for axis in range(3):
        for sign in (-1, 1):
            base = len(pos)
            for y in range(n + 1):
                for x in range(n + 1):
                    q = [0, 0, 0]
                    q[axis] = sign * n
                    q[(axis + 1) % 3] = 2 * x - n
                    q[(axis + 2) % 3] = 2 * y - n
                    ln = np.sqrt(sum(float(v) ** 2 for v in q))
                    pos.append([0.0 if v == 0 else np.float32(v / ln) for v in q])
            for y in range(n):
                for x in range(n):
                    a = base + y * (n + 1) + x
                    b, c = a + 1, a + n + 1
                    d = c + 1
                    idx += [a, b, d, a, d, c] if sign > 0 else [a, d, b, a, c, d]
    return np.array(pos, np.float32), np.array(idx, np.uint32)


def thin_sheet(n):
    """crates/cook/src/virtual_fixtures.rs:82-140 geometry: a curved two-part sheet + 48 fins."""
    pos, idx = [], []
    for side in range(2):
        base = len(pos)
        for y in range(n + 1):
            for x in range(side * n // 2, (side + 1) * n // 2 + 1):
                u, v = x / n, y / n
                pos.append([u * 4 - 2, 0.2 * np.sin(u * 6) * np.cos(v * 5), v * 4 - 2])
        row = n // 2 + 1
        for y in range(n):
            for x in range(n // 2):
                a = base + y * row + x
                b, c = a + 1, a + row
                d = c + 1
                idx += [a, d, b, a, c, d]
    for i in range(48):
        z = np.float32(i) / np.float32(47.0) * np.float32(3.8) - np.float32(1.9)
        a = len(pos)
        pos += [[-1.95, 0.25, z], [-1.945, 0.25, z + 0.025], [-1.94, 0.9, z + 0.0125]]
        idx += [a, a + 1, a + 2]
    return np.array(pos, np.float32), np.array(idx, np.uint32)


@pytest.mark.parametrize("fixture", [closed_sphere(24), thin_sheet(12)], ids=["closed_sphere", "thin_sheet"])
def test_trace_equals_trace_brute(fixture):
    """crates/cook/tests/cluster_bvh.rs:37-100: the f64 tree walk equals the brute force over
    every leaf on 300 Fibonacci-sphere rays and the axis rays."""
    p, i = fixture
    for mode in (0, 1):
        b = O.Bvh(p, i, mode)
        rays = fib_rays()
        tree, brute = b.trace64(rays), b.trace64(rays, brute=True)
        assert np.array_equal(tree, brute)
        assert tree[:300, 0].sum() == 300  # every inward Fibonacci ray meets the closed shape


# ---------------------------------------------------------------- packers (gi_bvh.rs tests)

def translate(x, y, z):
    m = np.zeros((1, 3, 4), np.float32)
    m[0, 0, 0] = m[0, 1, 1] = m[0, 2, 2] = 1.0
    m[0, :, 3] = (x, y, z)
    return m


def test_packs_instances_and_meshes():
    """gi_bvh.rs:343-419: the runtime layout bit for bit, world-to-object rows, the padded world
    box, and a singular transform rejected."""
    p, i = H.grid(6)
    model = np.concatenate([translate(5, 0, 0), translate(0, 0, 0)])
    inst = S.Instances(model, S.affine_inverse_rows(model.astype(np.float64)), np.zeros(2, np.uint32))
    w = A.pack_scene(A.LAYOUT_GI, [A.Blas(p, i)], inst)
    assert np.array_equal(w, O.scene_words(0, [(p, i)], H.oracle_instances(inst, 0)))
    b = O.Bvh(p, i, 1)
    info = b.info()
    nodes = 16 + 2 * 32 + O.tlas_reserve(2)
    r = 16
    assert list(w[r + 18:r + 22]) == [nodes, nodes + 16 * info["nodes"], nodes + 16 * info["nodes"] + 2 * info["leaves"],
                                      nodes + 16 * info["nodes"] + 2 * info["leaves"] + 3 * info["positions"]]
    assert np.array_equal(w[nodes:nodes + 16 * info["nodes"]], b.nodes().reshape(-1))
    lo = w[r + 12:r + 15].view(np.float32)
    assert abs(lo[0] - 5.0) < 1e-3
    row0 = w[r:r + 4].view(np.float32)
    assert abs(row0[0] * 5.0 + row0[3]) < 1e-6
    assert w[0] == 2 and w[1] == 0  # two instances: the flat list
    sing = S.Instances(np.zeros((1, 3, 4), np.float32), np.zeros((1, 3, 4), np.float32), np.zeros(1, np.uint32))
    with pytest.raises(A.RtError):
        A.pack_scene(A.LAYOUT_GI, [A.Blas(p, i)], sing)
    # The reflection writer skips a singular placement instead (reflection_software.rs:353-356).
    mixed = S.Instances(np.concatenate([translate(1, 2, 3), sing.model]), np.concatenate([translate(-1, -2, -3), sing.rows]),
                        np.zeros(2, np.uint32))
    wr = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(p, i)], mixed)
    assert wr[0] == 1
    assert np.array_equal(wr, O.scene_words(1, [(p, i)], H.oracle_instances(mixed, 1)))


def test_with_primitives_maps_reordered_triangles_including_duplicates():
    """gi_bvh.rs:421-443: a duplicated triangle gets a distinct source id; the table sits after
    the mesh's indices and instance word 28 points at it."""
    p, i = H.grid(6)
    i = np.concatenate([i, i[:3]]).astype(np.uint32)
    inst = S.identity_instances(1)
    w = A.pack_scene(A.LAYOUT_GI, [A.Blas(p, i)], inst, primitives=[True])
    assert np.array_equal(w, O.scene_words(0, [(p, i, 1)], H.oracle_instances(inst, 0)))
    b = O.Bvh(p, i, 1)
    prim_base = w[16 + 28]
    n = len(i) // 3
    prims = w[prim_base:prim_base + n]
    assert sorted(prims) == list(range(n))
    for tri, src in zip(b.indices().reshape(-1, 3), prims):
        assert list(tri) == list(i[3 * src:3 * src + 3])


def test_reflection_bvh_keeps_primitive_identity():
    """reflection_software.rs:475-510: on a 23 x 23 quad grid every triangle is found by a ray
    through 0.5a + 0.3b + 0.2c with its own primitive, u = 0.3, v = 0.2, t = 1 (within 1e-4);
    a rebuild is word-identical."""
    n = 23
    pos = np.array([[x, y, ((x * 7 + y * 3) % 5) * 0.01] for y in range(n + 1) for x in range(n + 1)], np.float32)
    idx = []
    for y in range(n):
        for x in range(n):
            a, wd = y * (n + 1) + x, n + 1
            idx += [a, a + 1, a + wd + 1, a, a + wd + 1, a + wd]
    idx = np.array(idx, np.uint32)
    inst = S.identity_instances(1)
    w = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(pos, idx)], inst)
    assert np.array_equal(w, A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(pos, idx)], inst))
    tri = idx.reshape(-1, 3)
    P = pos.astype(np.float32)
    target = P[tri[:, 0]] * np.float32(0.5) + P[tri[:, 1]] * np.float32(0.3) + P[tri[:, 2]] * np.float32(0.2)
    o = target + np.array([0.01, -0.02, 3.0], np.float32)
    d = target - o
    rays = S.pack_rays(o, d, 0.0, 1e30)
    hits, _ = O.rs_trace(w, rays)
    assert np.array_equal(hits[:, 2], np.arange(len(tri)))
    u, v, t = hits[:, 3].view(np.float32), hits[:, 4].view(np.float32), hits[:, 0].view(np.float32)
    assert np.abs(u - 0.3).max() < 1e-4 and np.abs(v - 0.2).max() < 1e-4 and np.abs(t - 1).max() < 1e-4
    f64, ident = O.fp64_trace(w, rays, 1)
    assert np.array_equal(ident[:, 3], np.arange(len(tri)))


def test_gi_hit_normal_follows_instance_transform():
    """gi_cache_tests.rs:3286-3408 on the oracle: one triangle under a scaled, rotated,
    translated instance; t within 1e-4 of the distance, normal . expected > 0.9999."""
    a, b, c = np.array([0, 0, 0.0]), np.array([1, 0, 0.0]), np.array([0, 0, 1.0])
    p = np.array([a, b, c], np.float32)
    i = np.array([0, 1, 2], np.uint32)
    ax, ay, az = 0.7, 0.3, -0.4
    Rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
    Ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
    Rz = np.array([[np.cos(az), -np.sin(az), 0], [np.sin(az), np.cos(az), 0], [0, 0, 1]])
    M = Rx @ Ry @ Rz @ np.diag([2.0, 0.5, 3.0])
    model = np.zeros((1, 3, 4))
    model[0, :, :3] = M
    model[0, :, 3] = [1, 2, -1]
    inst = S.Instances(model.astype(np.float32), S.affine_inverse_rows(model), np.zeros(1, np.uint32))
    w = A.pack_scene(A.LAYOUT_GI, [A.Blas(p, i)], inst)
    normal = np.linalg.inv(M).T @ np.cross(b - a, c - a)
    normal /= np.linalg.norm(normal)
    target = M @ ((a + b + c) / 3) + model[0, :, 3]
    ortho = np.cross(normal, [1, 0, 0] if abs(normal[0]) < 0.9 else [0, 1, 0])
    ortho /= np.linalg.norm(ortho)
    origin = target + 2 * normal + 0.3 * ortho
    d = (target - origin) / np.linalg.norm(target - origin)
    rays = S.pack_rays(origin[None], d[None], 0.0, 1e30)
    hits, _ = O.gi_trace(w, rays, 0)
    assert hits[0, 1] == 0
    assert abs(hits[0, 0].view(np.float32) - np.linalg.norm(target - origin)) < 1e-4
    assert hits[0, 7:10].view(np.float32) @ normal > 0.9999


# ---------------------------------------------------------------- top level (instance_bvh.rs tests)

def xorshift(seed, div, scale):
    s = np.uint32(seed)

    def nxt():
        nonlocal s
        s ^= np.uint32((int(s) << 13) & 0xFFFFFFFF)
        s ^= np.uint32(int(s) >> 17)
        s ^= np.uint32((int(s) << 5) & 0xFFFFFFFF)
        return np.float32(int(s) % div) / np.float32(scale)
    return nxt


def children(nodes, nid):
    at = nid * 32
    f = nodes.view(np.float32)
    out = []
    for c in range(4):
        cid = int(nodes[at + 24 + c])
        if cid == EMPTY:
            continue
        lo = np.array([f[at + a * 4 + c] for a in range(3)], np.float32)
        hi = np.array([f[at + 12 + a * 4 + c] for a in range(3)], np.float32)
        out.append((cid, lo, hi))
    return out


def wide_depth(nodes, nid):
    return 1 + max([wide_depth(nodes, c) for c, _, _ in children(nodes, nid) if not c & LEAF] or [0])


def test_top_level_covers_every_instance_once():
    """instance_bvh.rs:480-518 (257 boxes, xorshift 0x12345678): each instance reached once, its
    recorded box exact, every child box inside its parent's, depth within the stack."""
    nxt = xorshift(0x12345678, 1000, 10)
    boxes = []
    for _ in range(257):
        x, y, z = nxt(), nxt(), nxt()
        boxes.append([x, y, z, x + np.float32(1), y + np.float32(2), z + np.float32(0.5)])
    boxes = np.array(boxes, np.float32)
    nodes = O.tlas_build(boxes)
    assert np.array_equal(nodes, A.tlas_build(boxes))
    assert len(nodes) <= O.tlas_reserve(len(boxes))
    seen = np.zeros(len(boxes), int)
    stack = [(0, None)]
    while stack:
        nid, parent = stack.pop()
        if nid & LEAF:
            k = nid & ~LEAF
            seen[k] += 1
            assert np.array_equal(np.concatenate(parent), boxes[k])
            continue
        for cid, lo, hi in children(nodes, nid):
            if parent is not None:
                assert (parent[0] <= lo).all() and (hi <= parent[1]).all()
            stack.append((cid, (lo, hi)))
    assert (seen == 1).all()
    assert 1 + 3 * wide_depth(nodes, 0) <= 48


def test_top_level_walk_reaches_every_crossed_instance():
    """instance_bvh.rs:541-584 (3,000 boxes, 200 rays, xorshift 0x0bad5eed): a walk entering only
    crossed boxes reaches every crossed instance."""
    nxt = xorshift(0x0BAD5EED, 10_000, 100)
    boxes = []
    for i in range(3000):
        x, y, z = nxt(), nxt() * np.float32(0.1), nxt()
        s = np.float32(30.0) if i % 50 == 0 else np.float32(0.5) + np.float32(i % 7) * np.float32(0.3)
        boxes.append([x, y, z, x + s, y + s * np.float32(0.5), z + s])
    boxes = np.array(boxes, np.float32)
    nodes = A.tlas_build(boxes)
    assert np.array_equal(nodes, O.tlas_build(boxes))

    def crosses(lo, hi, o, d):
        with np.errstate(divide="ignore", invalid="ignore"):
            p, q = (lo - o) / d, (hi - o) / d
        near = max(np.float32(0), np.minimum(p, q).max())
        far = min(np.float32(np.inf), np.maximum(p, q).min())
        return near <= far

    for r in range(200):
        o = np.array([nxt(), nxt() * np.float32(0.1) + np.float32(1), nxt()], np.float32)
        d = np.array([nxt() - np.float32(50) + np.float32(0.01), np.float32(r % 5) * np.float32(0.1) - np.float32(0.2) + np.float32(0.003),
                      nxt() - np.float32(50) + np.float32(0.02)], np.float32)
        want = sorted(k for k in range(len(boxes)) if crosses(boxes[k, :3], boxes[k, 3:], o, d))
        got, stack = [], [0]
        while stack:
            nid = stack.pop()
            for cid, lo, hi in children(nodes, nid):
                if crosses(lo, hi, o, d):
                    (got.append(cid & ~LEAF) if cid & LEAF else stack.append(cid))
        assert sorted(got) == want, r


def test_refit_follows_moved_boxes():
    """instance_bvh.rs:687-703: refitting to boxes moved along y equals a fresh build."""
    boxes = np.array([[(i * 7) % 50, 0, 0, (i * 7) % 50 + 1, 1, 1] for i in range(50)], np.float32)
    nodes = O.tlas_build(boxes)
    moved = boxes.copy()
    moved[:, [1, 4]] += 3
    assert np.array_equal(O.tlas_refit(nodes, moved), O.tlas_build(moved))
    assert np.array_equal(A.tlas_refit(nodes, moved), O.tlas_build(moved))


def test_place_sets_the_header_and_reuses_unchanged_records():
    """instance_bvh.rs:706-722: header words, reserve, and reuse of unchanged records."""
    header, stride = 8, 24
    words = np.zeros(header + 3 * stride, np.uint32)
    words[0] = 3
    f = words.view(np.float32)
    for i in range(3):
        r = header + i * stride
        f[r + 12:r + 15] = i * 4.0
        f[r + 15:r + 18] = i * 4.0 + 1.0
    placed = O.tlas_place(words, header, stride, 3)
    assert len(placed) == len(words) + O.tlas_reserve(3)
    assert placed[1] == 0  # three instances: below MIN_INSTANCES, no top level
    forced = O.tlas_place(words, header, stride, 3, mode=1)
    assert (forced[1], forced[2]) == (len(words), 0)
    assert np.array_equal(O.tlas_place(words, header, stride, 3, previous=placed), placed)
    again = O.tlas_place(words, header, stride, 3, previous=forced, mode=1)
    assert np.array_equal(again, forced)


def test_gi_cell_rays_are_the_fixed_hemisphere_directions():
    """gi_direction (gi_cache.wgsl:1046-1054): 64 equal-solid-angle directions about the cell
    normal -- direction k at cos theta = 1 - (k + 0.5) / 64, golden-angle azimuths -- from the
    query point offset along the normal by gi_origin_offset (gi_cache.wgsl:1064-1068)."""
    from renderlab_b200 import scenes as S
    rng = np.random.default_rng(5)
    n = rng.normal(size=(40, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    q = rng.uniform(-50, 50, (40, 3)).astype(np.float32)
    cells = S.gi_cells(q, n, 0.25, S.Stream(3))
    rays = O.gi_cell_rays(cells).reshape(40, 64, 8)
    # the normal the producer decoded: close to the packed one (16-bit octahedral encoding)
    d = rays[:, :, 4:7].astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=2), 1.0, atol=2e-6)
    z = 1.0 - (np.arange(64) + 0.5) / 64.0
    cos = np.einsum("ckj,cj->ck", d, n)
    assert np.abs(cos - z[None, :]).max() < 2e-4
    # azimuths advance by the golden angle about the normal
    off = np.linalg.norm(rays[:, 0, 0:3].astype(np.float64) - q, axis=1)
    m = np.abs(q).max(axis=1)
    ulp = np.spacing(m.astype(np.float32)).astype(np.float64)
    want = np.maximum(np.maximum(1e-5, 32.0 * ulp) + 1e-4 * 0.25, 1e-4 + 4e-7 * m)
    assert np.abs(off - want).max() < 4 * ulp.max()  # q + n * off rounds at |q|'s ulp
    assert (rays[:, :, 7] == np.float32(1e20)).all() and (rays[:, :, 3] == 0).all()
    # turned by the key: the same cosines, other azimuths
    turned = O.gi_cell_rays(cells, rotate=True).reshape(40, 64, 8)
    assert np.abs(np.einsum("ckj,cj->ck", turned[:, :, 4:7].astype(np.float64), n) - z).max() < 2e-4
    assert not np.allclose(turned[:, :, 4:7], rays[:, :, 4:7])
