"""Cooked files: the RLB cluster-BVH codec and the RNF near-field codec (native, through the C
ABI), pinned by an independent struct-level reader of the formats written here, and the
reference's own codec tests restated (crates/asset/src/near_field.rs:783-827 and
crates/cook/tests/cluster_bvh.rs:179-212)."""
import struct

import numpy as np
import pytest

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import cooked as C
from renderlab_b200.scenes import Instances

LEAF = 0x80000000
EMPTY = 0xFFFFFFFF


def grid(n):
    """A unit grid in the xz plane, two triangles a cell (near_field.rs:723-739)."""
    p = [[x / n, 0.0, y / n] for y in range(n + 1) for x in range(n + 1)]
    i = []
    for y in range(n):
        for x in range(n):
            a = y * (n + 1) + x
            b, c = a + 1, a + n + 1
            i += [a, c, b, b, c, c + 1]
    return np.array(p, np.float32), np.array(i, np.uint32)


def blob_mesh(seed, tris=300):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-5, 5, (tris, 3)).astype(np.float32)
    pos = (centers[:, None, :] + rng.normal(0, 0.3, (tris, 3, 3))).astype(np.float32).reshape(-1, 3)
    return pos, np.arange(3 * tris, dtype=np.uint32)


def read_rlb(data: bytes) -> dict:
    """The RLB layout read field by field with struct (codec.rs:4-76), independent of the codec."""
    assert data[:4] == b"RLB\0"
    version, *counts = struct.unpack_from("<7I", data, 4)
    nn, nl, nt, nc, nv, ni = counts
    at = 32
    nodes, errors = [], []
    for _ in range(nn):
        nodes.append(struct.unpack_from("<16I", data, at))
        errors.append(struct.unpack_from("<4f", data, at + 64))
        at += 80
    leaves = [struct.unpack_from("<8I", data, at + 32 * k) for k in range(nl)]
    at += 32 * nl
    levels = [struct.unpack_from("<6I", data, at + 24 * k) for k in range(nt)]
    at += 24 * nt
    cut = struct.unpack_from(f"<{nc}I", data, at)
    at += 4 * nc
    pos = np.frombuffer(data, "<f4", 4 * nv, at).reshape(-1, 4)
    at += 16 * nv
    idx = np.frombuffer(data, "<u4", ni, at)
    assert at + 4 * ni == len(data)
    return dict(version=version, nodes=np.array(nodes, np.uint32).reshape(-1, 16), errors=errors, leaves=leaves,
                levels=levels, cut=list(cut), positions=pos, indices=idx)


def write_rlb(r: dict) -> bytes:
    out = bytearray(b"RLB\0") + struct.pack("<I", r["version"])
    out += struct.pack("<6I", len(r["nodes"]), len(r["leaves"]), len(r["levels"]), len(r["cut"]),
                       len(r["positions"]), len(r["indices"]))
    for n, e in zip(r["nodes"], r["errors"]):
        out += struct.pack("<16I", *map(int, n)) + struct.pack("<4f", *e)
    for rec in r["leaves"]:
        out += struct.pack("<8I", *rec)
    for rec in r["levels"]:
        out += struct.pack("<6I", *rec)
    out += struct.pack(f"<{len(r['cut'])}I", *r["cut"])
    out += np.ascontiguousarray(r["positions"], "<f4").tobytes() + np.ascontiguousarray(r["indices"], "<u4").tobytes()
    return bytes(out)


def rejected(data, message, **kw):
    with pytest.raises(C.CookedError) as e:
        C.decode_rlb(data, **kw)
    assert str(e.value) == message


@pytest.mark.parametrize("median", [False, True])
def test_rlb_is_the_near_field_builders_cluster_bvh(median):
    pos, idx = grid(6) if median else blob_mesh(3)
    b = A.Blas(pos, idx, median=median)
    data = C.encode_rlb(b)
    r = read_rlb(data)
    info = b.info()
    assert r["version"] == 1
    assert (r["nodes"] == b.nodes()).all()  # the 16 runtime words, then four zero errors
    assert all(e == (0.0, 0.0, 0.0, 0.0) for e in r["errors"])
    bvh = b.bvh_indices()
    assert (r["indices"] == bvh).all()
    assert (r["positions"][:, :3] == pos).all() and (r["positions"][:, 3] == 0).all()
    at = 0
    for k, (mesh, cluster, page, src, off, cnt, err, mat) in enumerate(r["leaves"]):
        assert (mesh, cluster, page, err, mat) == (0, k, 0, 0, 0)
        assert off == at and cnt % 3 == 0 and cnt > 0
        at += cnt
        # source_index_offset: 3 * the leaf's first triangle in the source list
        assert src % 3 == 0 and (idx[src:src + 3] == bvh[off:off + 3]).all()
    assert at == len(bvh)
    assert r["levels"] == [(0, info["root"], 0, 0, 0, info["leaves"])]
    assert r["cut"] == list(range(info["leaves"]))


def test_rlb_round_trip_is_exact():
    pos, idx = blob_mesh(7, 2000)
    b = A.Blas(pos, idx)
    data = C.encode_rlb(b)
    d = C.decode_rlb(data)
    assert d.info() == b.info()
    assert (d.nodes() == b.nodes()).all() and (d.bvh_indices() == b.bvh_indices()).all()
    assert (d.positions == b.positions).all()
    assert C.encode_rlb(d) == data
    # packing a decoded BLAS gives the words of packing the built one
    inst = Instances(np.eye(3, 4, dtype=np.float32)[None], np.eye(3, 4, dtype=np.float32)[None],
                     np.zeros(1, np.uint32))
    assert (A.pack_scene(A.LAYOUT_GI, [d], inst) == A.pack_scene(A.LAYOUT_GI, [b], inst)).all()
    # reflection: the same but for the primitive word of each triangle record, which a cooked
    # cut cannot carry (its source list is gone): it numbers the triangles in BVH order
    x, y = A.pack_scene(A.LAYOUT_REFLECTION, [d], inst), A.pack_scene(A.LAYOUT_REFLECTION, [b], inst)
    diff = np.nonzero(x != y)[0]
    assert len(x) == len(y) and len(diff) and len(set(diff % 12)) == 1


def test_rlb_rejections_follow_the_reference_checks():
    pos, idx = grid(6)
    data = C.encode_rlb(A.Blas(pos, idx))
    r = read_rlb(data)
    rejected(data[:-1], "BVH extent/count limit")
    rejected(data[:3], "truncated cluster BVH")
    rejected(data[:20], "truncated cluster BVH")
    rejected(data, "BVH file byte limit", max_bytes=len(data) - 1)
    rejected(b"RLX\0" + data[4:], "unknown cluster BVH schema")
    rejected(data[:4] + struct.pack("<I", 2) + data[8:], "unknown cluster BVH schema")
    rejected(data[:8] + struct.pack("<I", 0xFFFFFFFF) + data[12:], "BVH extent/count limit")
    with pytest.raises(C.CookedError, match="indirect geometry level"):
        C.decode_rlb(data, level=1)

    def bad(edit, message):
        q = {k: (v.copy() if isinstance(v, np.ndarray) else list(v)) for k, v in r.items() if k != "version"}
        q["version"] = 1
        edit(q)
        rejected(write_rlb(q), message)

    last = len(r["nodes"]) - 1

    def cyclic(q):
        q["nodes"][last, 6] = last
    bad(cyclic, "BVH unordered/cyclic node")

    def zero_step(q):
        q["nodes"][0, 3] = np.float32(0).view(np.uint32)
    bad(zero_step, "invalid cluster BVH node frame")

    def error(q):
        q["errors"][0] = (100.0, *q["errors"][0][1:])
    bad(error, "BVH child bounds/error do not enclose geometry")

    def root(q):
        q["levels"][0] = (0, LEAF | len(q["leaves"]), 0, 0, 0, len(q["leaves"]))
    bad(root, "BVH cut leaf reference")

    def duplicate(q):
        q["cut"][0] = q["cut"][1]
    bad(duplicate, "BVH duplicate/unordered cut leaf")

    def w(q):
        q["positions"][0, 3] = 1.0
    bad(w, "invalid cluster BVH position")

    def index(q):
        q["indices"][5] = len(q["positions"])
    bad(index, "cluster BVH vertex index")

    def shrink(q):  # a child's upper bound pulled below its geometry
        n = q["nodes"][last]
        slot = next(s for s in range(4) if n[6 + s] != EMPTY)
        n[13] &= ~np.uint32(0xFF << (8 * slot))
    bad(shrink, "BVH child bounds/error do not enclose geometry")

    def leaf_span(q):
        q["leaves"][0] = (*q["leaves"][0][:4], 1, *q["leaves"][0][5:])
    bad(leaf_span, "invalid cluster BVH leaf")

    def overflow(q):
        q["leaves"][0] = (*q["leaves"][0][:4], 0xFFFFFFFF, 3, *q["leaves"][0][6:])
    bad(overflow, "virtual span overflow")

    def noncanonical(q):
        for i, n in enumerate(q["nodes"]):
            for s in range(4):
                if n[6 + s] == EMPTY:
                    e = list(q["errors"][i])
                    e[s] = 1.0
                    q["errors"][i] = tuple(e)
                    return
        raise AssertionError("no empty slot in the grid BVH")
    bad(noncanonical, "noncanonical empty BVH child")

    def orphan(q):  # the only level's root moved to a subtree: the rest is unreachable
        q["levels"][0] = (0, 0, 0, 0, 0, len(q["leaves"]))
    bad(orphan, "BVH cut/root disagreement")


def test_rlb_decodes_any_level_of_a_lod_file():
    """Two levels, the second a subtree's cut at a coarser requested error: each level decodes to
    a BLAS rooted at its own root over the shared records (Blas::new, gi_bvh.rs:62-78)."""
    pos, idx = blob_mesh(11, 500)
    b = A.Blas(pos, idx)
    r = read_rlb(C.encode_rlb(b))
    nodes = r["nodes"]
    sub = 0  # node 0 is built first: a deepest subtree, its children leaves or lower nodes

    def leaves_of(c):
        if c & LEAF:
            return [c & ~LEAF]
        return sum((leaves_of(int(x)) for x in nodes[c, 6:10] if x != EMPTY), [])
    cut = sorted(leaves_of(sub))
    n_all = len(r["leaves"])
    r["levels"] = [r["levels"][0], (0, sub, np.float32(1.0).view(np.uint32).item(), 0, n_all, len(cut))]
    r["cut"] = r["cut"] + cut
    data = write_rlb(r)
    top, part = C.decode_rlb(data, level=0), C.decode_rlb(data, level=1)
    assert top.info()["root"] == b.info()["root"] and part.info()["root"] == sub
    assert (part.nodes() == b.nodes()).all()
    # requested errors must grow within a mesh
    r["levels"][1] = (0, sub, 0, 0, n_all, len(cut))
    rejected(write_rlb(r), "invalid BVH level/error order")


def field_of(bins=16, placements=1, seed=0):
    pos, idx = grid(6)
    meshes = [A.Blas(pos, idx, median=True), A.Blas(*blob_mesh(seed + 5, 120))]
    words = bins * bins // 32
    out = []
    for k in range(placements):
        m = k % 2
        t = np.eye(4, dtype=np.float32)
        t[3, :3] = [2.0 + 3 * k, 0.5 * k, -k]  # column 3 (translation), columns first
        if k % 3 == 2:
            t[0, 0] = -1.0  # a mirroring placement
        n = len(meshes[m].positions) * 2 * words
        masks = (np.arange(n, dtype=np.uint64) * 2654435761 % (1 << 32)).astype(np.uint32)
        out.append(C.Placement(m, t, masks))
    return C.NearField(1.0, 0.5, 0.01, bins, bytes([7] * 32), meshes, out)


def test_rnf_round_trip_and_reference_rejections():
    """encodes_validates_and_rejects_corruption (near_field.rs:783-827), restated."""
    f = field_of(placements=3)
    data = f.encode()
    assert data[:4] == b"RNF\0" and struct.unpack_from("<4I", data, 4) == (1, 2, 3, 16)
    assert struct.unpack_from("<3f", data, 20) == (1.0, 0.5, np.float32(0.01).item()) and data[32:64] == bytes([7] * 32)
    g = C.NearField.decode(data)
    assert (g.lod_error, g.reach, g.bins, g.source) == (f.lod_error, f.reach, f.bins, f.source)
    assert g.skip == np.float32(f.skip)
    for a, b in zip(g.meshes, f.meshes):
        assert (a.nodes() == b.nodes()).all() and (a.bvh_indices() == b.bvh_indices()).all()
    for a, b in zip(g.placements, f.placements):
        assert a.mesh == b.mesh and (a.transform == b.transform).all() and (a.masks == b.masks).all()
    assert g.encode() == data

    def refused(blob, message):
        with pytest.raises(C.CookedError) as e:
            C.NearField.decode(blob)
        assert str(e.value) == message
    refused(data[:-1], "near-field truncated")
    refused(data + b"\0", "near-field trailing bytes")
    refused(data[:4] + b"\x09" + data[5:], "unsupported near-field version")
    refused(data[:63], "near-field header or size")
    refused(b"RNX\0" + data[4:], "near-field header or size")
    refused(data[:8] + struct.pack("<I", 1 << 30) + data[12:], "near-field counts exceed the file")
    with pytest.raises(C.CookedError, match="near-field placement masks or transform"):
        short = field_of()
        short.placements[0].masks = short.placements[0].masks[:-1]
        short.encode()
    with pytest.raises(C.CookedError, match="invalid near-field settings"):
        bad = field_of()
        bad.skip = 1.0
        bad.encode()
    with pytest.raises(C.CookedError, match="near field byte limit or no meshes"):
        f.encode(max_bytes=64)
    with pytest.raises(C.CookedError, match="near-field mesh must have one level"):
        pos, idx = blob_mesh(11, 500)
        r = read_rlb(C.encode_rlb(A.Blas(pos, idx)))
        r["levels"].append((0, 0, np.float32(1.0).view(np.uint32).item(), 0, len(r["leaves"]), 0))
        cut = []

        def leaves_of(c):
            if c & LEAF:
                return [c & ~LEAF]
            return sum((leaves_of(int(x)) for x in r["nodes"][c, 6:10] if x != EMPTY), [])
        cut = sorted(leaves_of(0))
        r["levels"][1] = (*r["levels"][1][:5], len(cut))
        r["cut"] += cut
        blob = write_rlb(r)
        head = data[:64]
        head = head[:8] + struct.pack("<II", 1, 0) + head[16:]
        C.NearField.decode(head + struct.pack("<Q", len(blob)) + blob)


def test_rnf_pack_gi_appends_masks_and_finds_placements_by_transform_bits():
    f = field_of(placements=4)
    words = f.pack_gi()
    inst = f.instances()
    plain = A.pack_scene(A.LAYOUT_GI, f.meshes, inst)
    n = len(f.placements)
    assert words[0] == n and len(words) == len(plain) + sum(len(p.masks) for p in f.placements)
    rec = words[16:16 + 32 * n].reshape(n, 32)
    base = len(plain)
    # masks after every mesh's records, mesh by mesh, placements in file order
    expect = {}
    for m in range(len(f.meshes)):
        for k, p in enumerate(f.placements):
            if p.mesh == m:
                expect[k] = base
                assert (words[base:base + len(p.masks)] == p.masks).all()
                base += len(p.masks)
    for k in range(n):
        assert rec[k, 23] == expect[k]
    # everything else is the plain packing (word 23 aside)
    diff = words[:len(plain)] != plain
    diff[16 + 23:16 + 32 * n:32] = False
    assert not diff.any()
    # an instance whose model differs in one bit reads no masks
    moved = Instances(inst.model.copy(), inst.rows.copy(), inst.mesh.copy())
    moved.model[1, 0, 3] = np.nextafter(moved.model[1, 0, 3], np.float32(10))
    assert f.pack_gi(moved)[16 + 32 + 23] == 0
    assert A.validate(A.LAYOUT_GI, words)["instances"] == n


def test_rnf_world_merges_placements_in_world_space():
    f = field_of(bins=0, placements=3)
    for p in f.placements:
        p.masks = np.zeros(0, np.uint32)
    world, bases = f.world()
    at, pos, tris = 0, [], []
    for k, p in enumerate(f.placements):
        assert bases[k] == at
        m = f.meshes[p.mesh]
        t = p.transform.astype(np.float32)
        q = m.positions
        # transform_point3 rounded in turn: ((x*c0 + y*c1) + z*c2) + c3
        w = ((q[:, :1] * t[0, :3] + q[:, 1:2] * t[1, :3]) + q[:, 2:3] * t[2, :3]) + t[3, :3]
        pos.append(w.astype(np.float32))
        tri = m.bvh_indices().reshape(-1, 3).astype(np.int64) + at
        if np.linalg.det(t.astype(np.float64)) < 0:
            tri = tri[:, [0, 2, 1]]
        tris.append(tri)
        at += len(q)
    assert (world.positions == np.concatenate(pos)).all()
    built = A.Blas(np.concatenate(pos), np.concatenate(tris).astype(np.uint32).reshape(-1))
    assert (world.nodes() == built.nodes()).all() and (world.bvh_indices() == built.bvh_indices()).all()


@pytest.mark.gpu
def test_cooked_field_traces_as_the_built_meshes():
    """A decoded field's GI words trace exactly as the same meshes packed from the builder (the
    masks change word 23 and the tail, never what a ray hits), and PLAIN gives the oracle's hits."""
    import torch
    f = field_of(placements=6)
    g = C.NearField.decode(f.encode())
    inst = f.instances()
    words = g.pack_gi(inst)
    # The second mesh's node records start off a 16-byte boundary (GI meshes are not padded):
    # the FAST kernel's node loads must not assume alignment.
    assert words[16 + 32 + 18] % 4 != 0
    eng = A.Engine(0)
    try:
        a = eng.upload(A.LAYOUT_GI, words)
        b = eng.upload(A.LAYOUT_GI, A.pack_scene(A.LAYOUT_GI, f.meshes, inst))
        # rays aimed at the placements' vertices from above (about 30 % hit)
        rng = np.random.default_rng(5)
        n = 1 << 14
        pts = np.concatenate([f.meshes[p.mesh].positions @ p.transform[:3, :3] + p.transform[3, :3]
                              for p in f.placements])
        tgt = pts[rng.integers(0, len(pts), n)] + rng.normal(0, 0.05, (n, 3))
        o = tgt + np.array([0.0, 3.0, 0.0]) + rng.normal(0, 0.5, (n, 3))
        d = (tgt - o) / np.linalg.norm(tgt - o, axis=1, keepdims=True)
        rays = np.concatenate([o, np.zeros((n, 1)), d, np.full((n, 1), 1e4)], 1).astype(np.float32)
        r = torch.from_numpy(rays).cuda()
        a.prepare("wide8")
        b.prepare("wide8")
        plain = None
        for kernel in ("plain", "fast", "wide8"):
            ha = eng.trace(a, r, A.CLOSEST, kernel).cpu().numpy().view(np.uint32)
            hb = eng.trace(b, r, A.CLOSEST, kernel).cpu().numpy().view(np.uint32)
            assert (ha == hb).all(), kernel
            if kernel == "plain":
                plain = ha
                assert (plain[:, 1] != A.MISS).mean() > 0.2  # the rays do hit the field
                assert (plain == O.gi_trace(words, rays, 0)[0]).all()  # the oracle's hits, bit for bit
            elif kernel == "fast":
                assert (ha == plain).all()  # FAST is bit-identical to PLAIN
        torch.cuda.synchronize()
        a.release()
        b.release()
    finally:
        eng.close()
