"""Replay of renderlab's reflection geometry dumps through the engine.

A dump is what the renderer writes when RENDERLAB_REFLECTION_GEOMETRY_DUMP is set
(src/reflection_geometry_dump.rs): ``<name>.json`` metadata beside ``<name>.words.bin``, the
packed little-endian u32 words of the legacy median-BVH2 reflection layout
(format "reflection-bvh2-u32-le"). Rays come as JSON lines of exact shader rays: frame, view,
origin, direction, tmin, tmax, and optionally id, slot, any_hit and the GPU's own hit record
(gpu_record).

``Dump`` loads and checks a dump the way tools/sunrt/replay_geometry.py:31-53 does, and its
``inventory`` walks every mesh and the top level as that tool's ``inventory`` (:55-100) does.
``replay`` traces the rays on the GPU with the PLAIN kernel over the BVH2 layout (the WGSL of
shaders/reflections_software.wgsl restated) and writes ``rays.csv`` and ``replay-summary.json``:
hit records, t, and the identity check against gpu_record (primitive identity first, as the
reference tool compares). ``write_dump`` writes a dump in the same format (for tests and for
replaying scenes packed here).

    python -m renderlab_b200.replay dump.json --rays rays.jsonl --out outdir
"""
from __future__ import annotations

import argparse
import csv
import hashlib
import json
from pathlib import Path

import numpy as np

LEAF = 0x80000000
FORMAT = "reflection-bvh2-u32-le"
PATH = "nonrt-software-reflections"
STACK = 32  # the shader's pending-stack bound (reflections_software.wgsl)


def _walk(w: np.ndarray, root: int, base: int, top: bool) -> dict:
    """Nodes, leaves, primitives, depth and the largest pending stack of one BVH2 tree."""
    pending = [(int(root), 0)]
    seen = set()
    depth = nodes = leaves = primitives = max_pending = 0
    while pending:
        max_pending = max(max_pending, len(pending))
        item, d = pending.pop()
        depth = max(depth, d + 1)
        if item & LEAF:
            leaves += 1
            primitives += 1 if top else item & 7
            continue
        if item in seen:
            raise ValueError("tree node reached twice")
        seen.add(item)
        nodes += 1
        at = base + 16 * item
        pending.append((int(w[at + 13]), d + 1))
        pending.append((int(w[at + 12]), d + 1))
    return dict(nodes=nodes, leaves=leaves, primitives=primitives, depth=depth, max_pending=max_pending)


class Dump:
    """A reflection geometry dump: metadata and words, checked as the reference's replay checks."""

    def __init__(self, metadata):
        self.path = Path(metadata)
        self.meta = json.loads(self.path.read_text())
        m = self.meta
        if m["version"] != 1 or m["format"] != FORMAT:
            raise ValueError("unsupported geometry format")
        if m["path"] != PATH or m["hardware_acceleration_structures"]:
            raise ValueError("software geometry required")
        if (m["header_words"], m["instance_words"]) != (8, 24):
            raise ValueError("unexpected record layout")
        binary = self.path.with_suffix(".words.bin")
        if binary.stat().st_size != m["payload_words"] * 4:
            raise ValueError("incomplete payload")
        self.words = np.fromfile(binary, dtype="<u4").astype(np.uint32)
        w = self.words
        if int(w[0]) != m["written_instances"]:
            raise ValueError("instance count differs from header")
        if list(map(int, w[1:4])) != [m["tlas"][k] for k in ("base_word", "root", "refits")]:
            raise ValueError("TLAS metadata differs from payload")
        included = sum(p["included"] for d in m["source_draws"] for p in d["placements"])
        if included != m["written_instances"]:
            raise ValueError("included provenance differs from packing")

    def inventory(self) -> dict:
        w, m = self.words, self.meta
        meshes, by_base = [], {}
        for mesh in m["meshes"]:
            r = _walk(w, mesh["root"], mesh["node_base_word"], False)
            if (r["nodes"], r["primitives"], r["depth"]) != (mesh["nodes"], mesh["triangles"], mesh["depth"]):
                raise ValueError(f"mesh {mesh['mesh']}: tree differs from its metadata")
            meshes.append(dict(mesh=mesh["mesh"], **r))
            by_base[(mesh["node_base_word"], mesh["triangle_base_word"])] = mesh["mesh"]
        instances = {}
        for i in range(int(w[0])):
            at = 8 + 24 * i
            key = by_base[(int(w[at + 18]), int(w[at + 19]))]
            instances[key] = instances.get(key, 0) + 1
        top = _walk(w, int(w[2]), int(w[1]), True) if w[1] else None
        return dict(frame=m["frame"], view=m["view"], generation=m["generation"], written_instances=int(w[0]),
                    reserved_instances=m["reserved_instances"], mesh_instances=instances, meshes=meshes, tlas=top)


def write_dump(path, words, frame: int = 0, view: int = 0, generation: int = 0) -> Path:
    """Writes ``path`` (.json) and its .words.bin for BVH2 reflection-layout words, with the
    metadata the reader checks (meshes found from the instance records)."""
    path = Path(path)
    w = np.ascontiguousarray(words, np.uint32)
    n = int(w[0])
    meshes, seen = [], {}
    for i in range(n):
        at = 8 + 24 * i
        key = (int(w[at + 18]), int(w[at + 19]))
        if key in seen:
            continue
        seen[key] = len(meshes)
        r = _walk(w, int(w[at + 20]), key[0], False)
        meshes.append(dict(mesh=len(meshes), root=int(w[at + 20]), node_base_word=key[0], triangle_base_word=key[1],
                           nodes=r["nodes"], triangles=r["primitives"], depth=r["depth"]))
    meta = dict(version=1, format=FORMAT, path=PATH, hardware_acceleration_structures=False, header_words=8,
                instance_words=24, payload_words=int(w.size), written_instances=n, reserved_instances=n,
                tlas=dict(base_word=int(w[1]), root=int(w[2]), refits=int(w[3])), frame=frame, view=view,
                generation=generation, meshes=meshes,
                source_draws=[dict(placements=[dict(included=1) for _ in range(n)])])
    w.astype("<u4").tofile(path.with_suffix(".words.bin"))
    path.write_text(json.dumps(meta, indent=2) + "\n")
    return path


def read_rays(path, frame: int, view: int):
    """JSONL shader rays -> (rays (n, 8) float32, any_hit (n,) bool, ids, slots, gpu records or None)."""
    rays, anys, ids, slots, recs = [], [], [], [], []
    with Path(path).open() as source:
        for n, line in enumerate(source):
            ray = json.loads(line)
            if (ray["frame"], ray["view"]) != (frame, view):
                raise ValueError("geometry and ray frame/view mismatch")
            rays.append([*ray["origin"], ray["tmin"], *ray["direction"], ray["tmax"]])
            anys.append(bool(ray.get("any_hit", False)))
            ids.append(ray.get("id", n))
            slots.append(ray.get("slot"))
            recs.append(ray.get("gpu_record"))
    return np.array(rays, np.float32).reshape(-1, 8), np.array(anys, bool), ids, slots, recs


def replay(dump: Dump, rays_path, out, engine=None) -> dict:
    """Traces the JSONL rays through the engine over the dump's words; writes rays.csv and
    replay-summary.json in ``out``; returns the summary with the per-ray t and records."""
    import torch
    from . import api as A
    out = Path(out)
    out.mkdir(parents=True, exist_ok=True)
    own = engine is None
    engine = engine or A.Engine(0)
    scene = engine.upload(A.LAYOUT_REFLECTION_BVH2, dump.words)
    try:
        rays, anys, ids, slots, recs = read_rays(rays_path, dump.meta["frame"], dump.meta["view"])
        t = np.zeros(len(rays), np.float32)
        record = np.zeros((len(rays), 4), np.uint32)
        drops = engine.stats()["stack_overflows"]
        for flag in (False, True):
            sel = np.nonzero(anys == flag)[0]
            if len(sel) == 0:
                continue
            d = torch.from_numpy(np.ascontiguousarray(rays[sel])).cuda()
            h = engine.trace(scene, d, A.ANY_CASTERS if flag else A.CLOSEST, "plain")
            torch.cuda.synchronize()
            h = h.cpu().numpy().view(np.uint32)
            if flag:  # an any-hit query reports blocked or not; its record is the flag
                record[sel, 0] = h
                t[sel] = rays[sel, 7]
            else:
                t[sel] = h[:, 0].view(np.float32)
                record[sel] = h[:, 1:5]
        if engine.stats()["stack_overflows"] != drops:
            raise ValueError("pending stack exceeds shader bound; never silently drop")
        checked = matches = 0
        with (out / "rays.csv").open("w", newline="") as dest:
            writer = csv.DictWriter(dest, fieldnames=["id", "slot", "any_hit", "t", "record"])
            writer.writeheader()
            for k in range(len(rays)):
                writer.writerow(dict(id=ids[k], slot=slots[k], any_hit=bool(anys[k]), t=float(t[k]),
                                     record=[int(x) for x in record[k]]))
                if recs[k] is not None:  # primitive identity (any hit: blocked or not)
                    checked += 1
                    if anys[k]:
                        matches += int((record[k][0] != 0) == (recs[k][0] != 0))
                    else:
                        matches += int(list(map(int, record[k][:2])) == list(recs[k][:2]))
        summary = dict(rays=len(rays), gpu_identity_checked=checked, gpu_identity_matches=matches,
                       gpu_identity_mismatches=checked - matches,
                       traversal="PLAIN kernel over the legacy BVH2 layout (reflections_software.wgsl restated)")
        (out / "replay-summary.json").write_text(json.dumps(summary, indent=2) + "\n")
        return dict(summary, t=t, record=record)
    finally:
        scene.release()
        if own:
            engine.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("geometry", type=Path)
    ap.add_argument("--rays", type=Path)
    ap.add_argument("--out", type=Path, required=True)
    args = ap.parse_args(argv)
    dump = Dump(args.geometry)
    args.out.mkdir(parents=True, exist_ok=True)
    inventory = dump.inventory()
    inventory["metadata_sha256"] = hashlib.sha256(args.geometry.read_bytes()).hexdigest()
    (args.out / "inventory.json").write_text(json.dumps(inventory, indent=2) + "\n")
    if args.rays:
        s = replay(dump, args.rays, args.out)
        print(json.dumps({k: v for k, v in s.items() if k not in ("t", "record")}))
    else:
        print(json.dumps(dict(frame=inventory["frame"], instances=inventory["written_instances"],
                              meshes=len(inventory["meshes"]))))


if __name__ == "__main__":
    main()
