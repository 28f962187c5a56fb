"""Geometry dumps (src/reflection_geometry_dump.rs's format, read as tools/sunrt/replay_geometry.py
reads it) and their replay through the engine's BVH2 kernel. The golden scenes and rays were
traced by the reference's own replay tool (tests/golden/make_replay_golden.py); a dump of them,
replayed on the GPU with those results as gpu_record, must match every ray."""
from __future__ import annotations

import json

import numpy as np
import pytest

from renderlab_b200 import replay as R

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "replay_bvh2.npz"


def _write(tmp_path, case):
    g = np.load(GOLDEN)
    path = R.write_dump(tmp_path / f"{case}.json", g[case + "_words"], frame=30, view=1)
    rays = g[case + "_rays"]
    with (tmp_path / f"{case}.jsonl").open("w") as f:
        for k, r in enumerate(rays):
            for any_hit in (False, True):
                rec = g[f"{case}_{'any' if any_hit else 'closest'}_record"][k]
                f.write(json.dumps(dict(frame=30, view=1, id=2 * k + any_hit, origin=r[0:3].tolist(), tmin=float(r[3]),
                                        direction=r[4:7].tolist(), tmax=float(r[7]), any_hit=any_hit,
                                        gpu_record=[int(x) for x in rec])) + "\n")
    return path, g


@pytest.mark.parametrize("case", ["flat", "tlas"])
def test_dump_loads_and_inventories(tmp_path, case):
    path, g = _write(tmp_path, case)
    d = R.Dump(path)
    inv = d.inventory()
    assert inv["written_instances"] == int(g[case + "_words"][0])
    assert sum(inv["mesh_instances"].values()) == inv["written_instances"]
    assert (inv["tlas"] is not None) == (case == "tlas")
    meta = json.loads(path.read_text())
    meta["format"] = "reflection-bvh4"
    path.write_text(json.dumps(meta))
    with pytest.raises(ValueError, match="format"):
        R.Dump(path)
    meta["format"] = R.FORMAT
    meta["payload_words"] += 1
    path.write_text(json.dumps(meta))
    with pytest.raises(ValueError, match="incomplete"):
        R.Dump(path)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["flat", "tlas"])
def test_replay_on_the_gpu_matches_the_reference_replay(engine, tmp_path, case):
    path, g = _write(tmp_path, case)
    s = R.replay(R.Dump(path), tmp_path / f"{case}.jsonl", tmp_path / "out", engine)
    assert s["rays"] == 2 * len(g[case + "_rays"]) == s["gpu_identity_checked"]
    assert s["gpu_identity_mismatches"] == 0
    closest = s["record"][0::2]
    assert np.array_equal(s["t"][0::2].view(np.uint32), g[case + "_closest_t"])
    assert np.array_equal(closest, g[case + "_closest_record"])
    assert (tmp_path / "out" / "rays.csv").exists() and (tmp_path / "out" / "replay-summary.json").exists()
