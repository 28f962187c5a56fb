"""Traversal benchmark: Mrays/s of the tuned traversal against the plain kernel at matched hits,
one JSON line on stdout.

Workloads (seeded synthetic scenes and rays; splitmix64, seed 0x5EED0000 + config):

* --config 3 (default) precision-4M: 4,000,000 cluster triangles (8,000 clusters of 500),
  reflection layout; per step 16,777,216 mixed rays: 8,388,608 primary (4096 x 2048 pinhole),
  5,033,164 cosine-hemisphere GI rays from the primary hits (closest hit) and 3,355,444 shadow
  any-hit rays toward 16 point lights. It is the one workload that carries the metric whole:
  closest and any-hit rays in one step, against the plain kernel at matched hits, with the FP64
  report. The scene (about 200 MB of packed words) does not fit the 126 MB L2.
* --config 2 clusters-1M: 1,000,000 triangles in 2,000 clusters, reflection layout;
  per step 4,194,304 coherent primary rays (2048 x 2048 pinhole from (0, 0, -250), fov 60 deg)
  plus 4,194,304 cosine-hemisphere GI rays spawned from the primary hits, closest hit.
* --config 1 cubes-120k: 10,000 jittered unit cubes merged into one BLAS, GI layout; 1024 x 1024
  primaries closest hit plus one sun any-hit ray per hit.
* --config 4 batching: 64 BLAS (2k-500k triangles, log-uniform) under 10,000 randomly rotated,
  scaled and placed instances; 64 ray batches (1k-2M rays, log-uniform), closest / any hit.
* --config 5 serving: 8 resident scenes (100k-8M triangles, BLAS + TLAS as config 4) under a
  120 GB HBM budget; Poisson request arrivals at each --rates value; each request 4k-4M rays
  (log-uniform) of shadow any-hit / GI closest / reflection closest (40/40/20) on a uniformly
  chosen scene, from pinned host memory to pinned host memory through rt_server; beside it the
  plain kernel serving the same arrivals one request at a time.

Per step, the "plain" arm launches the plain kernel once per batch; the product arm replays the
plans the autotuner chose (kernel, wavefront width, sort key; one CUDA graph per plan). Scenes
and rays are device resident; L2 is flushed (a 256 MiB write) before each step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config 1|2|3|4] [--kernel auto|plain|fast|wide8]
    python bench.py --impl reference ...   # the reference CPU traversal on the host cores

Under torchrun (N > 1) every rank traces the full per-GPU workload on its own GPU (rays are
independent: weak scaling, no collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s closest+any-hit vs plain kernel at matched hits, 1 B200; p50/p99 latency"
UNIT = "Mrays/s"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=3, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000", help="--config 5: Poisson arrival rates (req/s)")
    ap.add_argument("--requests", type=int, default=48, help="--config 5: requests per rate")
    ap.add_argument("--kernel", default="auto",
                    help="auto: the autotuner's choice; or plain / fast / wide8 / wide8p for every launch group, or "
                         "one of them a group, comma-separated")
    ap.add_argument("--refill", type=int, default=0, help="with --kernel fast/wide8: the wavefront width")
    ap.add_argument("--order", default="none", help="with --kernel fast/wide8: the sort key")
    ap.add_argument("--stack", default="", help="with --kernel wide8: local or shared node-group stack")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target wall time of the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--small", action="store_true", help="a reduced workload (profiling captures)")
    ap.add_argument("--precision", type=int, default=-1,
                    help="rays sampled for the FP64 check (default 65,536; 4,096 for --config 4), plus every ray "
                         "where the product and the plain kernel differ; 0 skips the check")
    ap.add_argument("--blas-build", action="store_true",
                    help="time the GPU BLAS build (rt_blas_build_device) against the host build on cluster meshes")
    return ap.parse_args(argv)


# ---------------------------------------------------------------- workloads

@dataclass
class Batch:
    label: str
    rays: np.ndarray  # (n, 8) float32
    mode: int         # 0 closest, 1/2 any hit


@dataclass
class Workload:
    name: str
    layout: int
    words: np.ndarray
    batches: list
    groups: list            # one tuned plan per group of batch indices
    triangles: int
    info: dict = field(default_factory=dict)

    @property
    def rays(self) -> int:
        return sum(len(b.rays) for b in self.batches)


def gpu_closest(engine, scene, rays, mode):
    """Rays traced by the plain kernel; the hits of a step's first batch spawn its later ones."""
    import torch
    h = engine.trace(scene, torch.from_numpy(rays).cuda(), mode, "plain")
    torch.cuda.synchronize()
    return h.cpu().numpy().view(np.uint32)


def _hits(layout, h):
    """(hit mask, t, primitive column) of closest-hit results."""
    from renderlab_b200 import api as A
    if layout == A.LAYOUT_GI:
        return h[:, 1] != A.MISS, h[:, 0].view(np.float32), h[:, 2]
    return h[:, 1] != 0, h[:, 0].view(np.float32), h[:, 2]


def engine_pack(layout, meshes, instances, primitives=None):
    """Packed words from the engine's host builders (rt_blas_build, rt_pack_scene)."""
    from concurrent.futures import ThreadPoolExecutor
    from renderlab_b200 import api as A
    with ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        blas = list(ex.map(lambda m: A.Blas(m.positions, m.indices), meshes))
    return A.pack_scene(layout, blas, instances, primitives=primitives)


def oracle_pack(layout, meshes, instances, primitives=None):
    """Packed words from the oracle's restatement of the reference builders and packers."""
    from oracle import oracle as O
    n = len(instances)
    if layout == 0:
        aux = np.zeros((n, 9), np.uint32)
        aux[:, 4] = (~instances.casts).astype(np.uint32)
    else:
        aux = np.stack([np.arange(n), instances.casts.astype(np.uint32)], axis=1).astype(np.uint32)
    inst = dict(model=instances.model, rows=instances.rows, mesh=instances.mesh, aux=aux)
    ms = [(m.positions, m.indices, 1 if (primitives and primitives[k]) else 0) for k, m in enumerate(meshes)]
    return O.scene_words(layout, ms, inst, -1)


def workload(config: int, engine, small: bool = False, pack=engine_pack, closest=gpu_closest) -> tuple:
    """(Workload, uploaded scene). `closest(engine, scene, rays, mode)` traces the rays whose
    hits spawn a step's secondary batches."""
    from renderlab_b200 import api as A
    from renderlab_b200 import scenes as S
    div = 4 if small else 1
    if config == 1:
        mesh = S.cubes_merged(100)
        layout = A.LAYOUT_GI
        words = pack(layout, [mesh], S.identity_instances(1), primitives=[True])
        scene = engine.upload(layout, words)
        w = 1024 // (2 if small else 1)
        primary = S.cube_camera_rays(w, w)
        hit, t, _ = _hits(layout, closest(engine, scene, primary, 0))
        sun = S.sun_rays(S.hit_points(primary[hit], t[hit]))
        return Workload(f"cubes-120k: 10,000 jittered unit cubes ({mesh.triangles:,} triangles) merged into one BLAS, "
                        f"GI layout; {len(primary):,} primary closest-hit + {len(sun):,} sun any-hit rays per step",
                        layout, words, [Batch("primary", primary, 0), Batch("sun", sun, 2)], [[0], [1]],
                        mesh.triangles, dict(primary_hit_rate=float(hit.mean()))), scene
    if config in (2, 3):
        n_tris = (1_000_000 if config == 2 else 4_000_000) // div
        mesh = S.clusters(n_tris, config=config)
        layout = A.LAYOUT_REFLECTION
        words = pack(layout, [mesh], S.identity_instances(1))
        scene = engine.upload(layout, words)
        if config == 2:
            w = 2048 // (2 if small else 1)
            primary = S.cluster_camera_rays(w, w)
        else:
            primary = S.cluster_camera_rays(4096 // (2 if small else 1), 2048 // (2 if small else 1))
        hit, t, prim = _hits(layout, closest(engine, scene, primary, 0))
        pts = S.hit_points(primary[hit], t[hit])
        normals = S.triangle_normals(mesh, prim[hit])
        if config == 2:
            gi = S.hemisphere_rays(pts, normals, primary[hit, 4:7], len(primary), S.Stream(S.seed_for(2) + 1))
            return Workload(f"clusters-1M: {mesh.triangles:,} triangles in clusters of 500 (reflection layout); "
                            f"{len(primary):,} primary + {len(gi):,} GI hemisphere rays per step, closest hit",
                            layout, words, [Batch("primary", primary, 0), Batch("gi", gi, 0)], [[0], [1]],
                            mesh.triangles, dict(primary_hit_rate=float(hit.mean()))), scene
        total = 2 * len(primary)
        n_gi = (3 * total) // 10
        n_sh = total - len(primary) - n_gi
        gi = S.hemisphere_rays(pts, normals, primary[hit, 4:7], n_gi, S.Stream(S.seed_for(3) + 1))
        shadow = S.point_light_rays(pts, normals, n_sh, 16, 100.0, S.Stream(S.seed_for(3) + 2))
        return Workload(f"precision-4M: {mesh.triangles:,} cluster triangles (reflection layout); {total:,} rays per "
                        f"step: {len(primary):,} primary, {len(gi):,} GI hemisphere (closest), {len(shadow):,} shadow "
                        "any-hit toward 16 point lights", layout, words,
                        [Batch("primary", primary, 0), Batch("gi", gi, 0), Batch("shadow", shadow, 2)],
                        [[0], [1], [2]], mesh.triangles, dict(primary_hit_rate=float(hit.mean()))), scene
    ms = S.multi_blas(n_instances=10_000 // div)
    layout = A.LAYOUT_REFLECTION
    words = pack(layout, ms.meshes, ms.instances)
    scene = engine.upload(layout, words)
    batches = [Batch(f"b{k}", r, m) for k, (r, m) in enumerate(S.uneven_batches(hi=2e6 / div))]
    tris = sum(m.triangles for m in ms.meshes)
    return Workload(f"batching: {len(ms.meshes)} BLAS ({tris:,} triangles, 2k-500k each) under {len(ms.instances):,} "
                    f"rotated/scaled instances (reflection layout, TLAS); {len(batches)} batches of "
                    f"{min(len(b.rays) for b in batches):,}-{max(len(b.rays) for b in batches):,} rays "
                    f"({sum(len(b.rays) for b in batches):,} total, {sum(1 for b in batches if b.mode)} any-hit) "
                    "in one persistent launch", layout, words, batches, [list(range(len(batches)))], tris,
                    dict(instances=len(ms.instances))), scene


# ---------------------------------------------------------------- measurement helpers

class Clocks:
    """nvidia-smi sampler (200 ms) over the timed region."""

    FIELDS = "index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self):
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self, bus_id):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 10 and (bus_id is None or _bus_of(parts[1]) == bus_id):
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = np.array([float(r[2]) for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower() == "active"})
        power = [float(r[4]) for r in rows if r[4] not in ("", "[N/A]")]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][3]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(power) if power else None}


def _bus_of(pci: str):
    """The bus number of an nvidia-smi pci.bus_id ("00000000:E5:00.0")."""
    try:
        return int(pci.split(":")[1], 16)
    except (IndexError, ValueError):
        return None


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bvh4_bytes(counters, n_rays, layout, hit_bytes):
    """Algorithmic bytes of the BVH4-Q8 walk: ray 32 + hit + 128 per top-level node + the
    instance record per box test (GI 128, reflection 96) + 64 per BLAS node + 48 per triangle
    (GI: 8 more per leaf for its index span)."""
    c = counters
    rec = 128 if layout == 0 else 96
    return (32 + hit_bytes) * n_rays + 128 * c["tlas_nodes"] + rec * c["instance_box_tests"] \
        + 64 * c["blas_nodes"] + 48 * c["triangle_tests"] + (8 * c["leaves"] if layout == 0 else 0)


def wide8_bytes(counters, layout, hit_bytes):
    """The same for the 8-wide walk: 80 per node, 48 per triangle, 128 per top-level node, the
    instance record (and 8 bytes of its 8-wide table) per instance test."""
    c = counters
    rec = (128 if layout == 0 else 96) + 8
    return (32 + hit_bytes) * c["rays"] + 128 * c["top_nodes"] + rec * c["instance_tests"] + 80 * c["nodes"] \
        + 48 * c["triangles"]


# DRAM bytes per ray (read + write) that ncu measured on the dominant launch -- the GI batch's
# k_wide8 -- by (config, --small, kernel). Captured with
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum --clock-control none
#       -k regex:^k_wide8$ -s 1 -c 1 python bench.py [--small] --steps 1 --warmup 3 --no-cpu --precision 0 --kernel wide8
# (one pass; the launch is the first warm-up step's GI batch): precision-4M 944.3 MB read + 451.2 MB
# written for 5,033,164 rays; the 1M-triangle reduced case 234.5 + 103.0 MB for 1,258,291 rays (an
# earlier build, before the walk's ray and hit streams took the evict-first form).
# clusters-1M (--config 2 ... --kernel wide8p,wide8 --refill 8, -s 2: the first warm-up step's GI
# batch): 518.6 MB read + 319.8 MB written for 4,194,304 rays.
TRAFFIC = {(3, False, "k_wide8"): (944.30e6 + 451.18e6) / 5_033_164, (3, True, "k_wide8"): (234.53e6 + 102.95e6) / 1_258_291,
           (2, False, "k_wide8"): (518.57e6 + 319.81e6) / 4_194_304}


def hit_bytes(layout, mode):
    return 4 if mode else (40 if layout == 0 else 20)


def oracle_trace(words, layout, rays, mode, counters=False, threads=None):
    from oracle import oracle as O
    if layout == 0:
        return O.gi_trace(words, rays, mode, counters=counters, threads=threads)
    return O.rs_trace(words, rays, mode != 0, counters=counters, threads=threads)


def sample_of(wl: Workload, n_total: int):
    """A strided sample of every batch, n_total rays in proportion to the batch sizes."""
    frac = min(1.0, n_total / max(1, wl.rays))
    out = []
    for b in wl.batches:
        k = max(1, int(round(len(b.rays) * frac)))
        stride = max(1, len(b.rays) // k)
        out.append(b.rays[::stride][:k])
    return out, frac


def cpu_baseline_leg(wl: Workload, target_s: float, threads=None):
    """The reference traversal (the oracle's restatement of the WGSL loop) on the host cores over
    a strided sample of every batch of the step; also returns per-batch visit counters."""
    threads = threads or (os.cpu_count() or 1)
    probe, _ = sample_of(wl, 4096)
    t0 = time.perf_counter()
    for b, r in zip(wl.batches, probe):
        oracle_trace(wl.words, wl.layout, r, b.mode, threads=threads)
    per_ray = (time.perf_counter() - t0) / sum(len(r) for r in probe)
    def timed(n_rays):
        smp, f = sample_of(wl, n_rays)
        t0 = time.perf_counter()
        for b, r in zip(wl.batches, smp):
            oracle_trace(wl.words, wl.layout, r, b.mode, threads=threads)
        return smp, f, time.perf_counter() - t0

    sample, frac, wall = timed(int(max(4096, target_s / max(per_ray, 1e-9))))
    n = sum(len(r) for r in sample)
    if wall < 0.5 * target_s and frac < 1.0:  # the small probe overstated the cost a ray: resize once
        sample, frac, wall = timed(int(n * target_s / max(wall, 1e-3)))
        n = sum(len(r) for r in sample)
    counts = [oracle_trace(wl.words, wl.layout, r, b.mode, counters=True, threads=threads)[1]
              for b, r in zip(wl.batches, sample)]
    # the same traversal on one core, over a sample sized for about a tenth of the time
    one, _ = sample_of(wl, int(max(1024, 0.1 * target_s / max(per_ray * threads, 1e-9))))
    t0 = time.perf_counter()
    for b, r in zip(wl.batches, one):
        oracle_trace(wl.words, wl.layout, r, b.mode, threads=1)
    one_wall = time.perf_counter() - t0
    n_one = sum(len(r) for r in one)
    # and the FP64 reference traversal (reference.rs restated) on at most 65,536 rays of the sample
    from oracle import oracle as O
    sub, _ = sample_of(wl, 65_536)
    t0 = time.perf_counter()
    for b, r in zip(wl.batches, sub):
        if len(r):
            O.fp64_trace(wl.words, r, wl.layout, any_hit=b.mode != 0, threads=threads)
    f64_wall = time.perf_counter() - t0
    n_f64 = sum(len(r) for r in sub)
    return dict(value=n / wall / 1e6, unit=UNIT, cores=threads, kind="port",
                sample=f"{n:,} rays ({100 * frac:.2f} % of each batch of the step, strided), oracle "
                       f"{'gi_traverse' if wl.layout == 0 else 'rs_trace'} (scalar f32 C++) on {threads} threads, "
                       f"{wall:.2f} s",
                one_core=dict(value=n_one / one_wall / 1e6, unit=UNIT, rays=n_one),
                fp64=dict(value=n_f64 / f64_wall / 1e6, unit=UNIT, rays=n_f64, cores=threads)), \
        (counts, [len(r) for r in sample])


T_REL, TIE_REL, BARY_ABS = 1e-5, 1e-6, 1e-5


def fp64_classify(layout: int, mode: int, got: np.ndarray, rays: np.ndarray, r64: np.ndarray, ident: np.ndarray):
    """Each ray's result against the FP64 oracle's (r64 = [hit, t, u, v], ident). Returns
    (status, t_rel, bary_abs): status 0 the same hit (identity, or the any-hit flag), 1 a near tie
    (both hit, different identity, |t - t64| <= 1e-6 t64; any hit: the FP64 hit within 1e-5
    relative of tmin or tmax), 2 unexplained. t_rel and bary_abs are NaN except where status is 0
    and both hit: |t - t64| / t64 and max(|u - u64|, |v - v64|) (barycentrics range over [0, 1],
    so their error is taken against that range)."""
    ohit = r64[:, 0] > 0
    n = len(got)
    t_rel = np.full(n, np.nan)
    bary = np.full(n, np.nan)
    if mode:
        ghit = got.reshape(n) != 0
        t64 = r64[:, 1]
        near = ohit & ((np.abs(t64 - rays[:, 7]) <= T_REL * np.abs(rays[:, 7]))
                       | (np.abs(t64 - rays[:, 3]) <= T_REL * np.maximum(np.abs(rays[:, 3]), 1e-30)))
        status = np.where(ghit == ohit, 0, np.where(near, 1, 2))
        return status, t_rel, bary
    cols, ocols, uv = (slice(1, 3), slice(2, 4), slice(3, 5)) if layout == 1 else (slice(1, 5), slice(2, 6), slice(5, 7))
    ghit = got[:, 1] != (0 if layout == 1 else 0xFFFFFFFF)
    t = got[:, 0].view(np.float32).astype(np.float64)
    t64 = r64[:, 1]
    both = ghit & ohit
    same = both & (got[:, cols] == ident[:, ocols]).all(1)
    m = (ghit != ohit) | (both & ~same)
    tie = m & both & (np.abs(t - t64) <= TIE_REL * np.abs(t64))
    status = np.where(~m, 0, np.where(tie, 1, 2))
    t_rel[same] = np.abs(t[same] - t64[same]) / np.maximum(np.abs(t64[same]), 1e-30)
    g_uv = got[:, uv].view(np.float32).astype(np.float64)
    bary[same] = np.abs(g_uv[same] - r64[same, 2:4]).max(1)
    return status, t_rel, bary


def precision_report(wl: Workload, results: dict, n_sample: int, diff: list | None = None) -> dict:
    """Each arm's results against the FP64 oracle, per batch, on a strided sample of every batch
    plus (for the product arm) every ray where the product and the plain kernel disagree.

    Per batch and arm: the sample's hit-identity mismatch rate, near ties and unexplained
    mismatches; t error (relative) and barycentric error (absolute, on [0, 1]) over the sample's
    matching hits, max and mean. For the product arm, `vs_plain` classifies every ray where the
    two arms differ: the product agrees with FP64 (the plain kernel's f32 arithmetic erred), a
    near tie, or unexplained."""
    from oracle import oracle as O
    frac = min(1.0, n_sample / max(1, wl.rays))
    idx = [np.arange(0, len(b.rays), max(1, int(round(1 / frac)))) if len(b.rays) else np.zeros(0, np.int64)
           for b in wl.batches]
    diff = diff or [np.zeros(0, np.int64) for _ in wl.batches]
    out = {}
    ref = []
    for b, ix, dx in zip(wl.batches, idx, diff):
        ids = np.union1d(ix, dx).astype(np.int64)
        ref.append((ids, O.fp64_trace(wl.words, b.rays[ids], wl.layout, any_hit=b.mode != 0) if len(ids) else None))
    for arm, (hits, kernels) in results.items():
        per = {}
        for b, ix, dx, (ids, r), h, kern in zip(wl.batches, idx, diff, ref, hits, kernels):
            if r is None:
                continue
            r64, ident = r
            status, t_rel, bary = fp64_classify(wl.layout, b.mode, h[ids], b.rays[ids], r64, ident)
            smp = np.isin(ids, ix)
            st = status[smp]
            rec = dict(kernel=kern, rays=int(smp.sum()), mismatch_rate=float((st != 0).mean()) if len(st) else 0.0,
                       near_ties=int((st == 1).sum()), unexplained=int((st == 2).sum()))
            if not b.mode:
                tr, ba = t_rel[smp], bary[smp]
                tr, ba = tr[~np.isnan(tr)], ba[~np.isnan(ba)]
                rec.update(t_rel_max=float(tr.max()) if len(tr) else 0.0, t_rel_mean=float(tr.mean()) if len(tr) else 0.0,
                           bary_abs_max=float(ba.max()) if len(ba) else 0.0,
                           bary_abs_mean=float(ba.mean()) if len(ba) else 0.0)
            if arm == "product":
                dm = np.isin(ids, dx)
                sd = status[dm]
                rec["vs_plain"] = dict(differing=int(len(dx)), agrees_with_fp64=int((sd == 0).sum()),
                                       near_ties=int((sd == 1).sum()), unexplained=int((sd == 2).sum()))
            per[b.label] = rec
        out[arm] = per
    tot = lambda arm, key: sum(v.get(key, 0) for v in out.get(arm, {}).values())
    out["summary"] = dict(
        product_unexplained=tot("product", "unexplained")
        + sum(v["vs_plain"]["unexplained"] for v in out.get("product", {}).values() if "vs_plain" in v),
        product_t_rel_max=max([v.get("t_rel_max", 0.0) for v in out.get("product", {}).values()] or [0.0]),
        product_bary_abs_max=max([v.get("bary_abs_max", 0.0) for v in out.get("product", {}).values()] or [0.0]),
        bar=f"ids equal except near ties (|dt| <= {TIE_REL:g} t); t within {T_REL:g} relative; "
            f"barycentrics within {BARY_ABS:g}")
    return out


# ---------------------------------------------------------------- arms

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float) -> float:
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class HostScene:
    """The reference arm's scene holder: it builds the workload without a GPU."""

    def __init__(self):
        self.layout, self.words = None, None

    def upload(self, layout, words):
        self.layout, self.words = layout, words
        return self


def reference_serving(args):
    """Config 5 on the host cores: the oracle over a sample of every scene's three ray kinds."""
    from renderlab_b200 import scenes as S
    scenes = serving_scenes(args.small)
    rng = S.Stream(S.seed_for(5) + 7)
    threads = os.cpu_count() or 1
    n, wall = 0, 0.0
    for m in scenes:
        words = oracle_pack(1, m.meshes, m.instances)
        for kind, mode in (("shadow", 2), ("gi", 0), ("refl", 0)):
            rays = serving_rays(kind, 256, 500.0, rng)
            t0 = time.perf_counter()
            oracle_trace(words, 1, rays, mode, threads=threads)
            wall += time.perf_counter() - t0
            n += len(rays)
    value = n / wall / 1e6
    return value, dict(value=value, unit=UNIT, cores=threads, kind="port",
                       sample=f"{n:,} rays: 256 of each kind per scene, oracle rs_trace on {threads} threads, {wall:.2f} s")


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return  # rank 0 alone times the host-core reference
    if args.config == 5:
        value, cpu_line = reference_serving(args)
        print(json.dumps(dict(metric=METRIC, value=value, unit=UNIT, impl="reference", n_gpus=world, steps=args.steps,
                              warmup=args.warmup, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                              data="synthetic", config=dict(workload="serving scenes (config 5), oracle sample", config=5),
                              cpu_baseline=cpu_line, ms_per_step=None,
                              e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))), flush=True)
        return
    holder = HostScene()

    def cpu_closest(engine, scene, rays, mode):
        return oracle_trace(holder.words, holder.layout, rays, mode)[0]

    wl, _ = workload(args.config, holder, args.small, pack=oracle_pack, closest=cpu_closest)
    threads = os.cpu_count() or 1
    # One strided sample of every batch, sized once from a probe so that a step is about
    # min(20, 120 / steps) seconds of traversal; every step times the same sample.
    per_step = max(1.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    probe, _ = sample_of(wl, 4096)
    t0 = time.perf_counter()
    for b, r in zip(wl.batches, probe):
        oracle_trace(wl.words, wl.layout, r, b.mode, threads=threads)
    per_ray = (time.perf_counter() - t0) / sum(len(r) for r in probe)
    sample, frac = sample_of(wl, int(max(4096, per_step / max(per_ray, 1e-9))))
    n = sum(len(r) for r in sample)
    values, walls = [], []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for b, r in zip(wl.batches, sample):
            oracle_trace(wl.words, wl.layout, r, b.mode, threads=threads)
        wall = time.perf_counter() - t0
        if k >= args.warmup:
            values.append(n / wall / 1e6)
            walls.append(wall)
    value = float(np.median(values))
    cpu_line = dict(value=value, unit=UNIT, cores=threads, kind="port",
                    sample=f"{n:,} rays a step ({100 * frac:.2f} % of each batch of the step, strided), oracle "
                           f"{'gi_traverse' if wl.layout == 0 else 'rs_trace'} (scalar f32 C++) on {threads} threads, "
                           f"median {float(np.median(walls)):.2f} s a step")
    line = dict(metric=METRIC, value=value, unit=UNIT, impl="reference", n_gpus=world, steps=args.steps,
                warmup=args.warmup, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                data="synthetic", config=workload_config(wl, args.config),
                cpu_baseline=cpu_line, e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                ms_per_step=None, note="oracle restatement of the WGSL traversal loop on the host cores: the Rust/WGSL "
                                       "reference cannot run here (no rustc, no Vulkan/wgpu); each step traces the "
                                       "same strided sample of the step's rays")
    print(json.dumps(line), flush=True)


def workload_config(wl: Workload, config: int) -> dict:
    """The `config` object of the JSON line: the same on both arms for one workload."""
    return dict(workload=wl.name, config=config, layout="GI" if wl.layout == 0 else "reflection")


# ---------------------------------------------------------------- serving (config 5)

def serving_scenes(small: bool):
    """8 scenes, triangle counts log-uniform in [1e5, 8e6] (in [2.5e4, 2e6] with --small): 8 BLAS
    each (log-uniform shares) under 512 instances placed as in config 4."""
    from renderlab_b200 import scenes as S
    s = S.Stream(S.seed_for(5))
    lo, hi = (1e5, 8e6) if not small else (2.5e4, 2e6)
    totals = np.round(np.exp(s.range(np.log(lo), np.log(hi), 8))).astype(np.int64)
    out = []
    for k, t in enumerate(totals):
        ms = S.multi_blas(n_blas=8, n_instances=512, tri_lo=max(500.0, t / 16), tri_hi=max(1000.0, t / 4),
                          config=5 + 16 * (k + 1))
        out.append(ms)
    return out


def serving_rays(kind: str, n: int, half: float, stream):
    from renderlab_b200 import scenes as S
    o = stream.range(-half, half, n, 3)
    if kind == "shadow":  # toward a random point of the box, stopping short of it
        v = stream.range(-half, half, n, 3) - o
        dist = np.maximum(np.linalg.norm(v, axis=1), 1e-3)
        return S.pack_rays(o, v / dist[:, None], 0.0, dist * (1.0 - 1e-4))
    return S.pack_rays(o, stream.unit_vectors(n), 0.0, 1e30)


def run_serving(args):
    import threading
    import torch
    from renderlab_b200 import api as A
    from renderlab_b200 import scenes as S
    engine = A.Engine(0)
    kernel = "wide8" if args.kernel == "auto" else args.kernel
    scenes = serving_scenes(args.small)
    words = [engine_pack(A.LAYOUT_REFLECTION, m.meshes, m.instances) for m in scenes]
    tris = [sum(x.triangles for x in m.meshes) for m in scenes]
    budget = 120 << 30
    srv = A.Server(engine, hbm_budget=budget, launch_rays=1 << 22, slots=4, kernel=kernel)
    ids = [srv.add_scene(A.LAYOUT_REFLECTION, w) for w in words]
    plain_scenes = [engine.upload(A.LAYOUT_REFLECTION, w) for w in words]
    rng = S.Stream(S.seed_for(5) + 7)
    lo, hi = (4e3, 4e6) if not args.small else (1e3, 1e6)
    pools = {k: torch.from_numpy(serving_rays(k, int(hi), 500.0, rng)).pin_memory() for k in ("shadow", "gi", "refl")}
    rates = [float(x) for x in args.rates.split(",")]
    per_rate = []
    total_rays, total_s = 0, 0.0
    bus = None
    try:
        bus = torch.cuda.get_device_properties(0).pci_bus_id
    except AttributeError:
        pass
    clocks = Clocks()
    clocks.start()
    for rate in rates:
        n_req = args.requests
        gaps = -np.log(1.0 - rng.uniform(n_req)) / rate
        arrive = np.cumsum(gaps)
        sizes = np.round(np.exp(rng.range(np.log(lo), np.log(hi), n_req))).astype(np.int64)
        u = rng.uniform(n_req)
        kinds = np.where(u < 0.4, "shadow", np.where(u < 0.8, "gi", "refl"))
        which = np.minimum((rng.uniform(n_req) * len(ids)).astype(np.int64), len(ids) - 1)
        modes = [A.ANY_CASTERS if k == "shadow" else A.CLOSEST for k in kinds]
        reqs = [(int(which[i]), modes[i], pools[kinds[i]][: int(sizes[i])]) for i in range(n_req)]
        # every request its own slice of one pinned output buffer (overlapping requests share none)
        words_of = [5 if m == A.CLOSEST else 1 for m in modes]
        pool = torch.empty(int(sum(int(z) * w for z, w in zip(sizes, words_of))), dtype=torch.int32).pin_memory()
        outs, at = [], 0
        for z, w in zip(sizes, words_of):
            outs.append(pool[at: at + int(z) * w].view(int(z), w) if w > 1 else pool[at: at + int(z)])
            at += int(z) * w
        srv.stats(reset=True)
        tickets = [None] * n_req
        t0 = time.perf_counter()

        def producer():
            for i, (sid, mode, rays) in enumerate(reqs):
                delay = t0 + arrive[i] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = srv.submit(ids[sid], rays, mode, out=outs[i])

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        for t in tickets:
            srv.wait(t)
        wall = time.perf_counter() - t0
        st = srv.stats()
        rays = int(sizes.sum())
        # the plain kernel, one request at a time, on the same arrivals
        lat = []
        t0 = time.perf_counter()
        for i, (sid, mode, rays_i) in enumerate(reqs):
            delay = t0 + arrive[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            engine.trace_host(plain_scenes[sid], rays_i, mode, "plain", out=outs[i])
            lat.append((time.perf_counter() - t0 - arrive[i]) * 1e3)
        wall_plain = time.perf_counter() - t0
        per_rate.append(dict(rate=rate, requests=n_req, rays=rays, mrays=rays / wall / 1e6, p50_ms=st["p50_ms"],
                             p99_ms=st["p99_ms"], max_ms=st["max_ms"], launches=st["launches"],
                             offered_mrays=rays / float(arrive[-1]) / 1e6,
                             plain=dict(mrays=rays / wall_plain / 1e6, p50_ms=float(np.percentile(lat, 50)),
                                        p99_ms=float(np.percentile(lat, 99)), max_ms=float(np.max(lat)))))
        total_rays += rays
        total_s += wall
    clk = clocks.stop(bus)
    dev_bytes = srv.stats()["device_bytes"]
    srv.close()
    for sc in plain_scenes:
        sc.release()
    top = per_rate[-1]
    line = dict(metric=METRIC, value=total_rays / total_s / 1e6, unit=UNIT, n_gpus=1, steps=len(rates) * args.requests,
                warmup=0, ms_per_step=total_s / (len(rates) * args.requests) * 1e3, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                config=dict(workload=f"serving: 8 scenes ({', '.join(f'{t:,}' for t in tris)} triangles; 8 BLAS + "
                                     f"TLAS of 512 instances each) resident under a {budget >> 30} GB HBM budget "
                                     f"({dev_bytes / 1e9:.1f} GB used); Poisson arrivals, {args.requests} requests a "
                                     f"rate of {int(lo):,}-{int(hi):,} rays (shadow / GI / reflection 40/40/20)",
                            config=5, kernel=kernel, launch_rays=1 << 22, slots=4),
                latency_ms=dict(p50=top["p50_ms"], p99=top["p99_ms"], plain_p50=top["plain"]["p50_ms"],
                                plain_p99=top["plain"]["p99_ms"]),
                rates=per_rate, clocks=clk,
                e2e=dict(value=total_rays / total_s / 1e6, unit=UNIT, h2d_bytes_per_step=None, d2h_bytes_per_step=None,
                         path="rt_server_submit / rt_server_wait, pinned host buffers; timed from each rate's first "
                              "arrival to its last completion"),
                note="a step is one request; value = rays served / wall time over all rates")
    print(json.dumps(line), flush=True)
    engine.close()



def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from renderlab_b200 import api as A
    from renderlab_b200 import tune as T
    engine = A.Engine(local)
    wl, scene = workload(args.config, engine, args.small)
    t_prep = time.perf_counter()
    # --kernel: "auto" (the autotuner), one kernel for every launch group, or one a group
    # ("wide8p,wide8,wide8": how a profiling capture pins the plans the tuner chose)
    forced = args.kernel.split(",") if args.kernel != "auto" else []
    if forced and len(forced) == 1:
        forced = forced * len(wl.groups)
    if forced and len(forced) != len(wl.groups):
        raise SystemExit(f"--kernel names {len(forced)} kernels for {len(wl.groups)} launch groups")
    if args.kernel == "auto" or any(k in ("wide8", "wide8p") for k in forced):
        scene.prepare("wide8")  # derived layouts (the 8-wide BVH) are scene-upload work, untimed
    t_prep = time.perf_counter() - t_prep
    dev = [torch.from_numpy(b.rays).cuda() for b in wl.batches]

    def hit_tensor(b):
        words = A.hit_words(wl.layout, b.mode)
        return torch.empty((len(b.rays), words) if words > 1 else (len(b.rays),), dtype=torch.int32, device="cuda")

    plain_hits = [hit_tensor(b) for b in wl.batches]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    # ---- product plans: one per group, from the autotuner (or the forced kernel)
    t_tune = time.perf_counter()
    plans, tables = [], []
    for gk, g in enumerate(wl.groups):
        batches = [(dev[i], wl.batches[i].mode) for i in g]
        if args.kernel == "auto":
            heavy = len(g) > 8  # the many-batch launch runs for seconds: one timed launch a candidate,
            # and no packet walk (its incoherent random rays would take many seconds a trial)
            ch = T.tune(engine, scene, batches, flush=flush, reps=1 if heavy else 3, max_seconds=20.0,
                        kernels=("plain", "fast", "wide8") if heavy else T.KERNELS)
            plans.append(ch.plan)
            tables.append(ch.table()[:6])
        elif forced[gk] == "plain":
            plans.append(None)
        else:
            plans.append(engine.plan(scene, batches, forced[gk], refill=args.refill, order=args.order,
                                     stack=args.stack if forced[gk] == "wide8" else ""))
    t_tune = time.perf_counter() - t_tune

    def plain_step():
        for i, b in enumerate(wl.batches):
            engine.trace(scene, dev[i], b.mode, "plain", hits=plain_hits[i])

    def product_step(evs=None):
        for k, (g, p) in enumerate(zip(wl.groups, plans)):
            if evs is not None:
                evs[k].record(stream)
            if p is None:
                for i in g:
                    engine.trace(scene, dev[i], wl.batches[i].mode, "plain", hits=plain_hits[i])
            else:
                p.launch()
        if evs is not None:
            evs[-1].record(stream)

    for _ in range(max(3, args.warmup)):
        flush.zero_()
        plain_step()
        flush.zero_()
        product_step()
    torch.cuda.synchronize()
    # matched hits: product results against the plain kernel's, per ray (ids, or the any-hit flag);
    # the rays that differ go to the FP64 classification below
    matched, n_all = 0, 0
    diff = [np.zeros(0, np.int64) for _ in wl.batches]
    for g, p in zip(wl.groups, plans):
        for j, i in enumerate(g):
            ref = plain_hits[i]
            got = p.hits[j] if p is not None else ref
            if ref.dim() == 2:
                cols = slice(1, 3) if wl.layout == A.LAYOUT_REFLECTION else slice(1, 5)
                same = (got[:, cols] == ref[:, cols]).all(1)
            else:
                same = got == ref
            matched += int(same.sum().item())
            n_all += ref.shape[0]
            diff[i] = torch.nonzero(~same).flatten().cpu().numpy().astype(np.int64)

    bus = None
    try:
        bus = torch.cuda.get_device_properties(local).pci_bus_id
    except AttributeError:
        pass

    def timed(fn_step, groups):
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(groups + 1)] for _ in range(args.steps)]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            fn_step(evs[k])
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        return np.array([[evs[k][j].elapsed_time(evs[k][j + 1]) for j in range(groups)] for k in range(args.steps)])

    def plain_timed(evs):
        evs[0].record(stream)
        plain_step()
        evs[1].record(stream)

    clocks = Clocks()
    clocks.start()
    wall0 = time.perf_counter()
    prod_ms = timed(product_step, len(wl.groups))
    plain_ms = timed(plain_timed, 1)
    wall = time.perf_counter() - wall0
    clk = clocks.stop(bus)
    step_ms = prod_ms.sum(1)
    ms = float(step_ms.mean())
    ms_plain = float(plain_ms.sum(1).mean())
    if world > 1:
        ms, ms_plain = max_over_ranks(ms), max_over_ranks(ms_plain)
    n_step = wl.rays
    value = world * n_step / (ms * 1e-3) / 1e6
    plain_value = world * n_step / (ms_plain * 1e-3) / 1e6

    # e2e through the host-buffer C ABI call, with each group's kernel and wavefront width
    pinned = [torch.from_numpy(b.rays).pin_memory() for b in wl.batches]
    outs = [torch.empty(tuple(h.shape), dtype=torch.int32).pin_memory() for h in plain_hits]
    engine.reserve(min(max(len(b.rays) for b in wl.batches), 1 << 22))

    host_batches, tuning = [], {}
    for g, p in zip(wl.groups, plans):
        kern = p.desc["kernel"] if p is not None else "plain"
        if kern == "wide8":
            tuning.update(wide8_refill=p.desc["refill"] or 8, wide8_stack=A.STACKS[p.desc.get("stack", "local")])
        elif kern == "fast":
            tuning.update(fast_refill=p.desc["refill"] or 8)
        host_batches += [(pinned[i], wl.batches[i].mode, kern, outs[i]) for i in g]
    if tuning:
        engine.set_tuning(**tuning)

    def host_step():  # every batch of the step in one host-buffer pipeline
        engine.trace_host_batches(scene, host_batches)

    host_step()
    e2e_steps = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        e2e_s = max_over_ranks(e2e_s)
    e2e = dict(value=world * n_step / e2e_s / 1e6, unit=UNIT, h2d_bytes_per_step=n_step * 32,
               d2h_bytes_per_step=int(sum(len(b.rays) * hit_bytes(wl.layout, b.mode) for b in wl.batches)),
               ms_per_step=e2e_s * 1e3, path="rt_trace_host_batches (pinned host rays in, host hits out, the step's batches in one pipeline)")

    if rank != 0:
        return
    cpu, counts = (None, None)
    if not args.no_cpu:
        cpu, counts = cpu_baseline_leg(wl, args.cpu_seconds)
    peak, peak_kind = measured_peak()
    roof = None
    notes = []
    # Algorithmic bytes of each group's launch: the 8-wide walk's visit counters (every 16th ray)
    # for WIDE8 and its packet walk (which serves the same per-ray walks), else the oracle's BVH4
    # counters on its CPU sample.
    group_bytes = []
    for g, p in zip(wl.groups, plans):
        kern = p.desc["kernel"] if p is not None else "plain"
        gb = 0.0
        for i in g:
            b = wl.batches[i]
            hb = hit_bytes(wl.layout, b.mode)
            if kern in ("wide8", "wide8p"):
                c = engine.trace_counted(scene, dev[i][::16].contiguous(), b.mode, "wide8")
                gb += wide8_bytes(c, wl.layout, hb) * len(b.rays) / max(1, c["rays"])
            elif counts is not None:
                cnt, nsamp = counts
                gb += bvh4_bytes(cnt[i], nsamp[i], wl.layout, hb) * len(b.rays) / max(1, nsamp[i])
            else:
                gb = None
                notes.append("no oracle counters (--no-cpu): BVH4 bytes not counted")
                break
        group_bytes.append(gb)
    group_ms = prod_ms.mean(0)
    dom = int(np.argmax(group_ms))
    if group_bytes[dom]:
        p = plans[dom]
        kern = p.desc["kernel"] if p is not None else "plain"
        name = {"wide8": "k_wide8", "wide8p": "k_wide8_packet"}.get(
            kern, ("k_gi_" if wl.layout == A.LAYOUT_GI else "k_rs_") + kern)
        rays_dom = sum(len(wl.batches[i].rays) for i in wl.groups[dom])
        achieved = group_bytes[dom] / (group_ms[dom] * 1e-3) / 1e9
        traffic = TRAFFIC.get((args.config, bool(args.small), name))
        roof = dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                    traffic=traffic * rays_dom if traffic else None,
                    kernel=name, launch="+".join(wl.batches[i].label for i in wl.groups[dom]),
                    launch_ms=float(group_ms[dom]), share_of_step=float(group_ms[dom] / group_ms.sum()),
                    peak_source=f"{peak_kind} hbm_gbs", bytes_per_ray=group_bytes[dom] / rays_dom,
                    note="the longest launch of a step: its algorithmic bytes (visit counters) over its CUDA-event "
                         "time; scenes under 126 MB are L2-resident, so the HBM fraction is a ceiling check, "
                         "not the limit; traffic is ncu's DRAM bytes per ray on this launch, scaled to its rays")
        if all(x is not None for x in group_bytes):
            roof["step_achieved"] = sum(group_bytes) / (ms * 1e-3) / 1e9
        # The L2 ceiling beside the HBM one: this device's read bandwidth over a 48 MiB buffer
        # (L2-resident) and a 4 GiB one (HBM), measured here with rt_read_bandwidth.
        try:
            l2 = engine.read_bandwidth(48 << 20, 50)
            hbm_read = engine.read_bandwidth(4 << 30, 3)
            roof["l2"] = dict(peak=l2, unit="GB/s", frac=achieved / l2, hbm_read_peak=hbm_read,
                              note="read bandwidth measured in this run (16-byte loads, L1 bypassed) over a "
                                   "48 MiB buffer (L2) and a 4 GiB buffer (HBM); the algorithmic bytes are "
                                   "served by L1 and L2 when the scene fits L2, so this is the tighter ceiling")
        except Exception as exc:  # the probe needs 4 GiB free
            roof["l2"] = dict(peak=None, note=f"not measured: {exc}")
    def launches(g, p):  # traversal kernels (and ray-key kernels) a step launches
        if p is None or p.desc["kernel"] == "plain":
            return sum(1 for i in g if len(wl.batches[i].rays))
        return 1 + (1 if p.desc["order"] != "none" else 0)

    launches_per_step = sum(launches(g, p) for g, p in zip(wl.groups, plans))
    n_prec = args.precision if args.precision >= 0 else (4_096 if args.config == 4 else 65_536)
    precision = None
    if n_prec:
        prod = [None] * len(wl.batches)
        for g, p in zip(wl.groups, plans):
            for j, i in enumerate(g):
                prod[i] = (p.hits[j] if p is not None else plain_hits[i]).cpu().numpy().view(np.uint32)
        kern = [None] * len(wl.batches)
        for g, p in zip(wl.groups, plans):
            for i in g:
                kern[i] = p.desc["kernel"] if p is not None else "plain"
        precision = precision_report(wl, {"product": (prod, kern),
                                          "plain": ([h.cpu().numpy().view(np.uint32) for h in plain_hits],
                                                    ["plain"] * len(wl.batches))}, n_prec,
                                     diff=[d[:100_000] for d in diff])
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup, ms_per_step=ms,
        higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
        config=workload_config(wl, args.config),
        workload_info=dict(triangles=wl.triangles, rays_per_step=n_step, l2="flushed before each step (256 MiB write)",
                           parallelism=f"replicas x{world}", prepare_s=t_prep, tune_s=t_tune, **wl.info,
                           plans=[p.desc if p is not None else {"kernel": "plain"} for p in plans]),
        plain=dict(value=plain_value, ms_per_step=ms_plain, launches_per_step=len(wl.batches)),
        speedup_vs_plain=value / plain_value,
        matched_hits_vs_plain=matched / max(1, n_all),
        latency_ms=dict(p50=float(np.percentile(step_ms, 50)), p99=float(np.percentile(step_ms, 99)),
                        plain_p50=float(np.percentile(plain_ms.sum(1), 50)),
                        plain_p99=float(np.percentile(plain_ms.sum(1), 99))),
        breakdown={("+".join(wl.batches[i].label for i in g) if len(g) <= 3 else f"{len(g)} batches"):
                   float(sum(len(wl.batches[i].rays) for i in g) / (prod_ms[:, k].mean() * 1e-3) / 1e6)
                   for k, g in enumerate(wl.groups)},
        tuning=tables, wall_s=wall, precision_vs_fp64=precision,
        roofline=roof, cpu_baseline=cpu, clocks=clk, e2e=e2e, gpu_launches=launches_per_step * args.steps)
    if notes:
        line["notes"] = sorted(set(notes))
    print(json.dumps(line), flush=True)
    for p in plans:
        if p is not None:
            p.close()
    scene.release()
    engine.close()


def run_blas_build(args):
    """One JSON line per mesh size (cluster soup of 0.25M, 1M and 4M triangles): the host SAH build
    (rt_blas_build) once and the GPU build (rt_blas_build_device) --steps times after --warmup
    (at most 10), each end to end from host arrays to a host BLAS, wall clock; the median GPU time;
    and whether the two builds' records are equal. Then the same for the instance top level
    (rt_tlas_build against rt_tlas_build_device) at 10k and 100k instances."""
    import time

    from renderlab_b200 import api as A
    from renderlab_b200 import scenes as S
    engine = A.Engine(0)
    steps = max(1, min(args.steps, 10))
    for n in ((250_000,) if args.small else (250_000, 1_000_000, 4_000_000)):
        m = S.clusters(n, config=2 if n < 4_000_000 else 3)
        t = time.perf_counter()
        host = A.Blas(m.positions, m.indices)
        host_ms = (time.perf_counter() - t) * 1e3
        for _ in range(args.warmup):
            A.Blas.build_device(engine, m.positions, m.indices)
        times = []
        for _ in range(steps):
            t = time.perf_counter()
            dev = A.Blas.build_device(engine, m.positions, m.indices)
            times.append((time.perf_counter() - t) * 1e3)
        gpu_ms = float(np.median(times))
        same = bool(np.array_equal(host.nodes(), dev.nodes()) and np.array_equal(host.bvh_indices(), dev.bvh_indices()))
        print(json.dumps({"metric": "BLAS build, host arrays to host BLAS (SAH)", "triangles": n,
                          "host_ms": round(host_ms, 1), "gpu_ms": round(gpu_ms, 1),
                          "gpu_ms_range": [round(min(times), 1), round(max(times), 1)],
                          "gpu_mtris_per_s": round(n / gpu_ms / 1e3, 1), "speedup": round(host_ms / gpu_ms, 1),
                          "same_records": same, "steps": steps, "warmup": args.warmup}), flush=True)
    # The instance top level: host tlas_build against rt_tlas_build_device on random placements
    # (centres uniform in [-500, 500]^3, half extents uniform in [0.5, 4]).
    rng = np.random.default_rng(1)
    for n in ((10_000,) if args.small else (10_000, 100_000)):
        c = rng.uniform(-500, 500, (n, 3)).astype(np.float32)
        h = rng.uniform(0.5, 4, (n, 3)).astype(np.float32)
        boxes = np.concatenate([c - h, c + h], 1).astype(np.float32)
        t = time.perf_counter()
        want = A.tlas_build(boxes, True)
        host_ms = (time.perf_counter() - t) * 1e3
        for _ in range(args.warmup):
            A.tlas_build_device(engine, boxes, True)
        times = []
        for _ in range(steps):
            t = time.perf_counter()
            got = A.tlas_build_device(engine, boxes, True)
            times.append((time.perf_counter() - t) * 1e3)
        gpu_ms = float(np.median(times))
        print(json.dumps({"metric": "top-level build, host boxes to host words (SAH)", "instances": n,
                          "host_ms": round(host_ms, 2), "gpu_ms": round(gpu_ms, 2),
                          "gpu_ms_range": [round(min(times), 2), round(max(times), 2)],
                          "speedup": round(host_ms / gpu_ms, 1), "same_words": bool(np.array_equal(want, got)),
                          "steps": steps, "warmup": args.warmup}), flush=True)
    engine.close()


def main():
    args = parse()
    if args.blas_build:
        run_blas_build(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == 5:
        run_serving(args)
    else:
        run_ours(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
