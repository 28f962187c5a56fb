"""Traversal benchmark: Mrays/s on the 1M-triangle cluster scene, one JSON line on stdout.

Workload (one step): 4,194,304 coherent primary rays (2048 x 2048 pinhole from (0, 0, -250),
fov 60 deg) plus 4,194,304 cosine-hemisphere GI rays spawned from the primary hits, closest hit,
over 1,000,000 triangles in 2,000 seeded clusters, packed in renderlab's reflection layout
(BVH4 with 8-bit child boxes, 48-byte pre-edged triangles). Inputs are synthetic and seeded
(splitmix64), the scene is device resident; L2 is flushed (a 256 MiB write) before each step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--kernel plain|fast|wide8]
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
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s closest+any-hit vs plain kernel at matched hits, 1 B200; p50/p99 latency"
UNIT = "Mrays/s"
WORKLOAD = ("clusters-1M: 1,000,000 triangles in 2,000 clusters (reflection layout); "
            "4,194,304 primary + 4,194,304 GI hemisphere rays per step, closest hit")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--kernel", default="auto")
    ap.add_argument("--triangles", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=2048)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target wall time of the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--refill", type=int, default=0, help="persistent-kernel refill threshold (lanes)")
    return ap.parse_args()


# ---------------------------------------------------------------- workload

def make_scene(n_tris):
    from renderlab_b200 import api as A
    from renderlab_b200 import scenes as S
    mesh = S.clusters(n_tris, config=2)
    words = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(mesh.positions, mesh.indices)], S.identity_instances(1))
    return mesh, words


def make_rays(engine, scene, mesh, width, kernel):
    """Primary rays, then one GI ray per primary ray, spawned from the primary hits in turn."""
    import torch
    from renderlab_b200 import api as A
    from renderlab_b200 import scenes as S
    primary = S.cluster_camera_rays(width, width)
    dev = torch.from_numpy(primary).cuda()
    h = engine.trace(scene, dev, A.CLOSEST, "plain")
    torch.cuda.synchronize()
    h = h.cpu().numpy().view(np.uint32)
    hit = h[:, 1] != 0
    t = h[hit, 0].view(np.float32)
    pts = S.hit_points(primary[hit], t)
    gi = S.hemisphere_rays(pts, S.triangle_normals(mesh, h[hit, 2]), primary[hit, 4:7], len(primary), S.Stream(0x5EED0002 + 1))
    return primary, gi, float(hit.mean())


def pick_kernel(name):
    if name != "auto":
        return name
    from renderlab_b200 import api as A
    return os.environ.get("RT_BENCH_KERNEL", "plain") if "plain" in A.KERNELS else "plain"


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
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][3]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[4]) for r in rows if r[4] not in ("", "[N/A]"))}


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


def bytes_per_ray(counters, n_rays, hit_bytes):
    """Algorithmic bytes a ray reads/writes (reflection layout): ray 32 + hit + 128 per top
    node + 96 per instance record + 64 per BLAS node + 48 per triangle tested."""
    c = counters
    total = (32 + hit_bytes) * n_rays + 128 * c["tlas_nodes"] + 96 * c["instance_box_tests"] \
        + 64 * c["blas_nodes"] + 48 * c["triangle_tests"]
    return total / n_rays


def cpu_baseline_leg(words, primary, gi, target_s, threads=None):
    """The reference traversal (the oracle's restatement of rs_trace) on the host cores over a
    strided sample of the step's rays; also returns its visit counters for the roofline."""
    from oracle import oracle as O
    threads = threads or (os.cpu_count() or 1)
    probe = np.concatenate([primary[::997][:4096], gi[::997][:4096]])
    t0 = time.perf_counter()
    O.rs_trace(words, probe, threads=threads)
    per_ray = (time.perf_counter() - t0) / len(probe)
    n_each = int(min(len(primary), max(4096, target_s / max(per_ray, 1e-9) / 2)))
    stride = max(1, len(primary) // n_each)
    sample = np.concatenate([primary[::stride][:n_each], gi[::stride][:n_each]])
    t0 = time.perf_counter()
    O.rs_trace(words, sample, threads=threads)
    wall = time.perf_counter() - t0
    _, cp = O.rs_trace(words, primary[::stride][:n_each], counters=True, threads=threads)
    _, cg = O.rs_trace(words, gi[::stride][:n_each], counters=True, threads=threads)
    return dict(value=len(sample) / wall / 1e6, unit=UNIT, cores=threads, kind="port",
                sample=f"{len(sample)} rays: every {stride}th primary and GI ray of the step, "
                       f"oracle rs_trace (scalar f32 C++) on {threads} threads, {wall:.2f} s"), (cp, cg, n_each)


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


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return  # rank 0 alone times the host-core reference
    from oracle import oracle as O
    from renderlab_b200 import scenes as S
    mesh, words = make_scene(args.triangles)
    primary = S.cluster_camera_rays(args.width, args.width)
    hits, _ = O.rs_trace(words, primary[::64])  # GI rays from a sample of primary hits
    hit = hits[:, 1] != 0
    pts = S.hit_points(primary[::64][hit], hits[hit, 0].view(np.float32))
    gi = S.hemisphere_rays(pts, S.triangle_normals(mesh, hits[hit, 2]), primary[::64][hit, 4:7], len(primary),
                           S.Stream(0x5EED0002 + 1))
    threads = os.cpu_count() or 1
    per_step = max(1.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    steps = []
    for k in range(args.warmup + args.steps):
        base, _ = cpu_baseline_leg(words, primary, gi, per_step, threads)
        if k >= args.warmup:
            steps.append(base)
    value = float(np.median([s["value"] for s in steps]))
    cpu = dict(steps[-1])
    cpu["value"] = value
    line = dict(metric=METRIC, value=value, unit=UNIT, impl="reference", n_gpus=world, steps=args.steps,
                warmup=args.warmup, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                data="synthetic", config=dict(workload=WORKLOAD, layout="reflection"), cpu_baseline=cpu,
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                ms_per_step=None, note="oracle restatement of rs_trace: the Rust/WGSL reference cannot run here")
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from renderlab_b200 import api as A
    kernel = pick_kernel(args.kernel)
    engine = A.Engine(local)
    if args.refill:
        engine.set_tuning(fast_refill=args.refill, wide8_refill=args.refill)
    mesh, words = make_scene(args.triangles)
    scene = engine.upload(A.LAYOUT_REFLECTION, words)
    t_prep = time.perf_counter()
    scene.prepare(kernel)  # derived layouts (the 8-wide BVH) are scene-upload work, untimed
    t_prep = time.perf_counter() - t_prep
    primary, gi, hit_rate = make_rays(engine, scene, mesh, args.width, kernel)
    d_primary = torch.from_numpy(primary).cuda()
    d_gi = torch.from_numpy(gi).cuda()
    n_step = len(primary) + len(gi)
    h_p = torch.empty((len(primary), 5), dtype=torch.int32, device="cuda")
    h_g = torch.empty((len(gi), 5), dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        engine.trace(scene, d_primary, A.CLOSEST, kernel, hits=h_p)
        engine.trace(scene, d_gi, A.CLOSEST, kernel, hits=h_g)

    for _ in range(max(3, args.warmup)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    # matched hits: the kernel under test against the plain kernel on this step's rays
    ref_p = engine.trace(scene, d_primary, A.CLOSEST, "plain").cpu().numpy()
    ref_g = engine.trace(scene, d_gi, A.CLOSEST, "plain").cpu().numpy()
    matched = float(((h_p.cpu().numpy()[:, 1:3] == ref_p[:, 1:3]).all(1).sum()
                     + (h_g.cpu().numpy()[:, 1:3] == ref_g[:, 1:3]).all(1).sum()) / n_step)

    bus = None
    try:
        bus = torch.cuda.get_device_properties(local).pci_bus_id
    except AttributeError:
        pass
    clocks = Clocks()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        engine.trace(scene, d_primary, A.CLOSEST, kernel, hits=h_p)
        ev[k][1].record(stream)
        engine.trace(scene, d_gi, A.CLOSEST, kernel, hits=h_g)
        ev[k][2].record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop(bus)
    prim_ms = np.array([a.elapsed_time(b) for a, b, _ in ev])
    gi_ms = np.array([b.elapsed_time(c) for _, b, c in ev])
    step_ms = prim_ms + gi_ms
    ms = float(step_ms.mean())
    if world > 1:
        ms = max_over_ranks(ms)
    value = world * n_step / (ms * 1e-3) / 1e6

    # e2e through the host-buffer C ABI call: pinned rays in, hits out, copies inside the timing
    hp = torch.from_numpy(primary).pin_memory()
    hg = torch.from_numpy(gi).pin_memory()
    op = torch.empty((len(primary), 5), dtype=torch.int32).pin_memory()
    og = torch.empty((len(gi), 5), dtype=torch.int32).pin_memory()
    engine.reserve(len(primary))
    for _ in range(2):
        engine.trace_host(scene, hp, A.CLOSEST, kernel, out=op)
    e2e_steps = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        engine.trace_host(scene, hp, A.CLOSEST, kernel, out=op)
        engine.trace_host(scene, hg, A.CLOSEST, kernel, out=og)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        e2e_s = max_over_ranks(e2e_s)
    e2e = dict(value=world * n_step / e2e_s / 1e6, unit=UNIT, h2d_bytes_per_step=n_step * 32,
               d2h_bytes_per_step=n_step * 20, ms_per_step=e2e_s * 1e3)

    if rank != 0:
        return
    cpu, counts = (None, None)
    if not args.no_cpu:
        cpu, counts = cpu_baseline_leg(words, primary, gi, args.cpu_seconds)
    peak, peak_kind = measured_peak()
    roof = None
    if counts:
        cp, cg, n_each = counts
        bp, bg = bytes_per_ray(cp, n_each, 20), bytes_per_ray(cg, n_each, 20)
        alg_bytes = bp * len(primary) + bg * len(gi)
        achieved = alg_bytes / (ms * 1e-3) / 1e9
        roof = dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                    traffic=None, peak_source=f"{peak_kind} hbm_gbs",
                    bytes_per_ray=dict(primary=bp, gi=bg), roofline_mrays=peak * 1e9 / ((alg_bytes / n_step)) / 1e6,
                    note="scene (51 MB) is L2-resident: algorithmic bytes over the HBM peak may exceed 1")
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup, ms_per_step=ms,
        higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
        config=dict(workload=WORKLOAD, kernel=kernel, layout="reflection", triangles=args.triangles,
                    rays_per_step=n_step, primary_hit_rate=hit_rate, prepare_s=t_prep, l2="flushed before each step (256 MiB write)",
                    parallelism=f"replicas x{world}"),
        latency_ms=dict(p50=float(np.percentile(step_ms, 50)), p99=float(np.percentile(step_ms, 99))),
        breakdown=dict(primary_mrays=float(len(primary) / (prim_ms.mean() * 1e-3) / 1e6),
                       gi_mrays=float(len(gi) / (gi_ms.mean() * 1e-3) / 1e6)),
        matched_hits_vs_plain=matched, wall_s=wall,
        roofline=roof, cpu_baseline=cpu, clocks=clk, e2e=e2e, gpu_launches=2 * args.steps)
    print(json.dumps(line), flush=True)
    scene.release()
    engine.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
