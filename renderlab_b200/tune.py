"""The autotuner: picks, per scene and per batch set, the launch parameters of the persistent
traversal by timing candidate plans on the device.

Parameters searched (each candidate is one rt_plan, timed as a whole, sort included):

* kernel -- PLAIN (one thread per ray, a launch per batch), FAST (persistent warps over the
  BVH4-Q8, bit-exact with the reference loop like PLAIN) or WIDE8 (8-wide compressed nodes,
  watertight f32 test with f64 re-tests) or WIDE8 walked by warp-wide packets of 32 rays ("wide8p":
  the same results, the top level walked by the packet too);
* wavefront width -- the refill threshold: how many lanes of a 32-wide warp must be idle before
  the warp takes more rays (1 keeps every lane busy; 32 hands out whole runs of 32 consecutive
  rays, which keeps a coherent batch's 8 x 4 tiles together);
* sort key -- none, or a ray permutation by origin Morton code / octant + origin / octahedral
  direction cell + coarse origin (rt_order_rays over the plan's whole ray space, run inside the
  plan on every launch). The direction key gathers rays toward one light from nearby points,
  which lets the packet walk share their traversal.

* stack -- for WIDE8's per-ray walk, where each lane keeps its node-group stack: 32 entries in
  local memory (cached by L1), or 16 in a shared-memory column of the block (only when the
  scene's 8-wide trees are at most 16 levels deep; the walk stacks at most one group a level).

The bit-exact kernels' stack is not a free parameter: PLAIN and FAST keep the reference's
48-entry stack (gi_rays_software.wgsl:22, reflections_software_bvh4.wgsl:12), whose overflow
behaviour is part of their results.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import api as A

KERNELS = ("plain", "fast", "wide8", "wide8p")
REFILLS = (4, 8, 16, 32)
ORDERS = ("none", "origin", "octant", "direction")
STACKS = ("local", "shared")


@dataclass
class Trial:
    kernel: str
    refill: int
    order: str
    ms: float
    mrays: float
    stack: str = ""


@dataclass
class Choice:
    plan: A.Plan
    trials: list = field(default_factory=list)

    @property
    def best(self) -> Trial:
        return min(self.trials, key=lambda t: t.ms)

    def table(self) -> list:
        return [dict(kernel=t.kernel, refill=t.refill, order=t.order, stack=t.stack, ms=round(t.ms, 4),
                     mrays=round(t.mrays, 1)) for t in sorted(self.trials, key=lambda t: t.ms)]


def time_plan(plan: A.Plan, reps: int = 3, warmup: int = 1, flush=None) -> float:
    """Median device time (ms) of `reps` launches after `warmup` untimed ones; `flush` (a CUDA
    byte tensor larger than L2) is rewritten before every timed launch when given."""
    import torch
    for _ in range(warmup):
        plan.launch()
    times = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plan.launch()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return float(np.median(times))


def candidates(kernels=KERNELS, refills=REFILLS, orders=ORDERS, stacks=STACKS) -> list:
    """Every (kernel, refill, order, stack), the usual winners first: unsorted before sorted, the
    middle and widest wavefronts before the rest, the local stack before the shared one. Only
    WIDE8's per-ray walk has a stack choice ("" elsewhere); its shared stack is tried unsorted."""
    pri = {8: 0, 32: 1, 16: 2, 4: 3}
    grid = [(k, r, o, stacks[0] if k == "wide8" else "") for k in kernels for r in refills for o in orders
            if k not in ("plain", "wide8p")]
    if "wide8" in kernels:
        grid += [("wide8", r, orders[0], s) for r in refills for s in stacks[1:]]
    if "plain" in kernels:  # no ray queue and no sort: one candidate
        grid.append(("plain", 0, orders[0], ""))
    if "wide8p" in kernels:  # warps take whole packets of 32 rays: no wavefront width
        grid += [("wide8p", 32, o, "") for o in orders]
    return sorted(grid, key=lambda c: (orders.index(c[2]) > 0, c[3] not in ("", stacks[0]), pri.get(c[1], 4),
                                       kernels.index(c[0])))


def tune(engine: A.Engine, scene: A.Scene, batches, kernels=KERNELS, refills=REFILLS, orders=ORDERS,
         graph: bool = True, reps: int = 3, flush=None, max_seconds: float = 30.0, stacks=STACKS) -> Choice:
    """Times (kernel, refill, order, stack) plans over `batches` ((rays, mode[, hits]) on the device),
    in candidates() order until all are timed or `max_seconds` of device time is spent, and
    returns the fastest plan, built and ready to launch, with the trial table. WIDE8 candidates
    are skipped unless the scene has been prepared for WIDE8, and the shared stack unless its trees
    fit it."""
    import torch
    rays = sum(int(b[0].shape[0]) for b in batches)
    with_hits = []  # one set of hit buffers, shared by every candidate plan
    for b in batches:
        r, mode = b[0], b[1]
        h = b[2] if len(b) > 2 and b[2] is not None else None
        if h is None:
            words = A.hit_words(scene.layout, mode)
            n = int(r.shape[0])
            h = torch.empty((n, words) if words > 1 else (n,), dtype=torch.int32, device=r.device)
        with_hits.append((r, mode, h))
    best_plan, best_ms, trials, spent, skip = None, None, [], 0.0, set()
    for kernel, refill, order, stack in candidates(kernels, refills, orders, stacks):
        if kernel in skip or (kernel, stack) in skip:
            continue
        if trials and spent > max_seconds:
            break
        try:
            plan = engine.plan(scene, with_hits, kernel, refill=refill, order=order, graph=graph, stack=stack)
        except A.RtError as e:
            if "UNSUPPORTED" in str(e):
                skip.add((kernel, stack) if stack not in ("", stacks[0]) else kernel)
                continue
            raise
        ms = time_plan(plan, reps=reps, flush=flush)
        spent += ms * (reps + 1) * 1e-3
        trials.append(Trial(kernel, refill, order, ms, rays / (ms * 1e-3) / 1e6 if ms > 0 else 0.0, stack))
        if best_ms is None or ms < best_ms:
            if best_plan is not None:
                best_plan.close()
            best_plan, best_ms = plan, ms
        else:
            plan.close()
    return Choice(best_plan, trials)
