"""Ray sharding across GPUs, one process per GPU.

Rays are independent, so a batch shards with no exchange inside the traversal. Every rank holds
a replica of the scene (uploaded once per GPU) and the same batch description; rank r traces the
r-th contiguous slice of the batch -- in a Morton order of the ray origins when asked, so that
each GPU gets a spatially coherent part of the scene -- on its own device, and the slices' hits
are gathered through the process group: NCCL over NVLink between GPUs (tensors on the rank's
device), gloo on the host. Plain copies only: nothing here reads another GPU's memory with a
tensor-memory-accelerator load. The reference is single-device; this layer has no counterpart in
it.

    tracer = ShardedTrace(lambda rays, mode: engine.trace(scene, rays, mode, "wide8"))
    hits = tracer(rays, mode, hit_words(layout, mode))    # every rank gets all hits

`trace_fn(rays, mode)` traces one slice: rays a contiguous (k, 8) float32 tensor on the rank's
device (CPU with gloo), returning its (k, words) or (k,) int32 hits.
"""
from __future__ import annotations

import numpy as np


def slice_bounds(n: int, world: int, rank: int) -> tuple:
    """Rank `rank`'s contiguous slice [lo, hi) of n rays: the first n % world ranks take one more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _spread10(v: np.ndarray) -> np.ndarray:
    """The low 10 bits of v moved to every third bit (bit i to bit 3 i)."""
    v = v.astype(np.uint64) & np.uint64(0x3FF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x030000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x0300F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x030C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x09249249)
    return v


def morton_order(rays: np.ndarray) -> np.ndarray:
    """A stable permutation of the rays by the 30-bit Morton code of their origins, quantised to
    1024 steps a side over the origins' own bounding box."""
    o = np.asarray(rays, np.float32).reshape(-1, 8)[:, 0:3].astype(np.float64)
    if len(o) == 0:
        return np.zeros(0, np.int64)
    lo, hi = o.min(0), o.max(0)
    scale = np.where(hi > lo, 1023.0 / np.maximum(hi - lo, 1e-300), 0.0)
    q = np.clip(np.floor((o - lo) * scale), 0, 1023).astype(np.uint64)
    code = _spread10(q[:, 0]) | (_spread10(q[:, 1]) << np.uint64(1)) | (_spread10(q[:, 2]) << np.uint64(2))
    return np.argsort(code, kind="stable")


class ShardedTrace:
    """Splits a batch over the ranks of a process group and gathers the hits (see the module).

    order: None keeps the batch's order; "origin" slices it in the Morton order of the origins
    (results still come back in the batch's order). dst: None gathers to every rank; a rank
    index gathers to that rank alone (the others get None)."""

    def __init__(self, trace_fn, group=None, order: str | None = None):
        if order not in (None, "origin"):
            raise ValueError(f"unknown order {order!r}")
        self.trace_fn, self.group, self.order = trace_fn, group, order

    def __call__(self, rays, mode: int, hit_words: int, dst: int | None = None):
        import torch
        import torch.distributed as dist
        world = dist.get_world_size(self.group)
        rank = dist.get_rank(self.group)
        host = np.ascontiguousarray(rays.cpu().numpy() if hasattr(rays, "cpu") else rays, np.float32).reshape(-1, 8)
        n = len(host)
        perm = morton_order(host) if self.order == "origin" else None
        lo, hi = slice_bounds(n, world, rank)
        mine = host[perm[lo:hi]] if perm is not None else host[lo:hi]
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(self.group) == "nccl" \
            else torch.device("cpu")
        rays_dev = torch.from_numpy(np.ascontiguousarray(mine)).to(device)
        got = self.trace_fn(rays_dev, mode) if len(mine) else torch.zeros((0,), dtype=torch.int32, device=device)
        # every slice padded to the longest one, so the gather moves equal blocks
        m = (n + world - 1) // world
        shape = (m, hit_words) if hit_words > 1 else (m,)
        block = torch.zeros(shape, dtype=torch.int32, device=device)
        if hi > lo:
            block[: hi - lo] = got.reshape((hi - lo,) + shape[1:]).to(device=device, dtype=torch.int32)
        if dst is None:
            blocks = [torch.empty_like(block) for _ in range(world)]
            dist.all_gather(blocks, block, group=self.group)
        else:
            blocks = [torch.empty_like(block) for _ in range(world)] if rank == dst else None
            dist.gather(block, blocks, dst=dst, group=self.group)
            if rank != dst:
                return None
        parts = [b[: slice_bounds(n, world, r)[1] - slice_bounds(n, world, r)[0]] for r, b in enumerate(blocks)]
        out = torch.cat(parts) if parts else block[:0]
        if perm is not None:
            res = torch.empty_like(out)
            res[torch.from_numpy(perm).to(out.device)] = out
            out = res
        return out
