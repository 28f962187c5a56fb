"""Cooked scene files loaded straight into the engine.

RLB is renderlab's cooked cluster BVH (crates/asset/src/cluster_bvh/codec.rs): BVH4-Q8 nodes
with per-child errors, leaves with their cluster identity, LOD levels and their cuts, positions
and the reordered triangle list. RNF is a cooked near field (crates/asset/src/near_field.rs:
540-660): settings, the source digest, one single-level RLB per mesh (the far-field cut) and
placements, each a column-major transform with per-vertex octahedral masks.

Both codecs and their checks run in the native library (rt_rlb_decode, rt_rnf_decode, ...);
this module is the Python face of that C ABI:

    field = NearField.decode(open("scene.rnf", "rb").read())
    words = field.pack_gi(field.instances())       # masks appended, word 23 set per placement
    scene = engine.upload(LAYOUT_GI, words)

A mask-free field can instead be traced as one merged world BLAS (``field.world()``), as
src/gi_cache.rs:1234-1268 does.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field as dc_field

import numpy as np

from . import api as A
from .scenes import Instances, affine_inverse_rows

RLB_MAX_BYTES = 150_000_000  # cluster_bvh::Limits::default
RNF_MAX_BYTES = 160_000_000  # near_field::Limits::default


class CookedError(ValueError):
    """A cooked file the reference's checks reject; the message is the reference's."""


def _err():
    return ctypes.create_string_buffer(256)


def _raise(st: int, err) -> None:
    if st == 2:
        raise CookedError(err.value.decode())
    if st != 0:
        raise A.RtError(st, "invalid argument")


def _bytes_arg(data):
    buf = np.frombuffer(bytes(data), np.uint8)
    return buf, (buf.ctypes.data if len(buf) else None)


def encode_rlb(blas: A.Blas, max_bytes: int = RLB_MAX_BYTES) -> bytes:
    """The BLAS as an RLB file: one zero-error level over every leaf (near_field.rs:206-262)."""
    L, err, n = A.lib(), _err(), ctypes.c_size_t(0)
    _raise(L.rt_blas_encode_rlb(blas.h, max_bytes, None, ctypes.byref(n), err, len(err)), err)
    out = ctypes.create_string_buffer(n.value)
    _raise(L.rt_blas_encode_rlb(blas.h, max_bytes, out, ctypes.byref(n), err, len(err)), err)
    return out.raw[: n.value]


def decode_rlb(data, level: int = 0, max_bytes: int = RLB_MAX_BYTES) -> A.Blas:
    """Level ``level`` of an RLB file as a BLAS the packers take (gi_bvh.rs:62-78)."""
    buf, ptr = _bytes_arg(data)
    h, err = A._vp(), _err()
    _raise(A.lib().rt_rlb_decode(ptr, len(buf), max_bytes, level, ctypes.byref(h), err, len(err)), err)
    return A.Blas.adopt(h)


@dataclass
class Placement:
    mesh: int
    transform: np.ndarray  # (4, 4) float32, columns first: transform[c] is column c
    masks: np.ndarray      # uint32, positions * 2 * bins^2 / 32

    def model(self) -> np.ndarray:
        """The object-to-world model as the packers take it: 3 rows of 4."""
        return np.ascontiguousarray(self.transform.T[:3], np.float32)


@dataclass
class NearField:
    lod_error: float
    reach: float
    skip: float
    bins: int
    source: bytes
    meshes: list = dc_field(default_factory=list)       # A.Blas per field mesh (its far-field cut)
    placements: list = dc_field(default_factory=list)   # Placement

    @staticmethod
    def decode(data, max_bytes: int = RNF_MAX_BYTES) -> "NearField":
        buf, ptr = _bytes_arg(data)
        L, h, err = A.lib(), A._vp(), _err()
        _raise(L.rt_rnf_decode(ptr, len(buf), max_bytes, ctypes.byref(h), err, len(err)), err)
        try:
            s, src = A.RtRnfSettings(), ctypes.create_string_buffer(32)
            nm, npl = ctypes.c_uint32(), ctypes.c_uint32()
            L.rt_rnf_info(h, ctypes.byref(s), src, ctypes.byref(nm), ctypes.byref(npl))
            f = NearField(s.lod_error, s.reach, s.skip, s.bins, src.raw[:32])
            for m in range(nm.value):
                b = A._vp()
                L.rt_rnf_mesh(h, m, ctypes.byref(b))
                f.meshes.append(A.Blas.adopt(b))
            for k in range(npl.value):
                p = A.RtRnfPlacement()
                L.rt_rnf_placement_get(h, k, ctypes.byref(p))
                masks = np.ctypeslib.as_array(p.masks, (p.n_masks,)).copy() if p.n_masks else np.zeros(0, np.uint32)
                t = np.array(p.transform[:], np.float32).reshape(4, 4)
                f.placements.append(Placement(p.mesh, t, masks))
            return f
        finally:
            L.rt_rnf_free(h)

    def _native(self):
        """A library-side field (encoded and decoded again: one source of truth for its checks)."""
        buf, ptr = _bytes_arg(self.encode())
        h, err = A._vp(), _err()
        _raise(A.lib().rt_rnf_decode(ptr, len(buf), RNF_MAX_BYTES + len(buf), ctypes.byref(h), err, len(err)), err)
        return h

    def encode(self, max_bytes: int = RNF_MAX_BYTES) -> bytes:
        L, err, n = A.lib(), _err(), ctypes.c_size_t(0)
        s = A.RtRnfSettings(self.lod_error, self.reach, self.skip, self.bins)
        src = ctypes.create_string_buffer(bytes(self.source).ljust(32, b"\0")[:32], 32)
        m = len(self.meshes)
        handles = (A._vp * max(m, 1))(*[b.h for b in self.meshes])
        arr = (A.RtRnfPlacement * max(len(self.placements), 1))()
        keep = []
        for k, p in enumerate(self.placements):
            masks = np.ascontiguousarray(p.masks, np.uint32)
            keep.append(masks)
            arr[k].mesh = int(p.mesh)
            ctypes.memmove(arr[k].transform, np.ascontiguousarray(p.transform, np.float32).ctypes.data, 64)
            arr[k].masks = masks.ctypes.data_as(A._u32p) if len(masks) else None
            arr[k].n_masks = len(masks)
        args = (ctypes.byref(s), src, handles, m, arr, len(self.placements), max_bytes)
        _raise(L.rt_rnf_encode(*args, None, ctypes.byref(n), err, len(err)), err)
        out = ctypes.create_string_buffer(max(n.value, 1))
        _raise(L.rt_rnf_encode(*args, out, ctypes.byref(n), err, len(err)), err)
        return out.raw[: n.value]

    def instances(self, extra=None) -> Instances:
        """One instance per placement, its model the placement's transform (so its masks apply)
        and its world-to-object rows the float64 inverse rounded once."""
        model = np.stack([p.model() for p in self.placements]) if self.placements else np.zeros((0, 3, 4), np.float32)
        inst = Instances(model, affine_inverse_rows(model), np.array([p.mesh for p in self.placements], np.uint32))
        if extra is not None:
            inst.extra = extra
        return inst

    def pack_gi(self, instances: Instances | None = None, tlas_mode: int = -1) -> np.ndarray:
        """GI words: the field's meshes, their placements' masks, and ``instances`` (mesh = field
        mesh index); an instance with a placement's exact transform bits reads its masks."""
        instances = self.instances() if instances is None else instances
        arr, n = A._instance_array(A.LAYOUT_GI, instances)
        L, h, size = A.lib(), self._native(), ctypes.c_size_t(0)
        try:
            st = L.rt_rnf_pack_gi(h, arr, n, tlas_mode, None, ctypes.byref(size))
            if st != 0:
                raise A.RtError(st, "near-field packing failed (singular transform or bad mesh index)")
            out = np.zeros(size.value, np.uint32)
            st = L.rt_rnf_pack_gi(h, arr, n, tlas_mode, out.ctypes.data_as(A._u32p), ctypes.byref(size))
            if st != 0:
                raise A.RtError(st, "near-field packing failed")
            return out
        finally:
            L.rt_rnf_free(h)

    def world(self):
        """(BLAS, bases): every placement's cut in world space as one SAH BLAS, and each
        placement's first position in it (gi_cache.rs:1234-1268)."""
        L, h, b = A.lib(), self._native(), A._vp()
        try:
            bases = np.zeros(max(len(self.placements), 1), np.uint32)
            st = L.rt_rnf_world(h, ctypes.byref(b), bases.ctypes.data_as(A._u32p))
            if st != 0:
                raise A.RtError(st, "near-field world needs a nonempty triangle list")
            return A.Blas.adopt(b), bases[: len(self.placements)]
        finally:
            L.rt_rnf_free(h)
