"""CPU ORACLE — test infrastructure only.

ctypes binding of ``oracle/_build/liboracle.so``, the scalar C++ restatement of renderlab's
software-ray path (builders, packers, the two WGSL traversal loops, the f64 reference trace).
Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this module,
and only to check or time the reference algorithm; the product never routes through it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

COUNTERS = ("tlas_nodes", "tlas_box_tests", "tlas_instance_entries", "instance_box_tests",
            "instance_box_entries", "blas_visits", "blas_nodes", "blas_box_tests",
            "triangle_tests", "leaves", "stack_drops")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_bvh_build.restype = ctypes.c_void_p
        L.orc_bvh_build.argtypes = [_f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_int,
                                    ctypes.c_char_p, ctypes.c_int]
        for name in ("orc_bvh_free", "orc_words_free"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.orc_bvh_info.argtypes = [ctypes.c_void_p, _u32p]
        L.orc_bvh_nodes.argtypes = [ctypes.c_void_p, _u32p]
        L.orc_bvh_leaves.argtypes = [ctypes.c_void_p, _u32p]
        L.orc_bvh_indices.argtypes = [ctypes.c_void_p, _u32p]
        L.orc_bvh_refit.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_int]
        L.orc_bvh_validate.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_bvh_trace64.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_uint32, ctypes.c_int, _f64p]
        L.orc_quantized_node.argtypes = [_u32p, _f32p, ctypes.c_uint32, _u32p]
        L.orc_tlas_reserve.restype = ctypes.c_uint32
        L.orc_tlas_reserve.argtypes = [ctypes.c_uint32]
        L.orc_tlas_build.restype = ctypes.c_uint32
        L.orc_tlas_build.argtypes = [_f32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_uint32]
        L.orc_tlas_refit.argtypes = [_u32p, ctypes.c_uint32, _f32p, ctypes.c_uint32, ctypes.c_int]
        L.orc_tlas_place.restype = ctypes.c_uint32
        L.orc_tlas_place.argtypes = [_u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     _u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_uint32]
        L.orc_scene.restype = ctypes.c_void_p
        L.orc_scene.argtypes = [ctypes.c_int, ctypes.c_uint32, _f32p, _u32p, _u32p, _u32p, _u32p,
                                ctypes.c_uint32, _f32p, _f32p, _u32p, _u32p, ctypes.c_int,
                                ctypes.c_char_p, ctypes.c_int]
        L.orc_words_len.restype = ctypes.c_uint64
        L.orc_words_len.argtypes = [ctypes.c_void_p]
        L.orc_words_copy.argtypes = [ctypes.c_void_p, _u32p]
        L.orc_gi_trace.argtypes = [_u32p, _f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, _u32p,
                                   _u64p, ctypes.c_int]
        L.orc_rs_trace.argtypes = [_u32p, _f32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, _u32p,
                                   _u64p, ctypes.c_int]
        L.orc_rs_trace_counts.argtypes = [_u32p, _f32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                          _u32p, _u64p]
        L.orc_gi_cell_rays.argtypes = [_u32p, ctypes.c_uint32, ctypes.c_int, _f32p]
        L.orc_gi_cell_rays.restype = None
        L.orc_gi_light_rays.argtypes = [_u32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _f32p,
                                        ctypes.POINTER(ctypes.c_uint8)]
        L.orc_gi_light_rays.restype = None
        L.orc_fp64_trace.argtypes = [_u32p, ctypes.c_int, _f32p, ctypes.c_uint32, ctypes.c_int, _f64p,
                                     _u32p, ctypes.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Bvh:
    """A BVH4-Q8 built by the restated ``near_field::build`` (median / SAH)."""

    def __init__(self, positions, indices, mode: int = 1):
        pos = _c(positions, np.float32).reshape(-1, 3)
        idx = _c(indices, np.uint32).reshape(-1)
        err = ctypes.create_string_buffer(256)
        self._pos = pos
        self.h = lib().orc_bvh_build(_p(pos, _f32p), len(pos), _p(idx, _u32p), len(idx), mode, err, 256)
        if not self.h:
            raise ValueError(err.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bvh_free(self.h)
            self.h = None

    def info(self) -> dict:
        out = np.zeros(6, np.uint32)
        lib().orc_bvh_info(self.h, _p(out, _u32p))
        return dict(zip(("nodes", "leaves", "positions", "indices", "root", "depth"), map(int, out)))

    def nodes(self) -> np.ndarray:
        out = np.zeros((self.info()["nodes"], 16), np.uint32)
        lib().orc_bvh_nodes(self.h, _p(out, _u32p))
        return out

    def leaves(self) -> np.ndarray:
        out = np.zeros((self.info()["leaves"], 3), np.uint32)
        lib().orc_bvh_leaves(self.h, _p(out, _u32p))
        return out

    def indices(self) -> np.ndarray:
        out = np.zeros(self.info()["indices"], np.uint32)
        lib().orc_bvh_indices(self.h, _p(out, _u32p))
        return out

    def refit(self, positions) -> None:
        pos = _c(positions, np.float32).reshape(-1, 3)
        err = ctypes.create_string_buffer(256)
        if not lib().orc_bvh_refit(self.h, _p(pos, _f32p), len(pos), err, 256):
            raise ValueError(err.value.decode())

    def validate(self) -> None:
        err = ctypes.create_string_buffer(256)
        if not lib().orc_bvh_validate(self.h, err, 256):
            raise ValueError(err.value.decode())

    def trace64(self, rays64, brute=False) -> np.ndarray:
        r = _c(rays64, np.float64).reshape(-1, 8)
        out = np.zeros((len(r), 6), np.float64)
        lib().orc_bvh_trace64(self.h, _p(r, _f64p), len(r), int(brute), _p(out, _f64p))
        return out


def quantized_node(children, boxes) -> np.ndarray:
    ch = _c(children, np.uint32)
    bx = _c(boxes, np.float32).reshape(-1, 6)
    out = np.zeros(16, np.uint32)
    lib().orc_quantized_node(_p(ch, _u32p), _p(bx, _f32p), len(ch), _p(out, _u32p))
    return out


def tlas_reserve(n: int) -> int:
    return int(lib().orc_tlas_reserve(n))


def tlas_build(boxes, sah=True, wide=True) -> np.ndarray:
    b = _c(boxes, np.float32).reshape(-1, 6)
    cap = max(64, len(b) * 32)
    out = np.zeros(cap, np.uint32)
    n = lib().orc_tlas_build(_p(b, _f32p), len(b), int(sah), int(wide), _p(out, _u32p), cap)
    return out[:n].copy()


def tlas_refit(nodes, boxes, wide=True) -> np.ndarray:
    nodes = _c(nodes, np.uint32).copy()
    b = _c(boxes, np.float32).reshape(-1, 6)
    lib().orc_tlas_refit(_p(nodes, _u32p), len(nodes), _p(b, _f32p), len(b), int(wide))
    return nodes


def tlas_place(words, header, stride, slots, previous=None, mode=-1, wide=True) -> np.ndarray:
    w = _c(words, np.uint32)
    p = _c(previous if previous is not None else np.zeros(0), np.uint32)
    cap = len(w) + tlas_reserve(slots) + 64
    out = np.zeros(cap, np.uint32)
    n = lib().orc_tlas_place(_p(w, _u32p), len(w), header, stride, slots, _p(p, _u32p), len(p), mode,
                             int(wide), _p(out, _u32p), cap)
    return out[:n].copy()


KIND_GI, KIND_RS, KIND_RS_BVH2 = 0, 1, 2


def scene_words(kind, meshes, instances, tlas_mode=-1) -> np.ndarray:
    """Pack a scene with the restated builders/packers.

    meshes: list of (positions (V,3) f32, indices (3T,) u32[, flags]).
    instances: dict of arrays: model (N,3,4), rows (N,3,4), mesh (N,), aux (N,9) GI / (N,2) refl.
    """
    pos = np.concatenate([_c(m[0], np.float32).reshape(-1, 3) for m in meshes]) if meshes else np.zeros((0, 3), np.float32)
    idx = np.concatenate([_c(m[1], np.uint32).reshape(-1) for m in meshes]) if meshes else np.zeros(0, np.uint32)
    pos_off = np.zeros(len(meshes) + 1, np.uint32)
    idx_off = np.zeros(len(meshes) + 1, np.uint32)
    for i, m in enumerate(meshes):
        pos_off[i + 1] = pos_off[i] + len(np.asarray(m[0]).reshape(-1, 3))
        idx_off[i + 1] = idx_off[i] + len(np.asarray(m[1]).reshape(-1))
    flags = np.array([m[2] if len(m) > 2 else 0 for m in meshes], np.uint32)
    models = _c(instances["model"], np.float32).reshape(-1, 12)
    rows = _c(instances["rows"], np.float32).reshape(-1, 12)
    mesh = _c(instances["mesh"], np.uint32)
    aux = _c(instances["aux"], np.uint32)
    err = ctypes.create_string_buffer(256)
    h = lib().orc_scene(kind, len(meshes), _p(pos, _f32p), _p(pos_off, _u32p), _p(idx, _u32p),
                        _p(idx_off, _u32p), _p(flags, _u32p), len(mesh), _p(models, _f32p),
                        _p(rows, _f32p), _p(mesh, _u32p), _p(aux, _u32p), tlas_mode, err, 256)
    if not h:
        raise ValueError(err.value.decode())
    try:
        out = np.zeros(lib().orc_words_len(h), np.uint32)
        lib().orc_words_copy(h, _p(out, _u32p))
    finally:
        lib().orc_words_free(h)
    return out


def default_threads() -> int:
    return os.cpu_count() or 1


def gi_trace(words, rays, mode=0, top_wide=True, counters=False, threads=None):
    """gi_traverse over every ray: (hits (n,10) u32 words, counter sums or None)."""
    w = _c(words, np.uint32)
    r = _c(rays, np.float32).reshape(-1, 8)
    hits = np.zeros((len(r), 10), np.uint32)
    cnt = np.zeros(len(COUNTERS), np.uint64) if counters else None
    lib().orc_gi_trace(_p(w, _u32p), _p(r, _f32p), len(r), mode, int(top_wide), _p(hits, _u32p),
                       _p(cnt, _u64p), threads or default_threads())
    return hits, (dict(zip(COUNTERS, map(int, cnt))) if counters else None)


def rs_trace(words, rays, any_hit=False, bvh2=False, counters=False, threads=None):
    """rs_trace over every ray: (hits (n,5) u32 words [t bits, record], counter sums or None)."""
    w = _c(words, np.uint32)
    r = _c(rays, np.float32).reshape(-1, 8)
    hits = np.zeros((len(r), 5), np.uint32)
    cnt = np.zeros(len(COUNTERS), np.uint64) if counters else None
    lib().orc_rs_trace(_p(w, _u32p), _p(r, _f32p), len(r), int(any_hit), int(bvh2), _p(hits, _u32p),
                       _p(cnt, _u64p), threads or default_threads())
    return hits, (dict(zip(COUNTERS, map(int, cnt))) if counters else None)


def rs_trace_counts(words, rays, any_hit=False, bvh2=False):
    """rs_trace with per-ray counters: (hits (n,5), counters (n, len(COUNTERS)))."""
    w = _c(words, np.uint32)
    r = _c(rays, np.float32).reshape(-1, 8)
    hits = np.zeros((len(r), 5), np.uint32)
    cnt = np.zeros((len(r), len(COUNTERS)), np.uint64)
    lib().orc_rs_trace_counts(_p(w, _u32p), _p(r, _f32p), len(r), int(any_hit), int(bvh2),
                              _p(hits, _u32p), _p(cnt, _u64p))
    return hits, cnt


def gi_cell_rays(cells, rotate=False):
    """The GI cache cells' fixed-direction rays (gi_cache.wgsl gi_direction / gi_origin_offset):
    cells (n, 8) uint32 records (q xyz, edge, packed normal, key_b, 0, 0); (n * 64, 8) float32."""
    c = _c(cells, np.uint32).reshape(-1, 8)
    out = np.zeros((len(c) * 64, 8), np.float32)
    lib().orc_gi_cell_rays(_p(c, _u32p), len(c), int(bool(rotate)), _p(out, _f32p))
    return out


def gi_light_rays(cells, lights):
    """The GI cache's per-light visibility rays (gi_cache.wgsl gi_light / gi_light_direction /
    gi_light_affects): cells (n, 8) uint32 records as gi_cell_rays takes them, lights (m, 20) uint32
    80-byte light records. Returns (rays (n * m, 8) float32, affects (n, m) bool)."""
    c = _c(cells, np.uint32).reshape(-1, 8)
    lt = _c(lights, np.uint32).reshape(-1, 20)
    rays = np.zeros((len(c) * len(lt), 8), np.float32)
    affects = np.zeros((len(c), len(lt)), np.uint8)
    lib().orc_gi_light_rays(_p(c, _u32p), len(c), _p(lt, _u32p), len(lt), _p(rays, _f32p),
                            affects.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return rays, affects.astype(bool)


def gi_light_bits(words, cells, lights, threads=None):
    """gi_light's visibility words (gi_cache.wgsl:2054-2077) over a packed GI scene: per cell,
    ceil(m / 32) uint32 words, bit l % 32 of word l // 32 set when light l reaches the cell and
    gi_visible_within finds nothing in the way."""
    rays, affects = gi_light_rays(cells, lights)
    n, m = affects.shape
    hits, _ = gi_trace(words, rays, 2, threads=threads)
    visible = affects & (hits[:, 1] == 0xFFFFFFFF).reshape(n, m)
    words_out = np.zeros((n, (m + 31) // 32), np.uint32)
    for l in range(m):
        words_out[:, l // 32] |= visible[:, l].astype(np.uint32) << np.uint32(l % 32)
    return words_out


def fp64_trace(words, rays, layout, any_hit=False, threads=None):
    """FP64 reference over a packed scene: (out (n,4) f64 [hit,t,u,v], ident (n,6) u32)."""
    w = _c(words, np.uint32)
    r = _c(rays, np.float32).reshape(-1, 8)
    out = np.zeros((len(r), 4), np.float64)
    ident = np.zeros((len(r), 6), np.uint32)
    lib().orc_fp64_trace(_p(w, _u32p), layout, _p(r, _f32p), len(r), int(any_hit), _p(out, _f64p),
                         _p(ident, _u32p), threads or default_threads())
    return out, ident
