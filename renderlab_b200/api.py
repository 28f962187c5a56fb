"""Python host side of the engine, over the C ABI in ``include/rt_trace.h``.

Mirrors renderlab's ray-query seam (shaders/gi_rays_software.wgsl:280-291 and
shaders/reflections_software_bvh4.wgsl:206-207) for batches of rays:

* ``gi_closest(scene, rays)``          -> GI hits (t, instance, triangle, barycentrics, normal)
* ``gi_visible(scene, o, d)``          -> True where nothing blocks (tmin 0, tmax 1e20)
* ``gi_visible_within(scene, o, d, tmax)``
* ``rs_trace(scene, rays, any_hit)``   -> reflection records (slot + 1, primitive, u, v) and t
* ``rs_closest`` / ``rs_blocked``

Device buffers are torch CUDA tensors (PyTorch is only the allocator and stream source here);
``Engine.trace_host`` takes host arrays and copies through the library's pipelined staging.
Every traversal runs in ``_lib/librt_trace.so``; there is no CPU fallback, and importing this
module on a machine without the library raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "librt_trace.so"

LAYOUT_GI, LAYOUT_REFLECTION, LAYOUT_REFLECTION_BVH2 = 0, 1, 2
CLOSEST, ANY_SKY, ANY_CASTERS = 0, 1, 2
KERNELS = {"plain": 0, "fast": 1, "wide8": 2, "wide8p": 3}
ORDERS = {"none": 0, "origin": 1, "octant": 2, "direction": 3}
STACKS = {"": 0, "local": 1, "shared": 2}  # RT_STACK_LOCAL / RT_STACK_SHARED
STATUS = {0: "OK", 1: "INVALID_ARG", 2: "LAYOUT", 3: "OOM", 4: "STACK_OVERFLOW", 5: "TIMEOUT",
          6: "CUDA", 7: "BUSY", 8: "UNSUPPORTED"}
GI_HIT_WORDS, RS_HIT_WORDS = 10, 5
GI_DIRECTIONS, GI_ROTATE = 64, 4
MISS = 0xFFFFFFFF

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f32p = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class RtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class RtStats(ctypes.Structure):
    _fields_ = [("rays_traced", ctypes.c_uint64), ("stack_overflows", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("scene_bytes", ctypes.c_uint64)]


class RtInstance(ctypes.Structure):
    _fields_ = [("model", ctypes.c_float * 12), ("rows", ctypes.c_float * 12), ("mesh", ctypes.c_uint32),
                ("slot", ctypes.c_uint32), ("casts_shadow", ctypes.c_uint32), ("near_base", ctypes.c_uint32),
                ("extra", ctypes.c_uint32 * 8)]


class RtBatch(ctypes.Structure):
    _fields_ = [("d_rays", ctypes.c_void_p), ("d_hits", ctypes.c_void_p), ("n", ctypes.c_uint32), ("mode", ctypes.c_int)]


class RtHostBatch(ctypes.Structure):
    _fields_ = [("h_rays", ctypes.c_void_p), ("h_hits", ctypes.c_void_p), ("n", ctypes.c_uint32),
                ("mode", ctypes.c_int), ("kernel", ctypes.c_int)]


class RtPlanDesc(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("refill", ctypes.c_uint32), ("order", ctypes.c_int), ("graph", ctypes.c_uint32),
                ("stack", ctypes.c_uint32)]


class RtServerDesc(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_uint64), ("launch_rays", ctypes.c_uint32), ("slots", ctypes.c_uint32),
                ("kernel", ctypes.c_int)]


class RtServerStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_uint64), ("rays", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("wall_s", ctypes.c_double), ("device_bytes", ctypes.c_uint64), ("pending", ctypes.c_uint64)]


class RtRnfSettings(ctypes.Structure):
    _fields_ = [("lod_error", ctypes.c_float), ("reach", ctypes.c_float), ("skip", ctypes.c_float),
                ("bins", ctypes.c_uint32)]


class RtRnfPlacement(ctypes.Structure):
    _fields_ = [("mesh", ctypes.c_uint32), ("transform", ctypes.c_float * 16),
                ("masks", ctypes.POINTER(ctypes.c_uint32)), ("n_masks", ctypes.c_uint64)]


class RtTuning(ctypes.Structure):
    _fields_ = [("fast_refill", ctypes.c_uint32), ("wide8_refill", ctypes.c_uint32), ("wide8_stack", ctypes.c_uint32),
                ("wide8_entries", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 4)]


EXPORTS = ("rt_abi_version", "rt_ctx_create", "rt_ctx_destroy", "rt_get_last_error", "rt_get_stats",
           "rt_ctx_set_tuning", "rt_ctx_get_tuning",
           "rt_selftest", "rt_scene_upload", "rt_scene_update_records", "rt_scene_release",
           "rt_scene_device_bytes", "rt_scene_validate", "rt_scene_prepare", "rt_trace", "rt_trace_ex", "rt_trace_host", "rt_trace_host_batches", "rt_ctx_reserve", "rt_trace_counted", "rt_order_rays",
           "rt_trace_batches", "rt_plan_create", "rt_plan_launch", "rt_plan_info", "rt_plan_destroy",
           "rt_scene_refit", "rt_scene_read_words", "rt_scene_tune_top", "rt_gi_cell_rays", "rt_trace_gi_cells", "rt_trace_gi_lights", "rt_server_create", "rt_server_add_scene", "rt_server_remove_scene", "rt_server_submit",
           "rt_server_wait", "rt_server_get_stats", "rt_server_fail_next", "rt_server_destroy",
           "rt_trace_static", "rt_trace_static_stack_drops", "rt_read_bandwidth", "rt_scene_wide8_depth", "rt_wide8_check", "rt_object_box", "rt_move_instances_host",
           "rt_scene_move_instances", "rt_blas_build", "rt_blas_build_device", "rt_blas_info", "rt_blas_nodes", "rt_blas_indices", "rt_blas_refit",
           "rt_blas_free", "rt_pack_scene", "rt_tlas_build", "rt_tlas_build_device", "rt_tlas_refit", "rt_blas_positions",
           "rt_blas_encode_rlb", "rt_rlb_decode", "rt_rnf_decode", "rt_rnf_info", "rt_rnf_mesh",
           "rt_rnf_placement_get", "rt_rnf_encode", "rt_rnf_pack_gi", "rt_rnf_world", "rt_rnf_free")

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it was never built: there is no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m renderlab_b200.build` "
                           "(the engine has no CPU fallback)")
    L = ctypes.CDLL(str(LIB_PATH))
    L.rt_abi_version.restype = ctypes.c_uint32
    L.rt_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
    L.rt_ctx_destroy.argtypes = [_vp]
    L.rt_ctx_destroy.restype = None
    L.rt_get_last_error.argtypes = [_vp]
    L.rt_get_last_error.restype = ctypes.c_char_p
    L.rt_get_stats.argtypes = [_vp, ctypes.POINTER(RtStats)]
    L.rt_selftest.argtypes = [_vp, _u32p]
    L.rt_ctx_set_tuning.argtypes = [_vp, ctypes.POINTER(RtTuning)]
    L.rt_ctx_get_tuning.argtypes = [_vp, ctypes.POINTER(RtTuning)]
    L.rt_scene_upload.argtypes = [_vp, ctypes.c_int, _u32p, ctypes.c_size_t, ctypes.POINTER(_vp)]
    L.rt_scene_validate.argtypes = [ctypes.c_int, _u32p, ctypes.c_size_t, _u32p, ctypes.c_char_p, ctypes.c_size_t]
    L.rt_scene_update_records.argtypes = [_vp, _vp, _u32p, ctypes.c_size_t]
    L.rt_scene_release.argtypes = [_vp, _vp]
    L.rt_scene_prepare.argtypes = [_vp, _vp, ctypes.c_int]
    L.rt_scene_wide8_depth.argtypes = [_vp, _u32p]
    L.rt_scene_tune_top.argtypes = [_vp, _vp, _u32p, ctypes.c_uint32, ctypes.c_uint32, _u32p]
    L.rt_wide8_check.argtypes = [ctypes.c_int, _u32p, ctypes.c_size_t, _u32p, ctypes.c_char_p, ctypes.c_size_t]
    L.rt_object_box.argtypes = [ctypes.c_int, _vp, _f32p, _u32p, ctypes.c_uint32, _f32p]
    L.rt_move_instances_host.argtypes = [ctypes.c_int, _u32p, ctypes.c_size_t, ctypes.POINTER(RtInstance),
                                         ctypes.c_uint32, _f32p, ctypes.c_uint32]
    L.rt_scene_move_instances.argtypes = [_vp, _vp, ctypes.POINTER(RtInstance), ctypes.c_uint32, _f32p,
                                          ctypes.c_uint32, _vp]
    L.rt_scene_device_bytes.argtypes = [_vp]
    L.rt_scene_device_bytes.restype = ctypes.c_size_t
    L.rt_trace.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_uint32, _vp]
    L.rt_trace_ex.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_uint32, _vp]
    L.rt_trace_host.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_uint32]
    L.rt_trace_host_batches.argtypes = [_vp, _vp, ctypes.POINTER(RtHostBatch), ctypes.c_uint32]
    L.rt_ctx_reserve.argtypes = [_vp, ctypes.c_uint32]
    L.rt_order_rays.argtypes = [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_int, _vp, _vp]
    L.rt_trace_batches.argtypes = [_vp, _vp, ctypes.c_int, ctypes.POINTER(RtBatch), ctypes.c_uint32, _vp]
    L.rt_plan_create.argtypes = [_vp, _vp, ctypes.POINTER(RtBatch), ctypes.c_uint32, ctypes.POINTER(RtPlanDesc),
                                 ctypes.POINTER(_vp)]
    L.rt_plan_launch.argtypes = [_vp, _vp]
    L.rt_plan_info.argtypes = [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.rt_plan_destroy.argtypes = [_vp]
    L.rt_scene_refit.argtypes = [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_uint32, _vp, ctypes.c_uint32, _vp]
    L.rt_gi_cell_rays.argtypes = [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp]
    L.rt_trace_gi_cells.argtypes = [_vp, _vp, ctypes.c_int, _vp, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp]
    L.rt_trace_gi_lights.argtypes = [_vp, _vp, ctypes.c_int, _vp, ctypes.c_uint32, _vp, ctypes.c_uint32, _vp, _vp]
    L.rt_scene_read_words.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _u32p]
    L.rt_server_create.argtypes = [_vp, ctypes.POINTER(RtServerDesc), ctypes.POINTER(_vp)]
    L.rt_server_add_scene.argtypes = [_vp, ctypes.c_int, _u32p, ctypes.c_size_t, _u32p]
    L.rt_server_remove_scene.argtypes = [_vp, ctypes.c_uint32]
    L.rt_server_submit.argtypes = [_vp, ctypes.c_uint32, ctypes.c_int, _vp, ctypes.c_uint32, _vp,
                                   ctypes.POINTER(ctypes.c_uint64)]
    L.rt_server_wait.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int32]
    L.rt_server_get_stats.argtypes = [_vp, ctypes.POINTER(RtServerStats), ctypes.c_int]
    L.rt_server_fail_next.argtypes = [_vp, ctypes.c_uint32, ctypes.c_int]
    L.rt_server_destroy.argtypes = [_vp]
    L.rt_trace_static.argtypes = [ctypes.c_int, _vp, ctypes.c_size_t, ctypes.c_int, _vp, _vp, ctypes.c_uint32, _vp]
    L.rt_trace_static_stack_drops.argtypes = [_vp, ctypes.POINTER(ctypes.c_uint64)]
    L.rt_read_bandwidth.argtypes = [_vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]
    L.rt_trace_counted.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_uint64)]
    L.rt_blas_build.argtypes = [_f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_vp)]
    L.rt_blas_build_device.argtypes = [_vp, _f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.POINTER(_vp)]
    L.rt_blas_info.argtypes = [_vp, _u32p]
    L.rt_blas_nodes.argtypes = [_vp, _u32p]
    L.rt_blas_indices.argtypes = [_vp, _u32p]
    L.rt_blas_refit.argtypes = [_vp, _f32p, ctypes.c_uint32]
    L.rt_blas_free.argtypes = [_vp]
    L.rt_blas_free.restype = None
    L.rt_pack_scene.argtypes = [ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_uint32, ctypes.POINTER(_f32p),
                                ctypes.POINTER(_u32p), _u32p, _u32p, ctypes.POINTER(RtInstance), ctypes.c_uint32,
                                ctypes.c_int, _u32p, ctypes.POINTER(ctypes.c_size_t)]
    L.rt_tlas_build.argtypes = [_f32p, ctypes.c_uint32, ctypes.c_int, _u32p, ctypes.POINTER(ctypes.c_size_t)]
    L.rt_tlas_build_device.argtypes = [_vp, _f32p, ctypes.c_uint32, ctypes.c_int, _u32p, ctypes.POINTER(ctypes.c_size_t)]
    L.rt_tlas_refit.argtypes = [_u32p, ctypes.c_size_t, _f32p, ctypes.c_uint32]
    _sz = ctypes.POINTER(ctypes.c_size_t)
    L.rt_blas_positions.argtypes = [_vp, _f32p]
    L.rt_blas_encode_rlb.argtypes = [_vp, ctypes.c_uint64, _vp, _sz, ctypes.c_char_p, ctypes.c_size_t]
    L.rt_rlb_decode.argtypes = [_vp, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_vp),
                                ctypes.c_char_p, ctypes.c_size_t]
    L.rt_rnf_decode.argtypes = [_vp, ctypes.c_size_t, ctypes.c_uint64, ctypes.POINTER(_vp), ctypes.c_char_p,
                                ctypes.c_size_t]
    L.rt_rnf_info.argtypes = [_vp, ctypes.POINTER(RtRnfSettings), _vp, _u32p, _u32p]
    L.rt_rnf_mesh.argtypes = [_vp, ctypes.c_uint32, ctypes.POINTER(_vp)]
    L.rt_rnf_placement_get.argtypes = [_vp, ctypes.c_uint32, ctypes.POINTER(RtRnfPlacement)]
    L.rt_rnf_encode.argtypes = [ctypes.POINTER(RtRnfSettings), _vp, ctypes.POINTER(_vp), ctypes.c_uint32,
                                ctypes.POINTER(RtRnfPlacement), ctypes.c_uint32, ctypes.c_uint64, _vp, _sz,
                                ctypes.c_char_p, ctypes.c_size_t]
    L.rt_rnf_pack_gi.argtypes = [_vp, ctypes.POINTER(RtInstance), ctypes.c_uint32, ctypes.c_int, _u32p, _sz]
    L.rt_rnf_world.argtypes = [_vp, ctypes.POINTER(_vp), _u32p]
    L.rt_rnf_free.argtypes = [_vp]
    L.rt_rnf_free.restype = None
    for name in EXPORTS:
        if name not in ("rt_ctx_destroy", "rt_blas_free", "rt_abi_version", "rt_get_last_error",
                        "rt_scene_device_bytes", "rt_rnf_free"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _np_ptr(a, t):
    return a.ctypes.data_as(t)


# ---------------------------------------------------------------- host builders

class Blas:
    """A BVH4-Q8 over one triangle mesh (near_field.rs build_bvh_sah / build_bvh)."""

    def __init__(self, positions, indices, median: bool = False):
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        h = _vp()
        st = lib().rt_blas_build(_np_ptr(self.positions, _f32p), len(self.positions), _np_ptr(self.indices, _u32p),
                                 len(self.indices), 1 if median else 0, ctypes.byref(h))
        if st != 0:
            raise RtError(st, "BVH geometry needs a nonempty, finite triangle list")
        self.h = h

    @classmethod
    def build_device(cls, engine: "Engine", positions, indices, median: bool = False) -> "Blas":
        """The same BLAS built on the engine's GPU (rt_blas_build_device): word for word the host
        build's records."""
        self = cls.__new__(cls)
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        h = _vp()
        engine._check(lib().rt_blas_build_device(engine.ctx, _np_ptr(self.positions, _f32p), len(self.positions),
                                                 _np_ptr(self.indices, _u32p), len(self.indices), 1 if median else 0,
                                                 ctypes.byref(h)))
        self.h = h
        return self

    @classmethod
    def adopt(cls, h) -> "Blas":
        """Takes ownership of a library-made BLAS handle (a decoded file's mesh); its positions
        are the BLAS's own and its triangle list the BVH's (reordered) one."""
        self = cls.__new__(cls)
        self.h = h
        info = self.info()
        self.positions = np.zeros((info["positions"], 3), np.float32)
        lib().rt_blas_positions(h, _np_ptr(self.positions, _f32p))
        self.indices = self.bvh_indices()
        return self

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.rt_blas_free(self.h)
            self.h = None

    def info(self) -> dict:
        out = np.zeros(6, np.uint32)
        lib().rt_blas_info(self.h, _np_ptr(out, _u32p))
        return dict(zip(("nodes", "leaves", "positions", "indices", "root", "depth"), map(int, out)))

    def nodes(self) -> np.ndarray:
        out = np.zeros((self.info()["nodes"], 16), np.uint32)
        lib().rt_blas_nodes(self.h, _np_ptr(out, _u32p))
        return out

    def bvh_indices(self) -> np.ndarray:
        out = np.zeros(self.info()["indices"], np.uint32)
        lib().rt_blas_indices(self.h, _np_ptr(out, _u32p))
        return out

    def refit(self, positions) -> None:
        p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        st = lib().rt_blas_refit(self.h, _np_ptr(p, _f32p), len(p))
        if st != 0:
            raise RtError(st, "refit needs finite positions of the same vertices")
        self.positions = p


def _instance_array(layout: int, instances):
    """rt_instance records for an Instances-like object (see pack_scene)."""
    n = len(instances.mesh)
    arr = (RtInstance * max(n, 1))()
    model = np.ascontiguousarray(instances.model, np.float32).reshape(n, 12)
    rows = np.ascontiguousarray(instances.rows, np.float32).reshape(n, 12)
    casts = getattr(instances, "casts", None)
    slot = getattr(instances, "slot", None)
    near = getattr(instances, "near_base", None)
    extra = getattr(instances, "extra", None)
    for i in range(n):
        rec = arr[i]
        ctypes.memmove(rec.model, model[i].ctypes.data, 48)
        ctypes.memmove(rec.rows, rows[i].ctypes.data, 48)
        rec.mesh = int(instances.mesh[i])
        rec.slot = int(slot[i]) if slot is not None else i
        rec.casts_shadow = int(bool(casts[i])) if casts is not None else 1
        rec.near_base = int(near[i]) if near is not None else 0
        if extra is not None:
            for k in range(8):
                rec.extra[k] = int(extra[i][k])
        elif casts is not None and layout == LAYOUT_GI:
            rec.extra[3] = 0 if casts[i] else 1
    return arr, n


def pack_scene(layout: int, meshes, instances, tlas_mode: int = -1, primitives=None) -> np.ndarray:
    """Packed words of `layout` for meshes (list of Blas) placed by `instances`.

    instances: object with ``model`` (N,3,4), ``rows`` (N,3,4), ``mesh`` (N,), and optionally
    ``casts`` (N,) bool, ``slot`` (N,), ``near_base`` (N,), ``extra`` (N,8).
    primitives: per mesh, whether the GI layout carries its primitive table.
    """
    arr, n = _instance_array(layout, instances)
    m = len(meshes)
    handles = (_vp * max(m, 1))(*[b.h for b in meshes])
    pos_ptrs = (_f32p * max(m, 1))(*[_np_ptr(b.positions, _f32p) for b in meshes])
    idx_ptrs = (_u32p * max(m, 1))(*[_np_ptr(b.indices, _u32p) for b in meshes])
    nidx = np.array([len(b.indices) for b in meshes] or [0], np.uint32)
    prim = np.array([int(bool(p)) for p in (primitives or [False] * m)] or [0], np.uint32)
    size = ctypes.c_size_t(0)
    L = lib()
    args = (layout, handles, m, pos_ptrs, idx_ptrs, _np_ptr(nidx, _u32p), _np_ptr(prim, _u32p), arr, n, tlas_mode)
    st = L.rt_pack_scene(*args, None, ctypes.byref(size))
    if st != 0:
        raise RtError(st, "packing failed (singular transform, bad mesh index or unmappable triangles)")
    out = np.zeros(size.value, np.uint32)
    st = L.rt_pack_scene(*args, _np_ptr(out, _u32p), ctypes.byref(size))
    if st != 0:
        raise RtError(st, "packing failed")
    return out


def object_boxes(layout: int, meshes) -> np.ndarray:
    """(n_meshes, 6) float32: the object box rt_pack_scene places for each mesh (Blas objects)."""
    out = np.zeros((len(meshes), 6), np.float32)
    for m, b in enumerate(meshes):
        st = lib().rt_object_box(layout, b.h, _np_ptr(b.positions, _f32p), _np_ptr(b.indices, _u32p),
                                 len(b.indices), _np_ptr(out[m], _f32p))
        if st != 0:
            raise RtError(st, "object box")
    return out


def move_instances_host(layout: int, words, instances, mesh_boxes) -> np.ndarray:
    """A copy of packed words with `instances` (Instances-like, the scene's, in order) moved: new
    records, the top level refit (or rebuilt after 64 refits) and scene bounds
    (rt_move_instances_host)."""
    w = np.array(words, np.uint32, copy=True)
    arr, n = _instance_array(layout, instances)
    boxes = np.ascontiguousarray(mesh_boxes, np.float32).reshape(-1, 6)
    st = lib().rt_move_instances_host(layout, _np_ptr(w, _u32p), len(w), arr, n, _np_ptr(boxes, _f32p), len(boxes))
    if st != 0:
        raise RtError(st, "moved instances refused (count, mesh index or a singular placement)")
    return w


def wide8_check(layout: int, words) -> dict:
    """Builds the 8-wide layout on the host and checks it (rt_wide8_check); raises RtError(LAYOUT)
    with the reason, else returns its node, triangle, depth and BLAS counts."""
    w = np.ascontiguousarray(words, np.uint32)
    info = np.zeros(4, np.uint32)
    err = ctypes.create_string_buffer(256)
    st = lib().rt_wide8_check(layout, _np_ptr(w, _u32p), len(w), _np_ptr(info, _u32p), err, len(err))
    if st != 0:
        raise RtError(st, err.value.decode())
    return dict(zip(("nodes", "triangles", "depth", "blas"), map(int, info)))


def validate(layout: int, words) -> dict:
    """The upload admission check on the host; raises RtError(LAYOUT) with the reason."""
    w = np.ascontiguousarray(words, np.uint32)
    info = np.zeros(8, np.uint32)
    err = ctypes.create_string_buffer(256)
    st = lib().rt_scene_validate(layout, _np_ptr(w, _u32p), len(w), _np_ptr(info, _u32p), err, 256)
    if st != 0:
        raise RtError(st, err.value.decode())
    return dict(zip(("instances", "top", "root", "triangles", "nodes", "blas_depth", "top_depth"), map(int, info)))


def tlas_build(boxes, sah: bool = True) -> np.ndarray:
    b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    size = ctypes.c_size_t(0)
    st = lib().rt_tlas_build(_np_ptr(b, _f32p), len(b), int(sah), None, ctypes.byref(size))
    if st != 0:
        raise RtError(st, "top level needs at least two boxes")
    out = np.zeros(size.value, np.uint32)
    lib().rt_tlas_build(_np_ptr(b, _f32p), len(b), int(sah), _np_ptr(out, _u32p), ctypes.byref(size))
    return out


def tlas_build_device(engine: "Engine", boxes, sah: bool = True) -> np.ndarray:
    """tlas_build run on the engine's GPU (rt_tlas_build_device): the same node words."""
    b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    out = np.zeros(max(len(b) - 1, 1) * 32, np.uint32)  # the reserve: at most n - 1 nodes
    size = ctypes.c_size_t(out.size)
    engine._check(lib().rt_tlas_build_device(engine.ctx, _np_ptr(b, _f32p), len(b), int(sah), _np_ptr(out, _u32p),
                                             ctypes.byref(size)))
    return out[: size.value]


def tlas_refit(nodes, boxes) -> np.ndarray:
    nodes = np.ascontiguousarray(nodes, np.uint32).copy()
    b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    st = lib().rt_tlas_refit(_np_ptr(nodes, _u32p), len(nodes), _np_ptr(b, _f32p), len(b))
    if st != 0:
        raise RtError(st, "refit needs at least two boxes")
    return nodes


# ---------------------------------------------------------------- device side

def hit_words(layout: int, mode: int) -> int:
    if mode != CLOSEST:
        return 1
    return GI_HIT_WORDS if layout == LAYOUT_GI else RS_HIT_WORDS


@dataclass
class Scene:
    engine: "Engine"
    handle: int
    layout: int
    n_words: int

    def release(self):
        if self.handle:
            self.engine._check(lib().rt_scene_release(self.engine.ctx, self.handle))
            self.handle = None

    def prepare(self, kernel: str = "wide8"):
        """Build the derived layout `kernel` reads (the 8-wide BVH for "wide8")."""
        self.engine._check(lib().rt_scene_prepare(self.engine.ctx, self.handle, KERNELS[kernel]))

    def move_instances(self, instances, mesh_boxes, stream=None):
        """Moves the scene's instances on the device (rt_scene_move_instances); `instances` as
        pack_scene takes them (the scene's, in order), `mesh_boxes` from object_boxes()."""
        arr, n = _instance_array(self.layout, instances)
        boxes = np.ascontiguousarray(mesh_boxes, np.float32).reshape(-1, 6)
        if stream is None:
            import torch
            stream = torch.cuda.current_stream().cuda_stream
        s = stream
        self.engine._check(lib().rt_scene_move_instances(self.engine.ctx, self.handle, arr, n, _np_ptr(boxes, _f32p),
                                                         len(boxes), s))

    def tune_top(self, budgets=None, probe: int = 0) -> int:
        """rt_scene_tune_top: measures the WIDE8 top level's entries per instance over a probe of
        incoherent closest- and any-hit rays (after prepare("wide8")), keeps the fastest and
        returns it (0: the scene has no top level)."""
        b = None if budgets is None else np.ascontiguousarray(budgets, np.uint32)
        out = ctypes.c_uint32()
        self.engine._check(lib().rt_scene_tune_top(self.engine.ctx, self.handle, _np_ptr(b, _u32p) if b is not None else None,
                                                   0 if b is None else len(b), probe, ctypes.byref(out)))
        return int(out.value)

    def wide8_depth(self) -> int:
        """Levels of the deepest 8-wide BLAS (after prepare("wide8")); the shared stack takes 16."""
        d = ctypes.c_uint32()
        self.engine._check(lib().rt_scene_wide8_depth(self.handle, ctypes.byref(d)))
        return int(d.value)

    def refit(self, instance: int, positions, indices=None, stream=None):
        """rt_scene_refit: new positions (CUDA float32 tensor (V, 3)) for the BLAS of `instance`;
        the reflection layout also takes the mesh's triangle list (CUDA int32/uint32 tensor)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        n_idx = 0 if indices is None else int(indices.numel())
        self.engine._check(lib().rt_scene_refit(self.engine.ctx, self.handle, instance, positions.data_ptr(),
                                                int(positions.shape[0]), indices.data_ptr() if indices is not None else None,
                                                n_idx, s))

    def words(self, first: int = 0, n: int = -1) -> np.ndarray:
        """A host copy of the scene's device words [first, first + n)."""
        n = self.n_words - first if n < 0 else n
        out = np.zeros(n, np.uint32)
        self.engine._check(lib().rt_scene_read_words(self.engine.ctx, self.handle, first, n, _np_ptr(out, _u32p)))
        return out

    def update_records(self, words):
        w = np.ascontiguousarray(words, np.uint32)
        self.engine._check(lib().rt_scene_update_records(self.engine.ctx, self.handle, _np_ptr(w, _u32p), len(w)))

    @property
    def device_bytes(self) -> int:
        return int(lib().rt_scene_device_bytes(self.handle))


class Plan:
    """A many-batch launch prepared once and replayed (a CUDA graph unless graph=False). Holds
    the batches' ray tensors and owns their hit tensors (`hits`)."""

    def __init__(self, engine: "Engine", scene: Scene, handle, hits, rays, desc: dict):
        self.engine, self.scene, self.handle, self.hits, self.rays, self.desc = engine, scene, handle, hits, rays, desc

    def launch(self, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self.engine._check(lib().rt_plan_launch(self.handle, s))

    def info(self) -> dict:
        rays, nbytes = ctypes.c_uint64(), ctypes.c_uint64()
        self.engine._check(lib().rt_plan_info(self.handle, ctypes.byref(rays), ctypes.byref(nbytes)))
        return {"rays": int(rays.value), "device_bytes": int(nbytes.value)}

    def close(self):
        if self.handle:
            lib().rt_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (rt_server_*): submit host ray batches for resident scenes from any
    thread, wait for their hits. Keeps each request's buffers alive until it is waited for."""

    def __init__(self, engine: "Engine", hbm_budget: int, launch_rays: int = 1 << 22, slots: int = 4,
                 kernel: str = "wide8"):
        self.engine = engine
        desc = RtServerDesc(int(hbm_budget), int(launch_rays), int(slots), KERNELS[kernel])
        h = _vp()
        engine._check(lib().rt_server_create(engine.ctx, ctypes.byref(desc), ctypes.byref(h)))
        self.handle, self.kernel, self.layouts, self._held = h, kernel, {}, {}

    def add_scene(self, layout: int, words) -> int:
        w = np.ascontiguousarray(words, np.uint32)
        sid = ctypes.c_uint32()
        self.engine._check(lib().rt_server_add_scene(self.handle, layout, _np_ptr(w, _u32p), len(w), ctypes.byref(sid)))
        self.layouts[sid.value] = layout
        return sid.value

    def remove_scene(self, sid: int):
        self.engine._check(lib().rt_server_remove_scene(self.handle, sid))

    def submit(self, sid: int, rays, mode: int = CLOSEST, out=None) -> int:
        """rays: (n, 8) float32 host array (numpy, or a pinned torch CPU tensor). Returns a ticket."""
        n = len(rays)
        # an unknown scene id goes to the library, which refuses it (RT_ERR_INVALID_ARG)
        words = hit_words(self.layouts.get(sid, LAYOUT_REFLECTION), mode)
        if out is None:
            out = np.zeros((n, words) if words > 1 else (n,), np.uint32)
        rp = rays.data_ptr() if hasattr(rays, "data_ptr") else rays.ctypes.data
        hp = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        t = ctypes.c_uint64()
        self.engine._check(lib().rt_server_submit(self.handle, sid, mode, rp if n else None, n, hp if n else None,
                                                  ctypes.byref(t)))
        self._held[t.value] = (rays, out)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """The request's hits (raises RtError TIMEOUT if it is still running after timeout_ms)."""
        st = lib().rt_server_wait(self.handle, ticket, timeout_ms)
        if st == 5:
            raise RtError(st, "request still running")
        rays, out = self._held.pop(ticket, (None, None))  # released once waited for, whatever the status
        self.engine._check(st)
        return out

    def fail_next(self, launches: int, status: int = 6):
        """rt_server_fail_next: the next `launches` slot launches fail on the host with `status`
        (default RT_ERR_CUDA) before anything is enqueued -- failure injection for tests."""
        self.engine._check(lib().rt_server_fail_next(self.handle, launches, status))

    def stats(self, reset: bool = False) -> dict:
        s = RtServerStats()
        self.engine._check(lib().rt_server_get_stats(self.handle, ctypes.byref(s), 1 if reset else 0))
        return {f: (float(getattr(s, f)) if t is ctypes.c_double else int(getattr(s, f))) for f, t in RtServerStats._fields_}

    def close(self):
        if self.handle:
            lib().rt_server_destroy(self.handle)
            self.handle = None
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """One context on one CUDA device."""

    def __init__(self, device: int = 0):
        self.device = device
        h = _vp()
        st = lib().rt_ctx_create(device, ctypes.byref(h))
        if st != 0:
            raise RtError(st, f"cannot create a context on device {device}")
        self.ctx = h

    def close(self):
        if getattr(self, "ctx", None):
            lib().rt_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        if _lib is not None:
            self.close()

    def _check(self, st: int):
        if st != 0:
            raise RtError(st, lib().rt_get_last_error(self.ctx).decode())

    def selftest(self) -> np.ndarray:
        out = np.zeros(16, np.uint32)
        self._check(lib().rt_selftest(self.ctx, _np_ptr(out, _u32p)))
        return out

    def set_tuning(self, **kw):
        t = RtTuning()
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._check(lib().rt_ctx_set_tuning(self.ctx, ctypes.byref(t)))

    def tuning(self) -> dict:
        t = RtTuning()
        self._check(lib().rt_ctx_get_tuning(self.ctx, ctypes.byref(t)))
        return {f: int(getattr(t, f)) for f, _ in RtTuning._fields_ if f != "reserved"}

    def stats(self) -> dict:
        s = RtStats()
        self._check(lib().rt_get_stats(self.ctx, ctypes.byref(s)))
        return {f: int(getattr(s, f)) for f, _ in RtStats._fields_}

    def upload(self, layout: int, words) -> Scene:
        w = np.ascontiguousarray(words, np.uint32)
        h = _vp()
        self._check(lib().rt_scene_upload(self.ctx, layout, _np_ptr(w, _u32p), len(w), ctypes.byref(h)))
        return Scene(self, h, layout, len(w))

    def trace(self, scene: Scene, rays, mode: int = CLOSEST, kernel: str = "plain", order=None, hits=None,
              stream=None):
        """Trace a torch CUDA tensor of rays (n, 8) float32; returns the int32 hit tensor."""
        import torch
        assert rays.is_cuda and rays.dtype == torch.float32 and rays.is_contiguous()
        n = rays.shape[0]
        words = hit_words(scene.layout, mode)
        if hits is None:
            hits = torch.empty((n, words) if words > 1 else (n,), dtype=torch.int32, device=rays.device)
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        self._check(lib().rt_trace_ex(self.ctx, scene.handle, mode, KERNELS[kernel], rays.data_ptr(),
                                      order.data_ptr() if order is not None else None, hits.data_ptr(), n, s))
        return hits

    def trace_host(self, scene: Scene, rays, mode: int = CLOSEST, kernel: str = "plain", out=None):
        """Trace host rays (numpy or pinned torch CPU tensor, (n, 8) float32) into host hits."""
        n = len(rays)
        words = hit_words(scene.layout, mode)
        if out is None:
            out = np.zeros((n, words) if words > 1 else (n,), np.uint32)
        rp = rays.data_ptr() if hasattr(rays, "data_ptr") else rays.ctypes.data
        hp = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        self._check(lib().rt_trace_host(self.ctx, scene.handle, mode, KERNELS[kernel], rp, hp, n))
        return out

    def trace_host_batches(self, scene: Scene, batches):
        """Host-buffer batches in one pipeline: (rays, mode, kernel[, out]) tuples, rays numpy or
        pinned torch CPU tensors; returns the hit arrays (the given `out`s where passed)."""
        arr = (RtHostBatch * max(1, len(batches)))()
        outs = []
        for k, b in enumerate(batches):
            rays, mode, kernel = b[0], b[1], b[2]
            out = b[3] if len(b) > 3 and b[3] is not None else None
            n = len(rays)
            if out is None:
                words = hit_words(scene.layout, mode)
                out = np.zeros((n, words) if words > 1 else (n,), np.uint32)
            outs.append(out)
            arr[k].h_rays = rays.data_ptr() if hasattr(rays, "data_ptr") else rays.ctypes.data
            arr[k].h_hits = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
            arr[k].n, arr[k].mode, arr[k].kernel = n, mode, KERNELS[kernel]
        self._check(lib().rt_trace_host_batches(self.ctx, scene.handle, arr, len(batches)))
        return outs

    def _batch_array(self, scene: Scene, batches):
        """(rays, mode[, hits]) tuples -> (ctypes RtBatch array, hit tensors)."""
        import torch
        arr = (RtBatch * max(1, len(batches)))()
        outs = []
        for i, b in enumerate(batches):
            rays, mode = b[0], b[1]
            assert rays.is_cuda and rays.dtype == torch.float32 and rays.is_contiguous()
            hits = b[2] if len(b) > 2 and b[2] is not None else None
            words = hit_words(scene.layout, mode)
            n = rays.shape[0]
            if hits is None:
                hits = torch.empty((n, words) if words > 1 else (n,), dtype=torch.int32, device=rays.device)
            arr[i] = RtBatch(rays.data_ptr() if n else None, hits.data_ptr() if n else None, n, mode)
            outs.append(hits)
        return arr, outs

    def trace_batches(self, scene: Scene, batches, kernel: str = "fast", stream=None):
        """Trace many (rays, mode[, hits]) batches of one scene in one persistent launch; returns the
        hit tensors, one per batch."""
        import torch
        arr, outs = self._batch_array(scene, batches)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(lib().rt_trace_batches(self.ctx, scene.handle, KERNELS[kernel], arr, len(batches), s))
        return outs

    def plan(self, scene: Scene, batches, kernel: str = "fast", refill: int = 0, order: str = "none",
             graph: bool = True, stack: str = "") -> "Plan":
        """A prepared many-batch launch over fixed buffers (see rt_plan_create). `stack`: where
        WIDE8 keeps each lane's node-group stack, "local" or "shared" ("": the context's tuning)."""
        arr, outs = self._batch_array(scene, batches)
        desc = RtPlanDesc(KERNELS[kernel], refill, ORDERS[order], 1 if graph else 0, STACKS[stack])
        h = _vp()
        self._check(lib().rt_plan_create(self.ctx, scene.handle, arr, len(batches), ctypes.byref(desc), ctypes.byref(h)))
        desc = dict(kernel=kernel, refill=refill, order=order, graph=graph)
        if stack:
            desc["stack"] = stack
        return Plan(self, scene, h, outs, [b[0] for b in batches], desc)

    def gi_cell_rays(self, cells, rotate: bool = False, stream=None):
        """The GI cache cells' 64 fixed-direction rays each: cells (n, 8) int32 CUDA tensor of
        rt_gi_cell records; returns (n * 64, 8) float32."""
        import torch
        n = cells.shape[0]
        rays = torch.empty((n * GI_DIRECTIONS, 8), dtype=torch.float32, device=cells.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(lib().rt_gi_cell_rays(self.ctx, cells.data_ptr(), n, GI_ROTATE if rotate else 0, rays.data_ptr(), s))
        return rays

    def trace_gi_cells(self, scene: Scene, cells, mode: int = CLOSEST, rotate: bool = False, hits=None, stream=None):
        """The cells' rays generated inside the FAST kernel and traced (GI layout): rt_gi_hit per
        item for CLOSEST, a blocked flag per item for ANY_SKY."""
        import torch
        n = cells.shape[0] * GI_DIRECTIONS
        words = hit_words(scene.layout, mode)
        if hits is None:
            hits = torch.empty((n, words) if words > 1 else (n,), dtype=torch.int32, device=cells.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(lib().rt_trace_gi_cells(self.ctx, scene.handle, mode, cells.data_ptr(), cells.shape[0],
                                            GI_ROTATE if rotate else 0, hits.data_ptr(), s))
        return hits

    def trace_gi_lights(self, scene: Scene, cells, lights, kernel: str = "fast", out=None, stream=None):
        """gi_light's visibility words (GI layout): cells (n, 8) and lights (m, 20) 32-bit CUDA
        tensors (rt_gi_cell / rt_gi_light records); returns (n, ceil(m / 32)) int32 words, bit
        l % 32 of word l / 32 set when light l reaches the cell and nothing blocks its ray."""
        import torch
        n, m = cells.shape[0], lights.shape[0]
        if cells.shape[1:] != (8,) or lights.shape[1:] != (20,) or cells.element_size() != 4 or lights.element_size() != 4:
            raise ValueError("cells must be (n, 8) and lights (m, 20) tensors of 32-bit words")
        if not cells.is_contiguous() or not lights.is_contiguous():
            raise ValueError("cells and lights must be contiguous")
        if out is None:
            out = torch.empty((n, (m + 31) // 32), dtype=torch.int32, device=cells.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(lib().rt_trace_gi_lights(self.ctx, scene.handle, KERNELS[kernel], cells.data_ptr(), n,
                                             lights.data_ptr(), m, out.data_ptr(), s))
        return out

    def order(self, scene: Scene, rays, key: str = "octant", out=None, stream=None):
        """A permutation of `rays` (CUDA tensor) grouping alike rays; int32 CUDA tensor."""
        import torch
        n = rays.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.int32, device=rays.device)
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        self._check(lib().rt_order_rays(self.ctx, scene.handle, rays.data_ptr(), n, ORDERS[key], out.data_ptr(), s))
        return out

    COUNTERS = ("rays", "top_nodes", "instance_tests", "nodes", "leaves", "triangles", "f64_retests", "f64_final")

    def trace_counted(self, scene: Scene, rays, mode: int = CLOSEST, kernel: str = "wide8") -> dict:
        """Trace in the instrumented build; returns the visit counters over the batch."""
        import torch
        n = rays.shape[0]
        words = hit_words(scene.layout, mode)
        hits = torch.empty((n, words) if words > 1 else (n,), dtype=torch.int32, device=rays.device)
        out = (ctypes.c_uint64 * 8)()
        self._check(lib().rt_trace_counted(self.ctx, scene.handle, mode, KERNELS[kernel], rays.data_ptr(),
                                           hits.data_ptr(), n, out))
        return dict(zip(self.COUNTERS, map(int, out)))

    def read_bandwidth(self, nbytes: int, reps: int = 20) -> float:
        """rt_read_bandwidth: GB/s of 16-byte loads (L1 bypassed) over an `nbytes` device buffer --
        L2's read bandwidth for buffers well inside L2, HBM's for buffers far larger."""
        out = ctypes.c_double(0.0)
        self._check(lib().rt_read_bandwidth(self.ctx, int(nbytes), int(reps), ctypes.byref(out)))
        return out.value

    def reserve(self, max_rays: int):
        self._check(lib().rt_ctx_reserve(self.ctx, max_rays))


STATIC_MAX_RAYS = 1 << 31


def trace_static(layout: int, d_words, rays, mode: int = CLOSEST, hits=None, stream=None):
    """rt_trace_static: the FAST traversal with no allocation by the library and no context.

    d_words: the packed words in a caller-owned contiguous torch CUDA tensor (int32/uint32 view,
    words that `validate` accepted); rays: a contiguous (n, 8) float32 CUDA tensor on the same
    device. Returns the int32 hit tensor. The call runs with the rays' device current."""
    import torch
    if rays.dtype != torch.float32 or rays.dim() != 2 or rays.shape[1] != 8 or not rays.is_contiguous():
        raise ValueError("rays must be a contiguous (n, 8) float32 tensor")
    if not rays.is_cuda or not d_words.is_cuda or d_words.device != rays.device:
        raise ValueError("rays and d_words must be CUDA tensors on one device")
    if d_words.element_size() != 4 or not d_words.is_contiguous():
        raise ValueError("d_words must be a contiguous tensor of 32-bit words")
    n = rays.shape[0]
    words = hit_words(layout, mode)
    shape = (n, words) if words > 1 else (n,)
    if hits is None:
        hits = torch.empty(shape, dtype=torch.int32, device=rays.device)
    elif (hits.device != rays.device or hits.element_size() != 4 or not hits.is_contiguous()
          or hits.numel() != n * words):
        raise ValueError(f"hits must be a contiguous tensor of {n * words} 32-bit words on the rays' device")
    with torch.cuda.device(rays.device):
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        st = lib().rt_trace_static(layout, d_words.data_ptr(), d_words.numel(), mode, rays.data_ptr(),
                                   hits.data_ptr(), n, s)
    if st != 0:
        raise RtError(st, "rt_trace_static refused the call (sizes, alignment or layout)")
    return hits


def trace_static_stack_drops(device=None, stream=None) -> int:
    """rt_trace_static_stack_drops: pushes the last rt_trace_static call on `device` dropped on a
    full stack (read after its stream has finished)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    out = ctypes.c_uint64(0)
    with torch.cuda.device(dev):
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        st = lib().rt_trace_static_stack_drops(s, ctypes.byref(out))
    if st != 0:
        raise RtError(st, "rt_trace_static_stack_drops failed")
    return int(out.value)


# ---------------------------------------------------------------- the seam, batched

def _rays(origin, direction, tmin, tmax):
    import torch
    o = torch.as_tensor(origin, dtype=torch.float32)
    d = torch.as_tensor(direction, dtype=torch.float32)
    n = o.shape[0]
    r = torch.empty((n, 8), dtype=torch.float32, device=o.device)
    r[:, 0:3] = o
    r[:, 3] = torch.as_tensor(tmin, dtype=torch.float32, device=o.device)
    r[:, 4:7] = d
    r[:, 7] = torch.as_tensor(tmax, dtype=torch.float32, device=o.device)
    return r


def decode_gi(hits) -> dict:
    """Split (n, 10) GI hit words into named fields (torch int32 tensor or numpy)."""
    h = hits
    f = h.view(np.float32) if isinstance(h, np.ndarray) else h.view(__import__("torch").float32)
    return dict(t=f[:, 0], inst=h[:, 1], tri=h[:, 2:5], bary=f[:, 5:7], normal=f[:, 7:10])


def gi_closest(engine: Engine, scene: Scene, origin, direction, tmin, tmax, kernel="plain") -> dict:
    """gi_closest (gi_rays_software.wgsl:280-282) for a batch of rays on the device."""
    return decode_gi(engine.trace(scene, _rays(origin, direction, tmin, tmax), CLOSEST, kernel))


def gi_visible(engine: Engine, scene: Scene, origin, direction, kernel="plain"):
    """gi_visible (gi_rays_software.wgsl:285-287): sky visibility along [0, 1e20)."""
    return engine.trace(scene, _rays(origin, direction, 0.0, 1e20), ANY_SKY, kernel) == 0


def gi_visible_within(engine: Engine, scene: Scene, origin, direction, tmax, kernel="plain"):
    """gi_visible_within (gi_rays_software.wgsl:289-291): opaque casters within tmax."""
    return engine.trace(scene, _rays(origin, direction, 0.0, tmax), ANY_CASTERS, kernel) == 0


def rs_trace(engine: Engine, scene: Scene, origin, direction, tmin, tmax, any_hit=False, kernel="plain"):
    """rs_trace (reflections_software_bvh4.wgsl:140): (t, record) or the blocked flags."""
    import torch
    h = engine.trace(scene, _rays(origin, direction, tmin, tmax), ANY_CASTERS if any_hit else CLOSEST, kernel)
    if any_hit:
        return h != 0
    return h[:, 0].view(torch.float32), h[:, 1:5]


def rs_closest(engine, scene, origin, direction, tmin, tmax, kernel="plain"):
    """rs_closest (reflections_software_bvh4.wgsl:206): the hit record (slot+1, prim, u, v)."""
    return rs_trace(engine, scene, origin, direction, tmin, tmax, False, kernel)[1]


def rs_blocked(engine, scene, origin, direction, tmin, tmax, kernel="plain"):
    """rs_blocked (reflections_software_bvh4.wgsl:207)."""
    return rs_trace(engine, scene, origin, direction, tmin, tmax, True, kernel)
