"""The C ABI without a GPU: the library loads, exports every function include/rt_trace.h
declares, and its host-only entry points behave (version, argument errors, packing)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np

from renderlab_b200 import api as A
from renderlab_b200 import scenes as S

HEADER = Path(__file__).resolve().parents[1] / "include" / "rt_trace.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(rt_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = A.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(A.EXPORTS) | {"rt_trace_ex"}


def test_abi_version_and_null_arguments():
    lib = A.lib()
    assert lib.rt_abi_version() == 1
    assert lib.rt_ctx_create(0, None) == 1  # RT_ERR_INVALID_ARG
    assert lib.rt_blas_build(None, 0, None, 0, 0, None) == 1
    size = ctypes.c_size_t(0)
    assert lib.rt_tlas_build(None, 0, 1, None, ctypes.byref(size)) == 1
    # the device builders and the device move refuse null arguments before touching a device
    assert lib.rt_blas_build_device(None, None, 0, None, 0, 0, None) == 1
    assert lib.rt_tlas_build_device(None, None, 0, 1, None, ctypes.byref(size)) == 1
    assert lib.rt_scene_move_instances(None, None, None, 0, None, 0, None) == 1


def test_context_without_device_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    assert A.lib().rt_ctx_create(0, ctypes.byref(h)) == 6  # RT_ERR_CUDA: no device here


def test_host_builders_need_no_device():
    mesh, inst = S.cubes_instanced(8)
    w = A.pack_scene(A.LAYOUT_REFLECTION, [A.Blas(mesh.positions, mesh.indices)], inst)
    assert w[0] == 64 and w[1] != 0
    assert A.Blas(mesh.positions, mesh.indices).info()["positions"] == 8


def test_validation_rejects_unsafe_words():
    """The admission check accepts packed scenes and refuses words a traversal could follow out
    of the buffer or around a cycle."""
    from tests.test_gpu_parity import deep_chain_scene
    mesh, inst = S.cubes_instanced(8)
    for layout in (A.LAYOUT_GI, A.LAYOUT_REFLECTION):
        w = A.pack_scene(layout, [A.Blas(mesh.positions, mesh.indices)], inst)
        info = A.validate(layout, w)
        assert info["instances"] == 64 and info["triangles"] == 12 and info["top"] != 0
        rec = 16 if layout == A.LAYOUT_GI else 8
        for word, value in ((0, 1 << 24), (1, len(w) + 5), (rec + 18, len(w))):
            bad = w.copy()
            bad[word] = value
            try:
                A.validate(layout, bad)
            except A.RtError as e:
                assert e.status == 2
            else:
                raise AssertionError(f"word {word} = {value} accepted")
    deep = deep_chain_scene(24)
    assert A.validate(A.LAYOUT_REFLECTION, deep)["blas_depth"] == 24
    # a node that names itself as a child is a cycle
    cyc = deep.copy()
    node0 = 8 + 24 + 32 + 8
    cyc[node0 + 16 * 23 + 9] = 23
    try:
        A.validate(A.LAYOUT_REFLECTION, cyc)
    except A.RtError:
        pass
    else:
        raise AssertionError("cycle accepted")


def test_tuner_candidates_cover_the_grid_once():
    from renderlab_b200 import tune as T
    c = T.candidates()
    assert len(c) == len(set(c)) == ((len(T.KERNELS) - 2) * len(T.REFILLS) * len(T.ORDERS) + 1 + len(T.ORDERS)
                                     + len(T.REFILLS) * (len(T.STACKS) - 1))
    assert [x for x in c if x[0] == "plain"] == [("plain", 0, "none", "")]
    assert {x[1] for x in c if x[0] == "wide8p"} == {32}
    assert c[0][2] == "none" and c[-1][2] != "none"
    # the stack choice is WIDE8's alone, and its shared stack is tried unsorted
    assert {x[3] for x in c if x[0] == "wide8"} == set(T.STACKS) and {x[3] for x in c if x[0] != "wide8"} == {""}
    assert {x[2] for x in c if x[3] == "shared"} == {"none"}
