"""The read-bandwidth probe behind the benchmark's L2 and HBM ceilings (rt_read_bandwidth): a
buffer well inside L2 reads faster than one far larger than L2, both within the range a B200 can
reach, and bad arguments are refused without touching the device."""
from __future__ import annotations

import ctypes

import pytest

from renderlab_b200 import api as A

pytestmark = pytest.mark.gpu


def test_l2_reads_faster_than_hbm(engine):
    l2 = engine.read_bandwidth(48 << 20, 20)
    hbm = engine.read_bandwidth(2 << 30, 3)
    assert 1_000.0 < hbm < 10_000.0, hbm  # GB/s: HBM3e peaks near 8 TB/s
    assert l2 > 1.3 * hbm, (l2, hbm)


def test_bad_arguments_are_refused(engine):
    out = ctypes.c_double(0.0)
    assert A.lib().rt_read_bandwidth(engine.ctx, 1024, 5, ctypes.byref(out)) == 1  # under 1 MiB
    assert A.lib().rt_read_bandwidth(engine.ctx, 1 << 24, 0, ctypes.byref(out)) == 1
    assert A.lib().rt_read_bandwidth(engine.ctx, 1 << 24, 5, None) == 1
