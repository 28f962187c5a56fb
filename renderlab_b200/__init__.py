"""B200-native software ray traversal for renderlab's packed BVH4-Q8 geometry.

The traversal runs in ``_lib/librt_trace.so`` (CUDA, sm_100a) behind the C ABI of
``include/rt_trace.h``; ``renderlab_b200.api`` is the Python host side of that ABI.
"""
from . import api, scenes  # noqa: F401

__all__ = ["api", "scenes"]
