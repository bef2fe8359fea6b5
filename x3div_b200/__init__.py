"""x3div_b200: B200-native (sm_100a) drop-in for x3div's Euler-timestep hot path.

The compute lives in ``_lib/libx3d_b200.so`` (hand-written CUDA behind the C ABI
of ``include/x3d_b200.h``); this package is the Python face of that ABI.
"""
from .api import Batch, Context, Operator, X3DError, to_device, to_host  # noqa: F401
from .boxes import b48_boxes, box_points, shard_boxes  # noqa: F401
from .build import build  # noqa: F401

__all__ = ["Batch", "Context", "Operator", "X3DError", "to_device", "to_host", "build",
           "b48_boxes", "box_points", "shard_boxes"]
