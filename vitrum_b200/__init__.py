"""vitrum_b200 -- B200-native ray-tracing backend for the vitrum Engine contract.

Hot path: binned-SAH BVH build, 8-wide compressed-node closest/any-hit
traversal with the watertight f32 triangle test, all in libvitrum_pt.so
(hand-written CUDA for sm_100a behind the C ABI in include/vitrum_pt.h).
"""
from ._native import VtError, lib  # noqa: F401
from .bvh import Bvh, HIT_DTYPE, build_compressed_wide_bvh  # noqa: F401

__all__ = ["Bvh", "HIT_DTYPE", "VtError", "build_compressed_wide_bvh", "lib"]
