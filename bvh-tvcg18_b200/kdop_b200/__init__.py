"""kdop_b200 -- Python binding of the B200 kDOP BVH collision library.

The compute path is libkdop_cuda.so (hand-written sm_100a CUDA behind the C
ABI of include/kdop_cuda.h); this package only loads it with ctypes and moves
arrays in and out.  There is no CPU fallback: importing works anywhere, but
every call that needs the library raises if it is missing or no GPU exists.
"""
from __future__ import annotations

from .lib import (KdopError, Context, DeviceScene, TraverseOpts, Stats, CONTACT_DTYPE, load_library,
                  library_path, REFIT_VERTICES, REFIT_POSE, REFIT_DEFORM, TRAVERSE_BATCHED, TRAVERSE_PLAIN,
                  HOST, DEVICE, BUILD_DEVICE, BUILD_HOST)
from . import scenes

__all__ = ["KdopError", "Context", "DeviceScene", "TraverseOpts", "Stats", "CONTACT_DTYPE", "load_library",
           "library_path", "REFIT_VERTICES", "REFIT_POSE", "REFIT_DEFORM", "TRAVERSE_BATCHED", "TRAVERSE_PLAIN",
           "HOST", "DEVICE", "BUILD_DEVICE", "BUILD_HOST", "scenes"]
