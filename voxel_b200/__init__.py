"""VoxelVM execution backend for NVIDIA B200 (sm_100a).

The product is the native library ``voxel_b200/lib/libvoxel_c.so`` (C ABI in
``include/voxel_c.h``) and the ``voxel_py`` pybind module next to it.  This
package is the thin Python view used by tests and the benchmark.
"""
from __future__ import annotations

import os
import sys

from . import capi  # noqa: F401

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")


def voxel_py():
    """Import the pybind11 ``voxel_py`` module built next to the C ABI library."""
    if LIB_DIR not in sys.path:
        sys.path.insert(0, LIB_DIR)
    import voxel_py  # noqa: PLC0415

    return voxel_py
