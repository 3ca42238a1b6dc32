"""Build recipe for the test oracle (test infrastructure, not product code).

Two libraries come out of it:

* ``oracle/_build/libvoxel_oracle.so`` - the plain-C restatement in
  ``oracle/voxel_oracle.c`` (always built; gcc only).
* ``oracle/_ref/libvoxel_ref.so`` - ``oracle/ref_driver.cpp`` compiled against
  the reference VoxelVM's own header-only sources where they lie on disk
  (``VOXEL_REFERENCE_ROOT``, default ``/root/reference``).  Only built when that
  tree is present.  One header is overridden for the build: the reference's
  ``Arena`` clamps every block to 16 MiB but hands the clamped block to larger
  requests (``include/voxel/core/arena.hpp:21,172-182``), which corrupts the
  heap for hash tables above ~0.7M rows.  The override is produced in a
  temporary directory by changing that one constant, placed ahead of the
  reference on the include path, and deleted after the compile; nothing from
  the reference tree is written into this repository.

Flags follow the reference's own benchmark build (``-O3``), with
``-march=x86-64-v3`` (``-march=native`` fails on AVX-512 hosts at
``include/voxel/simd/x86.hpp:778``) and ``-ffp-contract=off`` so no FMA changes
the summation order the oracle is compared on.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD, "libvoxel_oracle.so")
REF_SO = os.path.join(REF_OUT, "libvoxel_ref.so")


# Where the reference sources are mounted in the build container.  This recipe
# is the one place that names it; everything else asks reference_root().
DEFAULT_REFERENCE_ROOT = "/root/reference"


def reference_root() -> str:
    """$VOXEL_REFERENCE_ROOT, else the build container's mount point."""
    return os.environ.get("VOXEL_REFERENCE_ROOT", DEFAULT_REFERENCE_ROOT)


def _newer(target: str, *sources: str) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build_restatement(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "voxel_oracle.c")
    hdr = os.path.join(HERE, "voxel_oracle.h")
    if force or not _newer(ORACLE_SO, src, hdr, __file__):
        cmd = ["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
               "-fno-strict-aliasing", "-fwrapv", src, "-o", ORACLE_SO, "-lm"]
        subprocess.check_call(cmd)
    return ORACLE_SO


def build_reference(force: bool = False) -> str | None:
    root = reference_root()
    inc = os.path.join(root, "include")
    arena = os.path.join(inc, "voxel", "core", "arena.hpp")
    if not os.path.isfile(arena):
        return REF_SO if os.path.exists(REF_SO) else None
    drv = os.path.join(HERE, "ref_driver.cpp")
    if not force and _newer(REF_SO, drv, __file__):
        return REF_SO
    os.makedirs(REF_OUT, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="voxel_ref_inc_")
    try:
        with open(arena) as f:
            text = f.read()
        old = "kMaxBlockSize    = 1 << 24;"
        if old not in text:
            raise RuntimeError("reference arena.hpp changed: block-size constant not found")
        os.makedirs(os.path.join(tmp, "voxel", "core"))
        with open(os.path.join(tmp, "voxel", "core", "arena.hpp"), "w") as f:
            f.write(text.replace(old, "kMaxBlockSize    = sz(1) << 40;"))
        cmd = ["g++", "-std=c++20", "-O3", "-march=x86-64-v3", "-ffp-contract=off",
               "-fPIC", "-shared", "-pthread", "-w",
               "-I", tmp, "-I", inc, "-I", root, drv, "-o", REF_SO]
        subprocess.check_call(cmd)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return REF_SO


REF_PY_DIR = os.path.join(REF_OUT, "refpy")


def build_reference_py(force: bool = False) -> str | None:
    """The reference's own pybind module (bindings/voxel_bindings.cpp) as
    oracle/_ref/refpy/voxel_py*.so, for running the reference's Python front
    end (bindings/voxel_query.py) to make golden vectors.  A separate
    directory, so it never shadows this backend's voxel_py."""
    import sysconfig

    root = reference_root()
    src = os.path.join(root, "bindings", "voxel_bindings.cpp")
    if not os.path.isfile(src):
        return None
    try:
        import pybind11
    except ImportError:
        return None
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(REF_PY_DIR, "voxel_py" + ext)
    if not force and _newer(out, src, __file__):
        return out
    os.makedirs(REF_PY_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared", "-pthread",
           "-w", "-I", os.path.join(root, "include"), "-I", root, "-I", pybind11.get_include(),
           "-I", sysconfig.get_paths()["include"], src, "-o", out]
    subprocess.check_call(cmd)
    return out


def build(force: bool = False) -> dict:
    out = {"oracle": build_restatement(force)}
    try:
        out["reference"] = build_reference(force)
    except (subprocess.CalledProcessError, RuntimeError, OSError) as exc:  # reference unbuildable
        print(f"[oracle] reference build skipped: {exc}", file=sys.stderr)
        out["reference"] = REF_SO if os.path.exists(REF_SO) else None
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
