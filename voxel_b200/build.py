"""Build recipe for the B200 backend (sm_100a only).

Produces, in-tree so the built files travel with the repository snapshot:

* ``voxel_b200/lib/libvoxel_c.so`` - the CUDA kernels, the C++ runtime and the
  C ABI declared in ``include/voxel_c.h`` (CUDA runtime linked statically).
* ``voxel_b200/lib/voxel_py*.so`` - the pybind11 module mirroring the
  reference's ``voxel_py`` classes over that C ABI.
* ``voxel_b200/lib/libvoxel_datagen.so`` - seeded synthetic column generators.

Every CUDA translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
             "-I", os.path.join(CUDA, "include")]

CORE_SOURCES = [
    "vx_runtime.cu",
    "scan.cu",
    "lower.cpp",
    "engine.cpp",
    "filter.cu",
    "decode.cu",
    "delta.cu",
    "groupby.cu",
    "radix.cu",
    "join.cu",
    "mjoin.cu",
    "window.cu",
    "ops.cu",
    "estimator.cu",
    "batch.cu",
    "serve.cpp",
    "tune.cpp",
    "capi.cpp",
]

LIB_SO = os.path.join(LIB, "libvoxel_c.so")
DATAGEN_SO = os.path.join(LIB, "libvoxel_datagen.so")


def _obj_for(src: str) -> str:
    return os.path.join(OBJ, os.path.basename(src) + ".o")


def _headers() -> list[str]:
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, hdrs: list[str], force: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = _obj_for(src)
    if force or _stale(obj, [path, __file__] + hdrs):
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", path, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    hdrs = _headers()
    srcs = [s for s in CORE_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdrs, force), srcs))
    if force or _stale(LIB_SO, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB_SO] + objs + ["-lcuda", "-lpthread"]
        subprocess.check_call(cmd)
    # pybind11 module over the C ABI
    try:
        import pybind11  # noqa: PLC0415

        ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
        py_so = os.path.join(LIB, "voxel_py" + ext)
        src = os.path.join(CSRC, "pybind_module.cpp")
        if os.path.exists(src) and (force or _stale(py_so, [src, LIB_SO] + hdrs)):
            cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC",
                   "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
                   "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                   src, "-o", py_so, "-L", LIB, "-lvoxel_c", "-Wl,-rpath,$ORIGIN"]
            subprocess.check_call(cmd)
    except ImportError:
        print("[build] pybind11 missing: voxel_py not built", file=sys.stderr)
    dsrc = os.path.join(CSRC, "datagen.cpp")
    if os.path.exists(dsrc) and (force or _stale(DATAGEN_SO, [dsrc])):
        subprocess.check_call(["g++", "-O3", "-std=c++17", "-shared", "-fPIC", dsrc, "-o", DATAGEN_SO, "-lpthread"])
    return LIB_SO


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
