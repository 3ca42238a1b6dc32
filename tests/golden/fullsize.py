"""Inputs of the full-size workloads and their reference digests.

Shared by tests/golden/make_fullsize.py (which runs the reference on them),
the full-size GPU tests and bench.py (which check their outputs against the
stored digests).  Every generator is deterministic: numpy PCG64 for the
scan + group-by columns, SplitMix64 / std::mt19937_64 / the alias-method probe
generator of the backend's C++ data generator for the rest.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if HERE not in sys.path:
    sys.path.insert(0, HERE)

FIXTURE = os.path.join(HERE, "fullsize.json")

ROWS_CONFIG2 = 1 << 25
SEED_CONFIG2 = 2001
PTHR, QLO, QHI = 20.0, 10, 50
ROWS_SORT = 1 << 28
SEED_SORT = 3001
BUILD_JOIN = 1 << 24
PROBE_JOIN = 1 << 29
SEED_JOIN_BUILD = 3002
SEED_JOIN_PROBE = 3003
ROWS_CONFIG1 = 1 << 28
SEED_CONFIG1 = 42


def load() -> dict:
    if not os.path.exists(FIXTURE):
        return {}
    with open(FIXTURE) as f:
        return json.load(f)


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(memoryview(np.ascontiguousarray(a)).cast("B"))
    return h.hexdigest()


def config2_input(n: int = ROWS_CONFIG2, seed: int = SEED_CONFIG2) -> dict:
    import inputs

    return inputs.config2(n, seed)


def sort_input(n: int = ROWS_SORT, seed: int = SEED_SORT) -> np.ndarray:
    from voxel_b200 import capi

    keys = np.empty(n, np.uint64)
    capi.datagen().vgen_splitmix64(seed, n, keys.ctypes.data)
    return keys


def join_build(nb: int = BUILD_JOIN, seed: int = SEED_JOIN_BUILD) -> np.ndarray:
    from voxel_b200 import capi

    b = np.empty(nb, np.uint64)
    capi.datagen().vgen_splitmix64(seed, nb, b.ctypes.data)
    b &= np.uint64(0xFFFFFFFFFFFFFFFE)  # build keys even, miss keys odd
    return b.view(np.int64)


def join_input(nb: int = BUILD_JOIN, npr: int = PROBE_JOIN, seed_build: int = SEED_JOIN_BUILD,
               seed_probe: int = SEED_JOIN_PROBE):
    from voxel_b200 import capi

    build = join_build(nb, seed_build)
    probe = np.empty(npr, np.int64)
    capi.datagen().vgen_join_probe_i64(seed_probe, build.ctypes.data, nb, 0.8, 0.1, npr, probe.ctypes.data,
                                       os.cpu_count() or 1)
    return build, probe


def config1_input(n: int = ROWS_CONFIG1, seed: int = SEED_CONFIG1) -> np.ndarray:
    import inputs

    return inputs.mt_uniform(seed, n)
